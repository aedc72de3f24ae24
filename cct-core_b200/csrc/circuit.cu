// Kernel circuits: a ComputeGraph's DAG of convolutions and elementwise
// operations, stepped as one CUDA graph over shared device buffers.
//
// The reference compiles a ComputeGraph into a KernelCircuit, enqueues its
// kernels in one fixed order every step (src/main/scala/cogx/runtime/
// execution/GPUSupervisor.scala:128-215) and lets fields share device
// buffers ("latches") once every kernel that reads them has run, assuming
// in-order execution (runtime/allocation/InOrderSharedLatchAllocator.scala:
// 34-243; latches binned by field size, SharedLatchesByBinnedFieldSize).
// Here the order is the node list, the buffers are assigned once at
// creation by the same in-order rule, and the step is captured into a CUDA
// graph on the first step and replayed after that.
#include <cuda_runtime.h>

#include <map>
#include <new>
#include <vector>

#include "cct_internal.h"

namespace {

struct FieldShape {
  int32_t rows, cols, planes;
  size_t elems() const { return (size_t)rows * cols * planes; }
};

FieldShape shape_of(const cct_field_shape &s) { return {s.rows, s.cols, s.planes < 1 ? 1 : s.planes}; }

// Shapes of every field (inputs, then one output per node), after checking
// that each node reads only earlier fields with the shapes it expects.
int circuit_shapes(const cct_field_shape *inputs, int32_t n_in, const cct_circuit_node *nodes, int32_t n_nodes,
                   const int32_t *outputs, int32_t n_out, std::vector<FieldShape> *shapes) {
  using cct::set_error;
  if ((n_in > 0 && !inputs) || (n_nodes > 0 && !nodes) || (n_out > 0 && !outputs))
    return set_error(CCT_EINVAL, "null argument");
  if (n_in < 0 || n_nodes < 1 || n_out < 0) return set_error(CCT_EINVAL, "a circuit needs at least one node");
  shapes->clear();
  for (int32_t i = 0; i < n_in; ++i) {
    const FieldShape s = shape_of(inputs[i]);
    if (s.rows < 1 || s.cols < 1) return set_error(CCT_EINVAL, "circuit input %d has an empty shape", i);
    shapes->push_back(s);
  }
  for (int32_t i = 0; i < n_nodes; ++i) {
    const cct_circuit_node &n = nodes[i];
    const int32_t nf = n_in + i;  // fields defined before this node
    auto field_ok = [&](int32_t f) { return f >= 0 && f < nf; };
    if (!field_ok(n.in0))
      return set_error(CCT_EINVAL, "circuit node %d reads field %d, which is not defined before it", i, n.in0);
    const FieldShape a = (*shapes)[n.in0];
    switch (n.op) {
      case CCT_NODE_CONV: {
        const cct_conv_desc &d = n.conv;
        const FieldShape want{d.image_rows, d.image_cols, d.image_planes < 1 ? 1 : d.image_planes};
        if (want.rows != a.rows || want.cols != a.cols || want.planes != a.planes)
          return set_error(CCT_EINVAL, "circuit node %d convolves a %dx%dx%d image but field %d is %dx%dx%d", i,
                           want.rows, want.cols, want.planes, n.in0, a.rows, a.cols, a.planes);
        cct::ConvGeom g;
        int rc = cct::resolve_geom(&d, &g);
        if (rc) return rc;
        if (n.in1 >= 0) {
          if (!field_ok(n.in1))
            return set_error(CCT_EINVAL, "circuit node %d reads filter field %d, which is not defined before it",
                             i, n.in1);
          const size_t need = (size_t)g.pf * g.fr * g.fs;
          if ((*shapes)[n.in1].elems() != need)
            return set_error(CCT_EINVAL, "circuit node %d needs a filter of %zu values but field %d holds %zu", i,
                             need, n.in1, (*shapes)[n.in1].elems());
        }
        shapes->push_back({g.OH, g.OW, g.pout});
        break;
      }
      case CCT_NODE_ADD:
      case CCT_NODE_SUB:
      case CCT_NODE_MUL:
        if (!field_ok(n.in1))
          return set_error(CCT_EINVAL, "circuit node %d reads field %d, which is not defined before it", i, n.in1);
        if ((*shapes)[n.in1].elems() != a.elems())
          return set_error(CCT_EINVAL, "circuit node %d combines fields of %zu and %zu values", i, a.elems(),
                           (*shapes)[n.in1].elems());
        shapes->push_back(a);
        break;
      case CCT_NODE_RELU:
      case CCT_NODE_SCALE:
        shapes->push_back(a);
        break;
      default:
        return set_error(CCT_EINVAL, "circuit node %d has unknown op %d", i, n.op);
    }
  }
  const int32_t nf = n_in + n_nodes;
  for (int32_t k = 0; k < n_out; ++k)
    if (outputs[k] < 0 || outputs[k] >= nf)
      return set_error(CCT_EINVAL, "circuit output %d names field %d (fields are 0..%d)", k, outputs[k], nf - 1);
  return CCT_OK;
}

// In-order shared-latch assignment.  Inputs and listed outputs are sealed
// (a buffer each, never shared).  Node i's output takes a free buffer of its
// size, or a new one; after node i, the buffers of the fields whose last
// reader is node i (and of an output nobody reads) are free again.  A node's
// output never shares a buffer with its own inputs: those are freed only
// after it.
int circuit_assign(int32_t n_in, const cct_circuit_node *nodes, int32_t n_nodes, const int32_t *outputs,
                   int32_t n_out, const std::vector<FieldShape> &shapes, std::vector<int32_t> *field_buffer,
                   std::vector<size_t> *buffer_elems) {
  const int32_t nf = n_in + n_nodes;
  std::vector<int32_t> last(nf, -1);
  for (int32_t i = 0; i < n_nodes; ++i) {
    last[nodes[i].in0] = i;
    if (nodes[i].in1 >= 0 && (nodes[i].op != CCT_NODE_RELU && nodes[i].op != CCT_NODE_SCALE))
      last[nodes[i].in1] = i;
  }
  std::vector<bool> sealed(nf, false);
  for (int32_t f = 0; f < n_in; ++f) sealed[f] = true;
  for (int32_t k = 0; k < n_out; ++k) sealed[outputs[k]] = true;
  field_buffer->assign(nf, -1);
  buffer_elems->clear();
  std::map<size_t, std::vector<int32_t>> free_by_size;  // binned by field size
  auto new_buffer = [&](size_t elems) {
    buffer_elems->push_back(elems);
    return (int32_t)buffer_elems->size() - 1;
  };
  for (int32_t f = 0; f < n_in; ++f) (*field_buffer)[f] = new_buffer(shapes[f].elems());
  for (int32_t i = 0; i < n_nodes; ++i) {
    const int32_t f = n_in + i;
    const size_t elems = shapes[f].elems();
    std::vector<int32_t> &pool = free_by_size[elems];
    if (!sealed[f] && !pool.empty()) {
      (*field_buffer)[f] = pool.back();
      pool.pop_back();
    } else {
      (*field_buffer)[f] = new_buffer(elems);
    }
    // fields whose last reader has now run give their buffers back
    auto release = [&](int32_t g) {
      if (g >= 0 && !sealed[g] && last[g] == i) {
        free_by_size[shapes[g].elems()].push_back((*field_buffer)[g]);
        last[g] = -2;  // released once
      }
    };
    release(nodes[i].in0);
    if (nodes[i].op != CCT_NODE_RELU && nodes[i].op != CCT_NODE_SCALE) release(nodes[i].in1);
    if (!sealed[f] && last[f] == -1) free_by_size[elems].push_back((*field_buffer)[f]);  // nobody reads it
  }
  return CCT_OK;
}

// Elementwise node: y = a op b, max(a, 0) or a * scalar, grid-stride, four
// values per thread where the buffers allow.
__global__ void circuit_elementwise(int op, const float *__restrict__ a, const float *__restrict__ b, float scalar,
                                    float *__restrict__ y, size_t n) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  auto apply = [&](float x, float z) {
    switch (op) {
      case CCT_NODE_ADD: return x + z;
      case CCT_NODE_SUB: return x - z;
      case CCT_NODE_MUL: return x * z;
      case CCT_NODE_RELU: return fmaxf(x, 0.0f);
      default: return x * scalar;
    }
  };
  const bool binary = op == CCT_NODE_ADD || op == CCT_NODE_SUB || op == CCT_NODE_MUL;
  const bool vec = (n % 4 == 0) && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(y) |
                                     (binary ? reinterpret_cast<uintptr_t>(b) : 0)) & 15) == 0;
  if (vec) {
    const size_t n4 = n / 4;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
      const float4 x = reinterpret_cast<const float4 *>(a)[i];
      const float4 z = binary ? reinterpret_cast<const float4 *>(b)[i] : make_float4(0, 0, 0, 0);
      reinterpret_cast<float4 *>(y)[i] = make_float4(apply(x.x, z.x), apply(x.y, z.y), apply(x.z, z.z), apply(x.w, z.w));
    }
  } else {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      y[i] = apply(a[i], binary ? b[i] : 0.0f);
  }
}

}  // namespace

struct cct_circuit {
  int device = 0;
  int32_t n_in = 0;
  std::vector<cct_circuit_node> nodes;
  std::vector<FieldShape> shapes;      // per field
  std::vector<int32_t> field_buffer;   // per field
  std::vector<float *> buffers;
  std::vector<size_t> buffer_elems;
  std::vector<int32_t> outputs;
  std::vector<cct_conv_plan *> plans;  // per node; null for elementwise nodes
  std::vector<bool> has_filter;        // per node: a static filter is set (or none is needed)
  cudaStream_t capture = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0;
  int64_t time = 0;
};

namespace {

float *field_ptr(const cct_circuit *c, int32_t f) { return c->buffers[c->field_buffer[f]]; }

void release(cct_circuit *c) {
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  if (c->capture) cudaStreamDestroy(c->capture);
  for (cct_conv_plan *p : c->plans)
    if (p) cct_conv_plan_destroy(p);
  for (float *b : c->buffers) cudaFree(b);
  delete c;
}

int run_node(const cct_circuit *c, int32_t i, cudaStream_t st) {
  const cct_circuit_node &n = c->nodes[i];
  float *y = field_ptr(c, c->n_in + i);
  if (n.op == CCT_NODE_CONV)
    return cct_conv_run(c->plans[i], field_ptr(c, n.in0), n.in1 >= 0 ? field_ptr(c, n.in1) : nullptr, y, st);
  const bool binary = n.op == CCT_NODE_ADD || n.op == CCT_NODE_SUB || n.op == CCT_NODE_MUL;
  const size_t elems = c->shapes[c->n_in + i].elems();
  const int blocks = (int)std::min<size_t>((elems / 4 + 255) / 256 + 1, 148 * 8);
  circuit_elementwise<<<blocks, 256, 0, st>>>(n.op, field_ptr(c, n.in0), binary ? field_ptr(c, n.in1) : nullptr,
                                               n.scalar, y, elems);
  cct::count_launches(1);
  return cct::check_cuda(cudaGetLastError(), "circuit elementwise launch");
}

int capture(cct_circuit *c) {
  for (size_t i = 0; i < c->nodes.size(); ++i)
    if (!c->has_filter[i]) return cct::set_error(CCT_EINVAL, "circuit node %zu has no filter", i);
  // one eager pass validates every node and leaves kernel attributes set,
  // so nothing but launches happens during capture
  for (int32_t i = 0; i < (int32_t)c->nodes.size(); ++i) {
    int rc = run_node(c, i, c->capture);
    if (rc) return rc;
  }
  int rc = cct::check_cuda(cudaStreamSynchronize(c->capture), "circuit warm-up pass");
  if (rc) return rc;
  rc = cct::check_cuda(cudaStreamBeginCapture(c->capture, cudaStreamCaptureModeThreadLocal),
                       "cudaStreamBeginCapture");
  if (rc) return rc;
  cct::set_launch_capture(true);
  int run_rc = CCT_OK;
  for (int32_t i = 0; i < (int32_t)c->nodes.size() && !run_rc; ++i) run_rc = run_node(c, i, c->capture);
  cct::set_launch_capture(false);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(c->capture, &graph);
  if (run_rc) {
    if (graph) cudaGraphDestroy(graph);
    return run_rc;
  }
  rc = cct::check_cuda(end, "cudaStreamEndCapture");
  if (rc) return rc;
  size_t n = 0;
  cudaGraphGetNodes(graph, nullptr, &n);
  std::vector<cudaGraphNode_t> gnodes(n);
  if (n) cudaGraphGetNodes(graph, gnodes.data(), &n);
  uint64_t kernels = 0;
  for (cudaGraphNode_t node : gnodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(node, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
  }
  cudaGraphExec_t exec = nullptr;
  rc = cct::check_cuda(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
  if (rc) {
    cudaGraphDestroy(graph);
    return rc;
  }
  c->graph = graph;
  c->exec = exec;
  c->kernels = kernels;
  return CCT_OK;
}

}  // namespace

extern "C" {

int cct_circuit_assign(const cct_field_shape *inputs, int32_t n_inputs, const cct_circuit_node *nodes,
                       int32_t n_nodes, const int32_t *outputs, int32_t n_outputs, int32_t *field_buffer,
                       int32_t *n_buffers) {
  if (!field_buffer || !n_buffers) return cct::set_error(CCT_EINVAL, "null argument");
  std::vector<FieldShape> shapes;
  int rc = circuit_shapes(inputs, n_inputs, nodes, n_nodes, outputs, n_outputs, &shapes);
  if (rc) return rc;
  std::vector<int32_t> fb;
  std::vector<size_t> be;
  rc = circuit_assign(n_inputs, nodes, n_nodes, outputs, n_outputs, shapes, &fb, &be);
  if (rc) return rc;
  for (size_t f = 0; f < fb.size(); ++f) field_buffer[f] = fb[f];
  *n_buffers = (int32_t)be.size();
  return CCT_OK;
}

int cct_circuit_create(const cct_field_shape *inputs, int32_t n_inputs, const cct_circuit_node *nodes,
                       int32_t n_nodes, const int32_t *outputs, int32_t n_outputs, cct_circuit **out) {
  if (!out) return cct::set_error(CCT_EINVAL, "null circuit output");
  *out = nullptr;
  std::vector<FieldShape> shapes;
  int rc = circuit_shapes(inputs, n_inputs, nodes, n_nodes, outputs, n_outputs, &shapes);
  if (rc) return rc;
  cct_circuit *c = new (std::nothrow) cct_circuit;
  if (!c) return cct::set_error(CCT_ENOMEM, "out of host memory");
  c->n_in = n_inputs;
  c->nodes.assign(nodes, nodes + n_nodes);
  c->outputs.assign(outputs, outputs + n_outputs);
  c->shapes = shapes;
  rc = circuit_assign(n_inputs, nodes, n_nodes, outputs, n_outputs, shapes, &c->field_buffer, &c->buffer_elems);
  if (!rc) rc = cct::check_cuda(cudaGetDevice(&c->device), "cudaGetDevice");
  for (int32_t i = 0; i < n_nodes && !rc; ++i) {
    cct_conv_plan *p = nullptr;
    if (nodes[i].op == CCT_NODE_CONV) {
      rc = cct_conv_plan_create(&nodes[i].conv, &p);
      if (rc) break;
    }
    c->plans.push_back(p);
    c->has_filter.push_back(nodes[i].op != CCT_NODE_CONV || nodes[i].in1 >= 0);
  }
  for (size_t b = 0; !rc && b < c->buffer_elems.size(); ++b) {
    float *ptr = nullptr;
    rc = cct::check_cuda(cudaMalloc(&ptr, c->buffer_elems[b] * sizeof(float)), "cudaMalloc(circuit buffer)");
    if (!rc) {
      c->buffers.push_back(ptr);
      rc = cct::check_cuda(cudaMemset(ptr, 0, c->buffer_elems[b] * sizeof(float)), "cudaMemset(circuit buffer)");
    }
  }
  if (!rc)
    rc = cct::check_cuda(cudaStreamCreateWithFlags(&c->capture, cudaStreamNonBlocking), "cudaStreamCreate(circuit)");
  if (rc) {
    release(c);
    return rc;
  }
  *out = c;
  return CCT_OK;
}

int cct_circuit_destroy(cct_circuit *c) {
  if (!c) return CCT_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaSetDevice(c->device);
  release(c);
  cudaSetDevice(dev);
  return CCT_OK;
}

int cct_circuit_set_filter(cct_circuit *c, int32_t node, const float *host_filter) {
  if (!c || !host_filter) return cct::set_error(CCT_EINVAL, "null argument");
  if (node < 0 || node >= (int32_t)c->nodes.size() || c->nodes[node].op != CCT_NODE_CONV ||
      c->nodes[node].in1 >= 0)
    return cct::set_error(CCT_EINVAL, "circuit node %d is not a convolution with a static filter", node);
  // the static filter buffer keeps its address, so a captured step stays valid
  int rc = cct_conv_plan_set_static_filter(c->plans[node], host_filter);
  if (rc) return rc;
  c->has_filter[node] = true;
  return CCT_OK;
}

int cct_circuit_field(const cct_circuit *c, int32_t field, float **device_ptr, size_t *elems) {
  if (!c || !device_ptr) return cct::set_error(CCT_EINVAL, "null argument");
  if (field < 0 || field >= (int32_t)c->field_buffer.size())
    return cct::set_error(CCT_EINVAL, "circuit has no field %d (fields are 0..%zu)", field,
                          c->field_buffer.size() - 1);
  *device_ptr = field_ptr(c, field);
  if (elems) *elems = c->shapes[field].elems();
  return CCT_OK;
}

int cct_circuit_buffers(const cct_circuit *c, int32_t *n_buffers, size_t *bytes) {
  if (!c) return cct::set_error(CCT_EINVAL, "null circuit");
  size_t total = 0;
  for (size_t e : c->buffer_elems) total += e * sizeof(float);
  if (n_buffers) *n_buffers = (int32_t)c->buffers.size();
  if (bytes) *bytes = total;
  return CCT_OK;
}

int cct_circuit_step(cct_circuit *c, int64_t count, void *stream) {
  if (!c) return cct::set_error(CCT_EINVAL, "null circuit");
  if (count < 0) return cct::set_error(CCT_EINVAL, "Negative step count seen: %lld", (long long)count);
  if (!c->exec) {
    int rc = capture(c);
    if (rc) return rc;
  }
  cudaStream_t st = (cudaStream_t)stream;
  for (int64_t i = 0; i < count; ++i) {
    int rc = cct::check_cuda(cudaGraphLaunch(c->exec, st), "cudaGraphLaunch");
    if (rc) return rc;
    cct::count_launches(c->kernels);
    ++c->time;
  }
  return CCT_OK;
}

int cct_circuit_step_host(cct_circuit *c, const float *const *host_inputs, float *const *host_outputs,
                          void *stream) {
  if (!c || (c->n_in > 0 && !host_inputs) || (!c->outputs.empty() && !host_outputs))
    return cct::set_error(CCT_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = CCT_OK;
  for (int32_t f = 0; f < c->n_in && !rc; ++f) {
    if (!host_inputs[f]) return cct::set_error(CCT_EINVAL, "circuit input %d has no host buffer", f);
    rc = cct::check_cuda(cudaMemcpyAsync(field_ptr(c, f), host_inputs[f], c->shapes[f].elems() * sizeof(float),
                                         cudaMemcpyHostToDevice, st),
                         "H2D circuit input");
  }
  if (!rc) rc = cct_circuit_step(c, 1, stream);
  for (size_t k = 0; k < c->outputs.size() && !rc; ++k) {
    if (!host_outputs[k]) return cct::set_error(CCT_EINVAL, "circuit output %zu has no host buffer", k);
    const int32_t f = c->outputs[k];
    rc = cct::check_cuda(cudaMemcpyAsync(host_outputs[k], field_ptr(c, f), c->shapes[f].elems() * sizeof(float),
                                         cudaMemcpyDeviceToHost, st),
                         "D2H circuit output");
  }
  if (!rc) rc = cct::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return rc;
}

int64_t cct_circuit_time(const cct_circuit *c) { return c ? c->time : -1; }

int cct_circuit_reset(cct_circuit *c) {
  if (!c) return cct::set_error(CCT_EINVAL, "null circuit");
  c->time = 0;
  return CCT_OK;
}

}  // extern "C"
