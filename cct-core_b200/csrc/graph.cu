// Stacked convolution graphs: a chain of convolution plans whose launches
// are captured once into a CUDA graph and replayed every step.
//
// The reference builds a ComputeGraph of fields and steps it through an
// evaluator that dispatches one OpenCL kernel per (merged) HyperKernel
// (src/main/scala/cogx/runtime/ComputeGraph.scala:56, 228-279).  For a graph
// whose fields are a stack of convolutions (the CNN layer stack) the launch
// sequence never changes between steps, so it is captured once: a step is one
// cudaGraphLaunch, with every field resident in graph-owned device buffers.
#include <cuda_runtime.h>

#include <new>
#include <string>
#include <vector>

#include "cct_internal.h"

struct cct_graph {
  int device = 0;
  std::vector<cct_conv_desc> desc;
  std::vector<cct_conv_plan *> plans;
  std::vector<float *> fields;      // 0: input; i: layer i's output
  std::vector<size_t> elems;
  std::vector<bool> has_filter;
  cudaStream_t capture = nullptr;   // private stream the sequence is captured on
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0;             // kernel nodes per replay
  int64_t time = 0;
};

namespace {

void release(cct_graph *g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->capture) cudaStreamDestroy(g->capture);
  for (cct_conv_plan *p : g->plans) cct_conv_plan_destroy(p);
  for (float *f : g->fields) cudaFree(f);
  delete g;
}

int capture(cct_graph *g) {
  for (size_t i = 0; i < g->plans.size(); ++i)
    if (!g->has_filter[i]) return cct::set_error(CCT_EINVAL, "graph layer %zu has no filter", i + 1);
  // one eager pass first: it validates every layer and leaves the kernels'
  // attributes set, so nothing but launches happens during capture
  for (size_t i = 0; i < g->plans.size(); ++i) {
    int rc = cct_conv_run(g->plans[i], g->fields[i], nullptr, g->fields[i + 1], g->capture);
    if (rc) return rc;
  }
  int rc = cct::check_cuda(cudaStreamSynchronize(g->capture), "graph warm-up pass");
  if (rc) return rc;
  rc = cct::check_cuda(cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal),
                       "cudaStreamBeginCapture");
  if (rc) return rc;
  cct::set_launch_capture(true);
  int run_rc = CCT_OK;
  for (size_t i = 0; i < g->plans.size() && !run_rc; ++i)
    run_rc = cct_conv_run(g->plans[i], g->fields[i], nullptr, g->fields[i + 1], g->capture);
  cct::set_launch_capture(false);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(g->capture, &graph);
  if (run_rc) {
    if (graph) cudaGraphDestroy(graph);
    return run_rc;
  }
  rc = cct::check_cuda(end, "cudaStreamEndCapture");
  if (rc) return rc;
  size_t n = 0;
  cudaGraphGetNodes(graph, nullptr, &n);
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) cudaGraphGetNodes(graph, nodes.data(), &n);
  uint64_t kernels = 0;
  for (cudaGraphNode_t node : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(node, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
  }
  cudaGraphExec_t exec = nullptr;
  rc = cct::check_cuda(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
  if (rc) {
    cudaGraphDestroy(graph);
    return rc;
  }
  g->graph = graph;
  g->exec = exec;
  g->kernels = kernels;
  return CCT_OK;
}

}  // namespace

extern "C" {

int cct_graph_create(const cct_conv_desc *layers, int32_t n_layers, cct_graph **out) {
  if (!layers || !out) return cct::set_error(CCT_EINVAL, "null argument");
  *out = nullptr;
  if (n_layers < 1) return cct::set_error(CCT_EINVAL, "a graph needs at least one layer");
  cct_graph *g = new (std::nothrow) cct_graph;
  if (!g) return cct::set_error(CCT_ENOMEM, "out of host memory");
  int rc = cct::check_cuda(cudaGetDevice(&g->device), "cudaGetDevice");
  int32_t prow = 0, pcol = 0, pplanes = 0;
  for (int32_t i = 0; i < n_layers && !rc; ++i) {
    const cct_conv_desc &d = layers[i];
    int32_t r, c, pl;
    rc = cct_conv_output_shape(&d, &r, &c, &pl);
    if (rc) break;
    if (i > 0 && (d.image_rows != prow || d.image_cols != pcol ||
                  (d.image_planes < 1 ? 1 : d.image_planes) != (pplanes < 1 ? 1 : pplanes))) {
      rc = cct::set_error(CCT_EINVAL,
                          "graph layer %d reads a %dx%dx%d field but layer %d writes %dx%dx%d", i + 1,
                          d.image_rows, d.image_cols, d.image_planes, i, prow, pcol, pplanes);
      break;
    }
    if (i == 0) {
      const size_t in = (size_t)d.image_rows * d.image_cols * (d.image_planes < 1 ? 1 : d.image_planes);
      g->elems.push_back(in);
    }
    g->elems.push_back((size_t)r * c * (pl < 1 ? 1 : pl));
    cct_conv_plan *p = nullptr;
    rc = cct_conv_plan_create(&d, &p);
    if (rc) break;
    g->plans.push_back(p);
    g->desc.push_back(d);
    g->has_filter.push_back(false);
    prow = r;
    pcol = c;
    pplanes = pl;
  }
  for (size_t i = 0; !rc && i < g->elems.size(); ++i) {
    float *f = nullptr;
    rc = cct::check_cuda(cudaMalloc(&f, g->elems[i] * sizeof(float)), "cudaMalloc(graph field)");
    if (!rc) {
      g->fields.push_back(f);
      rc = cct::check_cuda(cudaMemset(f, 0, g->elems[i] * sizeof(float)), "cudaMemset(graph field)");
    }
  }
  if (!rc)
    rc = cct::check_cuda(cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking),
                         "cudaStreamCreate(graph)");
  if (rc) {
    release(g);
    return rc;
  }
  *out = g;
  return CCT_OK;
}

int cct_graph_destroy(cct_graph *g) {
  if (!g) return CCT_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaSetDevice(g->device);
  release(g);
  cudaSetDevice(dev);
  return CCT_OK;
}

int cct_graph_set_filter(cct_graph *g, int32_t layer, const float *host_filter) {
  if (!g || !host_filter) return cct::set_error(CCT_EINVAL, "null argument");
  if (layer < 1 || layer > (int32_t)g->plans.size())
    return cct::set_error(CCT_EINVAL, "graph has no layer %d (layers are 1..%zu)", layer, g->plans.size());
  // the static filter buffers keep their addresses, so a captured graph
  // stays valid and reads the new filter
  int rc = cct_conv_plan_set_static_filter(g->plans[layer - 1], host_filter);
  if (rc) return rc;
  g->has_filter[layer - 1] = true;
  return CCT_OK;
}

int cct_graph_field(const cct_graph *g, int32_t index, float **device_ptr, size_t *elems) {
  if (!g || !device_ptr) return cct::set_error(CCT_EINVAL, "null argument");
  if (index < 0 || index >= (int32_t)g->fields.size())
    return cct::set_error(CCT_EINVAL, "graph has no field %d (fields are 0..%zu)", index, g->fields.size() - 1);
  *device_ptr = g->fields[index];
  if (elems) *elems = g->elems[index];
  return CCT_OK;
}

int cct_graph_step(cct_graph *g, int64_t count, void *stream) {
  if (!g) return cct::set_error(CCT_EINVAL, "null graph");
  if (count < 0) return cct::set_error(CCT_EINVAL, "Negative step count seen: %lld", (long long)count);
  if (!g->exec) {
    int rc = capture(g);
    if (rc) return rc;
  }
  cudaStream_t st = (cudaStream_t)stream;
  for (int64_t i = 0; i < count; ++i) {
    int rc = cct::check_cuda(cudaGraphLaunch(g->exec, st), "cudaGraphLaunch");
    if (rc) return rc;
    cct::count_launches(g->kernels);
    ++g->time;
  }
  return CCT_OK;
}

int cct_graph_step_host(cct_graph *g, const float *host_in, float *host_out, void *stream) {
  if (!g || !host_in || !host_out) return cct::set_error(CCT_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = cct::check_cuda(cudaMemcpyAsync(g->fields.front(), host_in, g->elems.front() * sizeof(float),
                                           cudaMemcpyHostToDevice, st),
                           "H2D graph input");
  if (!rc) rc = cct_graph_step(g, 1, stream);
  if (!rc)
    rc = cct::check_cuda(cudaMemcpyAsync(host_out, g->fields.back(), g->elems.back() * sizeof(float),
                                         cudaMemcpyDeviceToHost, st),
                         "D2H graph output");
  if (!rc) rc = cct::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return rc;
}

int64_t cct_graph_time(const cct_graph *g) { return g ? g->time : -1; }

int cct_graph_save(const cct_graph *g, uint32_t *words, size_t capacity, size_t *n_words) {
  if (!g) return cct::set_error(CCT_EINVAL, "null graph");
  std::vector<cct::RecordLayer> layers(g->plans.size());
  for (size_t i = 0; i < g->plans.size(); ++i) {
    int rc = cct::record_plan_layer(g->plans[i], &layers[i]);
    if (rc) return rc;
    layers[i].desc = g->desc[i];
  }
  std::vector<uint32_t> w;
  cct::record_encode(2, g->time, layers, &w);
  return cct::record_store(w, words, capacity, n_words);
}

int cct_graph_restore(const uint32_t *words, size_t n_words, cct_graph **out) {
  if (!out) return cct::set_error(CCT_EINVAL, "null graph output");
  *out = nullptr;
  int kind = 0;
  int64_t time = 0;
  std::vector<cct::RecordLayer> layers;
  int rc = cct::record_decode(words, n_words, &kind, &time, &layers);
  if (rc) return rc;
  if (kind != 2) return cct::set_error(CCT_EINVAL, "the record holds a plan, not a graph");
  std::vector<cct_conv_desc> descs;
  for (const cct::RecordLayer &l : layers) descs.push_back(l.desc);
  cct_graph *g = nullptr;
  rc = cct_graph_create(descs.data(), (int32_t)descs.size(), &g);
  if (rc) return rc;
  for (size_t i = 0; !rc && i < layers.size(); ++i) {
    if (layers[i].filter.empty()) continue;
    size_t need = 0;
    rc = cct::plan_filter_elems(g->plans[i], &need);
    if (!rc && need != layers[i].filter.size())
      rc = cct::set_error(CCT_EINVAL, "record layer %zu filter has %zu values, the layer needs %zu", i + 1,
                          layers[i].filter.size(), need);
    if (!rc) rc = cct_graph_set_filter(g, (int32_t)i + 1, layers[i].filter.data());
  }
  if (rc) {
    cct_graph_destroy(g);
    return rc;
  }
  g->time = time;
  *out = g;
  return CCT_OK;
}

int cct_graph_reset(cct_graph *g) {
  if (!g) return cct::set_error(CCT_EINVAL, "null graph");
  g->time = 0;
  return CCT_OK;
}

}  // extern "C"
