// Request serving with continuous batching.
//
// A scheduler thread per server admits requests as device memory for their
// fields can be had from free HBM, copies their inputs in, and packs the
// admitted ones into one
// persistent launch per slot: `serve_batch_kernel` CTAs pull (request,
// output plane, tile) work units from an atomic counter until the batch is
// done, so requests of uneven sizes share one launch.  Each slot's launch
// (table upload, counter reset, kernel) is a captured CUDA graph; up to
// `slots` launches are in flight on separate streams.  Completion is
// signalled by a host function queued after each slot's output copies.
//
// Every route keeps the reference's per-output FP32 order (fma chain per
// filter row from 0, row sums added in order, per-plane sums added in order:
// ConvolveHyperKernel.scala:509-521, 593-603), so a request's result does
// not depend on which route or batch it ran in.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cct_internal.h"

namespace cct {
namespace {

constexpr int kMaxItems = 256;
constexpr int kThreads = 256;
constexpr int kTileW = 32;
constexpr int kMaxR = 9;
constexpr int kHaloMax = (32 + kMaxR - 1) * (kTileW + kMaxR - 1);

struct Item {
  const float *x, *f;
  float *y;
  int H, W, C, K, R;  // K: output planes; C: input planes (mode 1 sums over them)
  int mode;           // 0 plane by plane, 1 frame with block reduce
  int conv;           // 1 convolution (flipped filter), 0 cross-correlation
  int fplanes;        // mode 0: 1 (shared filter) or C
  int relu;
  int th;             // tile rows (8, 16 or 32); tiles are th x 32
  int tiles_x, tiles_y;
  long long first;    // first work unit of this item
};

struct Batch {
  int n;
  int pad;
  long long total;
  Item items[kMaxItems];
};

// One th x 32 output tile of output plane o: each thread owns column tx and
// rows ty, ty + 8, ...  The halo of every input plane is staged in shared
// memory with the zero border applied, then the taps run in the reference's
// order.
template <int R, int TH>
__device__ void tile_unit(const Item &it, int o, int ty0, int tx0, float *halo, float *w) {
  constexpr int HC = kTileW + R - 1, HR = TH + R - 1, h = (R - 1) / 2, NO = TH / 8;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int terms = it.mode == 0 ? 1 : it.C;
  float acc[NO];
#pragma unroll
  for (int j = 0; j < NO; ++j) acc[j] = 0.0f;
  const size_t page = (size_t)it.H * it.W;
  for (int t = 0; t < terms; ++t) {
    int ip, fp;
    if (it.mode == 0) {
      ip = o;
      fp = it.fplanes == 1 ? 0 : o;
    } else {
      ip = t;
      fp = o * it.C + t;
    }
    const float *xp = it.x + (size_t)ip * page;
    const float *fpp = it.f + (size_t)fp * R * R;
    for (int i = tid; i < HR * HC; i += kThreads) {
      const int r = i / HC, c = i - r * HC;
      const int gr = ty0 - h + r, gc = tx0 - h + c;
      halo[i] = (gr >= 0 && gr < it.H && gc >= 0 && gc < it.W) ? __ldg(xp + (size_t)gr * it.W + gc) : 0.0f;
    }
    if (tid < R * R) w[tid] = __ldg(fpp + (it.conv ? R * R - 1 - tid : tid));
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NO; ++j) {
      const float *hp = halo + (ty + 8 * j) * HC + tx;
      float rowSum = 0.0f;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        float colSum = 0.0f;
#pragma unroll
        for (int s = 0; s < R; ++s) colSum = __fmaf_rn(hp[r * HC + s], w[r * R + s], colSum);
        rowSum = __fadd_rn(rowSum, colSum);
      }
      acc[j] = terms == 1 ? rowSum : __fadd_rn(acc[j], rowSum);
    }
    __syncthreads();
  }
  float *yp = it.y + (size_t)o * page;
  const int col = tx0 + tx;
#pragma unroll
  for (int j = 0; j < NO; ++j) {
    const int row = ty0 + ty + 8 * j;
    if (row < it.H && col < it.W) yp[(size_t)row * it.W + col] = it.relu ? fmaxf(acc[j], 0.0f) : acc[j];
  }
}

template <int R>
__device__ void dispatch_th(const Item &it, int o, int ty0, int tx0, float *halo, float *w) {
  switch (it.th) {
    case 8: tile_unit<R, 8>(it, o, ty0, tx0, halo, w); break;
    case 16: tile_unit<R, 16>(it, o, ty0, tx0, halo, w); break;
    default: tile_unit<R, 32>(it, o, ty0, tx0, halo, w); break;
  }
}

__global__ void __launch_bounds__(kThreads) serve_batch_kernel(const Batch *__restrict__ b,
                                                               unsigned long long *counter) {
  __shared__ float halo[kHaloMax];
  __shared__ float w[kMaxR * kMaxR];
  __shared__ long long unit_s;
  const long long total = b->total;
  const int n = b->n;
  for (;;) {
    if (threadIdx.x == 0) unit_s = (long long)atomicAdd(counter, 1ULL);
    __syncthreads();
    const long long u = unit_s;
    __syncthreads();
    if (u >= total) break;
    // the item holding unit u: the last one whose first unit is <= u
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (b->items[mid].first <= u) lo = mid;
      else hi = mid - 1;
    }
    const Item &it = b->items[lo];
    long long rest = u - it.first;
    const int per_plane = it.tiles_x * it.tiles_y;
    const int o = (int)(rest / per_plane);
    const int tile = (int)(rest - (long long)o * per_plane);
    const int ty0 = (tile / it.tiles_x) * it.th, tx0 = (tile % it.tiles_x) * kTileW;
    switch (it.R) {
      case 1: dispatch_th<1>(it, o, ty0, tx0, halo, w); break;
      case 3: dispatch_th<3>(it, o, ty0, tx0, halo, w); break;
      case 5: dispatch_th<5>(it, o, ty0, tx0, halo, w); break;
      case 7: dispatch_th<7>(it, o, ty0, tx0, halo, w); break;
      default: dispatch_th<9>(it, o, ty0, tx0, halo, w); break;
    }
  }
}

using Clock = std::chrono::steady_clock;

// Device memory for admitted requests, claimed from free HBM in chunks.  A
// request is admitted when a chunk has room for its fields (first fit,
// 256-byte aligned blocks), or when the device's free memory, less the
// reserve left for other work, can hold a new chunk for it.  With a cap, the
// chunks together never exceed it.  Chunks are kept until the server is
// destroyed: cudaFree synchronises the device, which the scheduler must not
// do while launches are in flight.
class Pool {
 public:
  void init(size_t cap, size_t reserve, size_t chunk) {
    cap_ = cap;
    reserve_ = reserve;
    chunk_ = chunk;
  }
  ~Pool() {
    for (auto &c : chunks_) cudaFree(c.base);
  }
  // Largest request the server can ever hold: the cap, or the device's
  // total memory less the reserve.
  size_t capacity() const {
    if (cap_) return cap_;
    size_t fr = 0, total = 0;
    if (cudaMemGetInfo(&fr, &total) != cudaSuccess) return 0;
    return total > reserve_ ? total - reserve_ : 0;
  }
  // A block of `bytes`, or nullptr when there is no room now.
  char *alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto &c : chunks_) {
      char *p = take(c, bytes);
      if (p) return p;
    }
    size_t size = std::max(bytes, chunk_);
    if (cap_) {
      if (held_ + bytes > cap_) return nullptr;
      size = std::min(size, cap_ - held_);
    }
    size_t fr = 0, total = 0;
    if (cudaMemGetInfo(&fr, &total) != cudaSuccess) return nullptr;
    if (fr < reserve_ + bytes) return nullptr;
    size = std::min(size, fr - reserve_);
    size = (size + 255) & ~(size_t)255;
    Chunk c;
    if (cudaMalloc(&c.base, size) != cudaSuccess) {
      cudaGetLastError();  // out of memory now: wait for releases
      return nullptr;
    }
    c.cap = size;
    c.free[0] = size;
    held_ += size;
    chunks_.push_back(std::move(c));
    return take(chunks_.back(), bytes);
  }
  void release(char *p, size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto &c : chunks_) {
      if (p < c.base || p >= c.base + c.cap) continue;
      used_ -= bytes;
      auto it = c.free.emplace((size_t)(p - c.base), bytes).first;
      auto next = std::next(it);
      if (next != c.free.end() && it->first + it->second == next->first) {
        it->second += next->second;
        c.free.erase(next);
      }
      if (it != c.free.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
          prev->second += it->second;
          c.free.erase(it);
        }
      }
      return;
    }
  }
  size_t peak() const { return peak_; }

 private:
  struct Chunk {
    char *base = nullptr;
    size_t cap = 0;
    std::map<size_t, size_t> free;  // offset -> bytes
  };
  char *take(Chunk &c, size_t bytes) {
    for (auto it = c.free.begin(); it != c.free.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, rem = it->second - bytes;
      c.free.erase(it);
      if (rem) c.free[off + bytes] = rem;
      used_ += bytes;
      peak_ = std::max(peak_, used_);
      return c.base + off;
    }
    return nullptr;
  }
  std::vector<Chunk> chunks_;
  size_t cap_ = 0, reserve_ = 0, chunk_ = 0, held_ = 0, used_ = 0, peak_ = 0;
};

struct Req {
  uint64_t ticket = 0;
  cct_serve_request r{};
  ConvGeom g{};
  bool batchable = false;
  size_t x_elems = 0, f_elems = 0, y_elems = 0;
  char *dev = nullptr;  // device block: x, then f (host filters), then y
  size_t bytes = 0;
  size_t off_f = 0, off_y = 0;  // offsets of f and y inside the block (256-byte aligned)
  Clock::time_point t_submit;
  double latency_us = 0.0;
  int status = CCT_OK;
  std::string msg;  // the scheduler thread's error text, for the waiting thread
  bool done = false;
  double flops = 0.0;
};
using ReqPtr = std::shared_ptr<Req>;

struct Slot {
  cudaStream_t st = nullptr;
  Batch *h_table = nullptr;  // pinned
  Batch *d_table = nullptr;
  unsigned long long *d_counter = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<ReqPtr> reqs;
  std::vector<cct_graph *> graphs;
  std::atomic<bool> finished{false};
  Clock::time_point t_done;
  bool busy = false;
  void *owner = nullptr;
};

}  // namespace
}  // namespace cct

using namespace cct;

struct cct_server {
  cct_server_config cfg{};
  int device = 0;
  int grid = 0;
  Pool pool;
  std::vector<std::unique_ptr<Slot>> slots;
  std::vector<float *> filters;
  std::vector<size_t> filter_elems;
  int tile_rows[kMaxR + 1] = {32, 32, 32, 32, 32, 32, 32, 32, 32, 32};
  double solo_flops = 1e30;  // requests at least this large run on their own kernel

  std::mutex m;
  std::condition_variable cv;       // scheduler wake-ups
  std::condition_variable done_cv;  // waiters
  std::deque<ReqPtr> incoming;      // submitted, not yet seen by the scheduler
  std::unordered_map<uint64_t, ReqPtr> table;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread worker;

  // scheduler-only state
  std::deque<ReqPtr> waiting;   // not yet admitted (arrival order)
  std::deque<ReqPtr> admitted;  // holding device memory, not yet launched
  std::set<cct_graph *> busy_graphs;

  std::atomic<uint64_t> completed{0}, batches{0}, solo{0};
};

namespace {

void host_done(void *arg) {
  Slot *s = static_cast<Slot *>(arg);
  s->t_done = Clock::now();
  s->finished.store(true, std::memory_order_release);
  cct_server *srv = static_cast<cct_server *>(s->owner);
  std::lock_guard<std::mutex> lk(srv->m);
  srv->cv.notify_all();
}

// The direct or frame kernel a request runs on when it is not batched.
int launch_solo(cct_server *s, Req &q, const float *x, const float *f, float *y, cudaStream_t st) {
  if (q.r.kind == CCT_SERVE_GRAPH_STEP) return cct_graph_step(q.r.graph, 1, st);
  if (frame_f32_supported(q.g)) return launch_frame_f32(q.g, x, f, y, st);
  if (direct_tma_supported(q.g, x)) return launch_direct_tma(q.g, x, f, y, st, device_error_word());
  return launch_direct(q.g, x, f, y, st);
}

const float *filter_ptr(cct_server *s, const Req &q) {
  return q.r.filter ? reinterpret_cast<float *>(q.dev + q.off_f) : s->filters[q.r.filter_id];
}

int copy_in(cct_server *s, Req &q, cudaStream_t st) {
  if (q.r.kind == CCT_SERVE_GRAPH_STEP) {
    float *in = nullptr;
    size_t n = 0;
    int rc = cct_graph_field(q.r.graph, 0, &in, &n);
    if (rc) return rc;
    return check_cuda(cudaMemcpyAsync(in, q.r.image, n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D request");
  }
  int rc = check_cuda(cudaMemcpyAsync(q.dev, q.r.image, q.x_elems * sizeof(float),
                                      cudaMemcpyHostToDevice, st),
                      "H2D request image");
  if (!rc && q.r.filter)
    rc = check_cuda(cudaMemcpyAsync(q.dev + q.off_f, q.r.filter,
                                    q.f_elems * sizeof(float), cudaMemcpyHostToDevice, st),
                    "H2D request filter");
  return rc;
}

int copy_out(cct_server *s, Req &q, cudaStream_t st) {
  if (q.r.kind == CCT_SERVE_GRAPH_STEP) {
    int32_t last = 0;
    float *out = nullptr;
    size_t n = 0;
    while (cct_graph_field(q.r.graph, last + 1, &out, &n) == CCT_OK) ++last;
    int rc = cct_graph_field(q.r.graph, last, &out, &n);
    if (rc) return rc;
    return check_cuda(cudaMemcpyAsync(q.r.out, out, n * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H request");
  }
  return check_cuda(cudaMemcpyAsync(q.r.out, q.dev + q.off_y, q.y_elems * sizeof(float),
                                    cudaMemcpyDeviceToHost, st),
                    "D2H request output");
}

float *out_ptr(cct_server *, const Req &q) { return reinterpret_cast<float *>(q.dev + q.off_y); }

void fill_item(cct_server *s, const Req &q, Item *it) {
  const ConvGeom &g = q.g;
  it->x = reinterpret_cast<float *>(q.dev);
  it->f = filter_ptr(s, q);
  it->y = out_ptr(s, q);
  it->H = g.H;
  it->W = g.W;
  it->R = g.R;
  it->conv = g.orient == CCT_CONVOLUTION;
  it->relu = (g.flags & CCT_FLAG_RELU) != 0;
  if (g.mode == CCT_PLANE_BY_PLANE) {
    it->mode = 0;
    it->C = g.pout;
    it->K = g.pout;
    it->fplanes = g.pf;
  } else {
    it->mode = 1;
    it->C = g.n;
    it->K = g.groups;
    it->fplanes = g.pf;
  }
  it->th = s->tile_rows[g.R];
  it->tiles_x = (g.W + kTileW - 1) / kTileW;
  it->tiles_y = (g.H + it->th - 1) / it->th;
}

void finish(cct_server *s, Req &q, int status, Clock::time_point t) {
  q.status = status;
  if (status != CCT_OK) q.msg = cct_last_error_string();
  q.latency_us = std::chrono::duration<double, std::micro>(t - q.t_submit).count();
  if (q.r.kind == CCT_SERVE_CONV) s->pool.release(q.dev, q.bytes);
  q.done = true;
  s->completed.fetch_add(1, std::memory_order_relaxed);
}

// Scheduler: retire finished slots.
bool retire(cct_server *s) {
  bool any = false;
  for (auto &sp : s->slots) {
    Slot &sl = *sp;
    if (!sl.busy || !sl.finished.load(std::memory_order_acquire)) continue;
    const cudaError_t e = cudaStreamQuery(sl.st);
    const int status = (e == cudaSuccess || e == cudaErrorNotReady) ? CCT_OK : check_cuda(e, "served launch");
    {
      std::lock_guard<std::mutex> lk(s->m);
      for (ReqPtr &q : sl.reqs) finish(s, *q, status, sl.t_done);
    }
    for (cct_graph *g : sl.graphs) s->busy_graphs.erase(g);
    sl.reqs.clear();
    sl.graphs.clear();
    sl.busy = false;
    sl.finished.store(false, std::memory_order_relaxed);
    any = true;
  }
  if (any) s->done_cv.notify_all();
  return any;
}

// Scheduler: admit waiting requests, in arrival order, while device memory
// for their fields can be had.
bool admit(cct_server *s) {
  bool any = false;
  while (!s->waiting.empty()) {
    ReqPtr q = s->waiting.front();
    if (q->r.kind == CCT_SERVE_CONV && !(q->dev = s->pool.alloc(q->bytes))) break;
    s->waiting.pop_front();
    s->admitted.push_back(q);
    any = true;
  }
  return any;
}

// Scheduler: launch admitted requests on a free slot.
bool launch(cct_server *s) {
  if (s->admitted.empty()) return false;
  Slot *free_slot = nullptr;
  for (auto &sp : s->slots)
    if (!sp->busy) {
      free_slot = sp.get();
      break;
    }
  if (!free_slot) return false;
  Slot &sl = *free_slot;
  const bool per_call = (s->cfg.flags & CCT_SERVE_PER_CALL) != 0;
  const int cap = per_call ? 1 : s->cfg.max_batch;
  std::vector<ReqPtr> take;
  std::deque<ReqPtr> keep;
  while (!s->admitted.empty() && (int)take.size() < cap) {
    ReqPtr q = s->admitted.front();
    s->admitted.pop_front();
    if (q->r.kind == CCT_SERVE_GRAPH_STEP) {
      // one step of a graph at a time: its fields are shared
      if (s->busy_graphs.count(q->r.graph) ||
          std::find(sl.graphs.begin(), sl.graphs.end(), q->r.graph) != sl.graphs.end()) {
        keep.push_back(q);
        continue;
      }
      sl.graphs.push_back(q->r.graph);
    }
    take.push_back(q);
  }
  for (auto it = keep.rbegin(); it != keep.rend(); ++it) s->admitted.push_front(*it);
  if (take.empty()) {
    sl.graphs.clear();
    return false;
  }
  for (cct_graph *g : sl.graphs) s->busy_graphs.insert(g);
  int rc = CCT_OK;
  Batch &b = *sl.h_table;
  b.n = 0;
  b.total = 0;
  for (ReqPtr &q : take) {
    if (!rc) rc = copy_in(s, *q, sl.st);
    if (rc) break;
    if (!per_call && q->batchable) {
      Item &it = b.items[b.n++];
      fill_item(s, *q, &it);
      it.first = b.total;
      b.total += (long long)it.K * it.tiles_x * it.tiles_y;
    } else {
      rc = launch_solo(s, *q, reinterpret_cast<float *>(q->dev), q->r.kind == CCT_SERVE_CONV ? filter_ptr(s, *q) : nullptr,
                       q->r.kind == CCT_SERVE_CONV ? out_ptr(s, *q) : nullptr, sl.st);
      s->solo.fetch_add(1, std::memory_order_relaxed);
    }
  }
  if (!rc && b.n > 0) {
    rc = check_cuda(cudaGraphLaunch(sl.exec, sl.st), "cudaGraphLaunch(serve batch)");
    count_launches(1);
    s->batches.fetch_add(1, std::memory_order_relaxed);
  }
  for (ReqPtr &q : take)
    if (!rc) rc = copy_out(s, *q, sl.st);
  sl.reqs = take;
  sl.busy = true;
  sl.owner = s;
  if (!rc) rc = check_cuda(cudaLaunchHostFunc(sl.st, host_done, &sl), "cudaLaunchHostFunc");
  if (rc) {
    // the slot's work is abandoned: wait for what was queued, then fail its requests
    cudaStreamSynchronize(sl.st);
    std::lock_guard<std::mutex> lk(s->m);
    for (ReqPtr &q : take) finish(s, *q, rc, Clock::now());
    for (cct_graph *g : sl.graphs) s->busy_graphs.erase(g);
    sl.reqs.clear();
    sl.graphs.clear();
    sl.busy = false;
    s->done_cv.notify_all();
    return true;
  }
  if (per_call) {
    // plain per-call dispatch: each request completes before the next starts
    cudaStreamSynchronize(sl.st);
    retire(s);
  }
  return true;
}

void scheduler(cct_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->m);
      while (!s->incoming.empty()) {
        s->waiting.push_back(s->incoming.front());
        s->incoming.pop_front();
      }
      bool busy = false;
      for (auto &sp : s->slots) busy = busy || sp->busy;
      if (s->stop && s->waiting.empty() && s->admitted.empty() && !busy) return;
    }
    bool progressed = retire(s);
    progressed = admit(s) || progressed;
    while (launch(s)) progressed = true;
    if (!progressed) {
      std::unique_lock<std::mutex> lk(s->m);
      bool finished = false;
      for (auto &sp : s->slots) finished = finished || (sp->busy && sp->finished.load());
      if (s->incoming.empty() && !finished && !s->stop)
        s->cv.wait_for(lk, std::chrono::milliseconds(2));
    }
  }
}

int capture_slot(cct_server *s, Slot &sl) {
  int rc = check_cuda(cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking), "cudaStreamCreate(slot)");
  if (!rc) rc = check_cuda(cudaMallocHost(&sl.h_table, sizeof(Batch)), "cudaMallocHost(batch table)");
  if (!rc) rc = check_cuda(cudaMalloc(&sl.d_table, sizeof(Batch)), "cudaMalloc(batch table)");
  if (!rc) rc = check_cuda(cudaMalloc(&sl.d_counter, sizeof(unsigned long long)), "cudaMalloc(counter)");
  if (rc) return rc;
  std::memset(sl.h_table, 0, sizeof(Batch));
  cudaGraph_t graph = nullptr;
  rc = check_cuda(cudaStreamBeginCapture(sl.st, cudaStreamCaptureModeThreadLocal), "capture(serve)");
  if (rc) return rc;
  cudaMemcpyAsync(sl.d_table, sl.h_table, sizeof(Batch), cudaMemcpyHostToDevice, sl.st);
  cudaMemsetAsync(sl.d_counter, 0, sizeof(unsigned long long), sl.st);
  serve_batch_kernel<<<s->grid, kThreads, 0, sl.st>>>(sl.d_table, sl.d_counter);
  rc = check_cuda(cudaStreamEndCapture(sl.st, &graph), "end capture(serve)");
  if (rc) return rc;
  rc = check_cuda(cudaGraphInstantiate(&sl.exec, graph, 0), "cudaGraphInstantiate(serve)");
  cudaGraphDestroy(graph);
  return rc;
}

// Autotuner: for each filter size, the tile height that serves a mixed
// synthetic batch fastest; and whether large frame requests run faster on
// their own kernel than in the batch (and from what size).
int autotune(cct_server *s) {
  const int sizes[] = {1, 3, 5, 7, 9};
  Slot &sl = *s->slots[0];
  const int H = 96, W = 96, C = 4, K = 16, items = 8;
  const size_t x_el = (size_t)C * H * W, f_el = (size_t)K * C * kMaxR * kMaxR, y_el = (size_t)K * H * W;
  const size_t bytes = (x_el + f_el + y_el) * sizeof(float);
  char *blk = s->pool.alloc(bytes);
  if (!blk) return CCT_OK;  // no device memory to tune with: keep defaults
  float *x = reinterpret_cast<float *>(blk), *f = x + x_el, *y = f + f_el;
  cudaMemsetAsync(x, 0, bytes, sl.st);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  for (int R : sizes) {
    float best = 1e30f;
    for (int th : {8, 16, 32}) {
      Batch &bt = *sl.h_table;
      bt.n = items;
      bt.total = 0;
      for (int i = 0; i < items; ++i) {
        Item &it = bt.items[i];
        it = Item{x, f, y, H, W, C, K, R, 1, 0, K * C, 0, th, (W + kTileW - 1) / kTileW, (H + th - 1) / th, 0};
        it.first = bt.total;
        bt.total += (long long)K * it.tiles_x * it.tiles_y;
      }
      cudaGraphLaunch(sl.exec, sl.st);  // warm
      cudaEventRecord(a, sl.st);
      for (int rep = 0; rep < 3; ++rep) cudaGraphLaunch(sl.exec, sl.st);
      cudaEventRecord(b, sl.st);
      cudaEventSynchronize(b);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, a, b);
      if (ms < best) {
        best = ms;
        s->tile_rows[R] = th;
      }
    }
  }
  // A large frame request (C = 4 -> K = 16, 96x96, 5x5) batched alone vs on
  // the frame kernel: if the frame kernel is faster, requests worth more
  // than ~20 us of its time run on it (launch cost is then under a few %).
  {
    ConvGeom g{};
    cct_conv_desc d;
    cct_conv_desc_init(&d);
    d.image_rows = H;
    d.image_cols = W;
    d.image_planes = C;
    d.filter_rows = d.filter_cols = 5;
    d.filter_planes = K * C;
    d.batch_size = 1;
    d.vector_mode = CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM;
    float t_batch = 0.0f, t_solo = 0.0f;
    if (resolve_geom(&d, &g) == CCT_OK && frame_f32_supported(g)) {
      Batch &bt = *sl.h_table;
      bt.n = 1;
      bt.items[0] = Item{x, f, y, H, W, C, K, 5, 1, 0, K * C, 0, s->tile_rows[5], (W + kTileW - 1) / kTileW,
                         (H + s->tile_rows[5] - 1) / s->tile_rows[5], 0};
      bt.total = (long long)K * bt.items[0].tiles_x * bt.items[0].tiles_y;
      cudaGraphLaunch(sl.exec, sl.st);
      cudaEventRecord(a, sl.st);
      for (int rep = 0; rep < 5; ++rep) cudaGraphLaunch(sl.exec, sl.st);
      cudaEventRecord(b, sl.st);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&t_batch, a, b);
      launch_frame_f32(g, x, f, y, sl.st);
      cudaEventRecord(a, sl.st);
      for (int rep = 0; rep < 5; ++rep) launch_frame_f32(g, x, f, y, sl.st);
      cudaEventRecord(b, sl.st);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&t_solo, a, b);
      const double flops = 2.0 * K * H * W * C * 25;
      if (t_solo > 0.0f && t_solo * 1.2f < t_batch) s->solo_flops = flops / (t_solo / 5 * 1e-3) * 20e-6;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  s->pool.release(blk, bytes);
  return check_cuda(cudaStreamSynchronize(sl.st), "server autotune");
}

}  // namespace

extern "C" {

void cct_server_config_init(cct_server_config *cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->struct_size = sizeof(*cfg);
  cfg->slots = 3;
  cfg->max_batch = 64;
  cfg->arena_bytes = 0;                 // no cap: admission by free HBM
  cfg->hbm_reserve_bytes = 2ull << 30;  // left free for other work on the device
}

void cct_serve_request_init(cct_serve_request *req) {
  if (!req) return;
  std::memset(req, 0, sizeof(*req));
  req->struct_size = sizeof(*req);
  cct_conv_desc_init(&req->desc);
  req->filter_id = -1;
}

int cct_server_create(const cct_server_config *cfg, cct_server **out) {
  if (!out) return set_error(CCT_EINVAL, "null argument");
  *out = nullptr;
  cct_server_config c;
  cct_server_config_init(&c);
  if (cfg) {
    if (cfg->struct_size != (int32_t)sizeof(cct_server_config))
      return set_error(CCT_EINVAL, "cct_server_config.struct_size %d != %zu", cfg->struct_size,
                       sizeof(cct_server_config));
    if (cfg->slots) c.slots = cfg->slots;
    if (cfg->max_batch) c.max_batch = cfg->max_batch;
    c.arena_bytes = cfg->arena_bytes;
    if (cfg->hbm_reserve_bytes) c.hbm_reserve_bytes = cfg->hbm_reserve_bytes;
    c.flags = cfg->flags;
  }
  if (c.slots < 1 || c.slots > 8) return set_error(CCT_EINVAL, "slots must be 1..8, got %d", c.slots);
  if (c.max_batch < 1 || c.max_batch > kMaxItems)
    return set_error(CCT_EINVAL, "max_batch must be 1..%d, got %d", kMaxItems, c.max_batch);
  if (c.flags & CCT_SERVE_PER_CALL) c.slots = 1;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(CCT_ENODEV, "no CUDA device");
  std::unique_ptr<cct_server> s(new (std::nothrow) cct_server);
  if (!s) return set_error(CCT_ENOMEM, "out of host memory");
  s->cfg = c;
  int rc = check_cuda(cudaGetDevice(&s->device), "cudaGetDevice");
  int sms = 148, per_sm = 0;
  if (!rc) rc = check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device), "SM count");
  if (!rc)
    rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_batch_kernel, kThreads, 0),
                    "occupancy(serve)");
  if (rc) return rc;
  s->grid = sms * std::max(per_sm, 1);
  // chunks of 1 GiB (or the cap, if smaller), a larger request gets a chunk of its own
  s->pool.init(c.arena_bytes, c.hbm_reserve_bytes, std::min<size_t>(c.arena_bytes ? c.arena_bytes : ~(size_t)0, (size_t)1 << 30));
  for (int i = 0; i < c.slots && !rc; ++i) {
    s->slots.emplace_back(new Slot);
    rc = capture_slot(s.get(), *s->slots.back());
  }
  if (!rc && !(c.flags & CCT_SERVE_PER_CALL)) rc = autotune(s.get());
  if (rc) {
    for (auto &sl : s->slots) {
      if (sl->exec) cudaGraphExecDestroy(sl->exec);
      if (sl->st) cudaStreamDestroy(sl->st);
      cudaFreeHost(sl->h_table);
      cudaFree(sl->d_table);
      cudaFree(sl->d_counter);
    }
    return rc;
  }
  cct_server *raw = s.release();
  raw->worker = std::thread(scheduler, raw);
  *out = raw;
  return CCT_OK;
}

int cct_server_destroy(cct_server *s) {
  if (!s) return CCT_OK;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  for (auto &sl : s->slots) {
    if (sl->st) cudaStreamSynchronize(sl->st);
    if (sl->exec) cudaGraphExecDestroy(sl->exec);
    if (sl->st) cudaStreamDestroy(sl->st);
    cudaFreeHost(sl->h_table);
    cudaFree(sl->d_table);
    cudaFree(sl->d_counter);
  }
  for (float *f : s->filters) cudaFree(f);
  delete s;
  return CCT_OK;
}

int cct_server_add_filter(cct_server *s, const float *host_filter, size_t elems, int32_t *id) {
  if (!s || !host_filter || !id || elems == 0) return set_error(CCT_EINVAL, "null or empty argument");
  float *d = nullptr;
  int rc = check_cuda(cudaMalloc(&d, elems * sizeof(float)), "cudaMalloc(resident filter)");
  if (!rc) rc = check_cuda(cudaMemcpy(d, host_filter, elems * sizeof(float), cudaMemcpyHostToDevice), "H2D filter");
  if (rc) {
    cudaFree(d);
    return rc;
  }
  std::lock_guard<std::mutex> lk(s->m);
  s->filters.push_back(d);
  s->filter_elems.push_back(elems);
  *id = (int32_t)s->filters.size() - 1;
  return CCT_OK;
}

int cct_server_submit(cct_server *s, const cct_serve_request *req, uint64_t *ticket) {
  if (!s || !req || !ticket) return set_error(CCT_EINVAL, "null argument");
  if (req->struct_size != (int32_t)sizeof(cct_serve_request))
    return set_error(CCT_EINVAL, "cct_serve_request.struct_size %d != %zu", req->struct_size,
                     sizeof(cct_serve_request));
  if (!req->image || !req->out) return set_error(CCT_EINVAL, "null request image or output");
  auto q = std::make_shared<Req>();
  q->r = *req;
  if (req->kind == CCT_SERVE_GRAPH_STEP) {
    if (!req->graph) return set_error(CCT_EINVAL, "graph step request without a graph");
  } else if (req->kind == CCT_SERVE_CONV) {
    int rc = resolve_geom(&req->desc, &q->g);
    if (rc) return rc;
    const ConvGeom &g = q->g;
    int32_t orows, ocols, oplanes;
    rc = cct_conv_output_shape(&req->desc, &orows, &ocols, &oplanes);
    if (rc) return rc;
    if (g.mode != CCT_PLANE_BY_PLANE && !(g.mode == CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM && g.batch == 1))
      return set_error(CCT_EINVAL, "served convolutions are plane by plane or a block-reduced frame of batch 1");
    if (req->desc.precision != CCT_PREC_FP32) return set_error(CCT_EINVAL, "served convolutions are FP32");
    q->x_elems = (size_t)g.pin * g.H * g.W;
    q->f_elems = (size_t)g.pf * g.R * g.S;
    q->y_elems = (size_t)orows * ocols * (oplanes < 1 ? 1 : oplanes);
    if (!req->filter) {
      std::lock_guard<std::mutex> lk(s->m);
      if (req->filter_id < 0 || req->filter_id >= (int32_t)s->filters.size())
        return set_error(CCT_EINVAL, "no resident filter %d", req->filter_id);
      if (s->filter_elems[req->filter_id] != q->f_elems)
        return set_error(CCT_EINVAL, "resident filter %d holds %zu values, the request needs %zu", req->filter_id,
                         s->filter_elems[req->filter_id], q->f_elems);
    }
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    q->off_f = al(q->x_elems * sizeof(float));
    q->off_y = q->off_f + (req->filter ? al(q->f_elems * sizeof(float)) : 0);
    q->bytes = q->off_y + al(q->y_elems * sizeof(float));
    const size_t cap = s->pool.capacity();
    if (q->bytes > cap)
      return set_error(CCT_EINVAL, "request needs %zu bytes of device memory, the server's arena holds %zu",
                       q->bytes, cap);
    q->flops = 2.0 * q->y_elems * g.R * g.S * g.terms;
    q->batchable = g.border == CCT_BORDER_ZERO && g.down == 1 && g.up == 1 && g.R == g.S && (g.R & 1) &&
                   g.R <= kMaxR && g.pin >= 1 && q->flops < s->solo_flops;
    // the batch kernel reads input plane o for output plane o
    if (g.mode == CCT_PLANE_BY_PLANE && g.pin != g.pout) q->batchable = false;
  } else {
    return set_error(CCT_EINVAL, "unknown request kind %d", req->kind);
  }
  std::lock_guard<std::mutex> lk(s->m);
  if (s->stop) return set_error(CCT_EINVAL, "server is shutting down");
  q->ticket = s->next_ticket++;
  q->t_submit = Clock::now();
  s->table[q->ticket] = q;
  s->incoming.push_back(q);
  *ticket = q->ticket;
  s->cv.notify_all();
  return CCT_OK;
}

int cct_server_wait(cct_server *s, uint64_t ticket, int32_t timeout_ms, double *latency_us) {
  if (!s) return set_error(CCT_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->table.find(ticket);
  if (it == s->table.end()) return set_error(CCT_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
  ReqPtr q = it->second;
  auto pred = [&] { return q->done; };
  if (timeout_ms < 0) {
    s->done_cv.wait(lk, pred);
  } else if (!s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
    return set_error(CCT_ETIMEOUT, "request %llu not finished after %d ms", (unsigned long long)ticket, timeout_ms);
  }
  if (latency_us) *latency_us = q->latency_us;
  s->table.erase(ticket);
  if (q->status != CCT_OK) return set_error(q->status, "request %llu: %s", (unsigned long long)ticket, q->msg.c_str());
  return CCT_OK;
}

int cct_server_replay(cct_server *s, const cct_serve_request *reqs, const double *arrival_s, int32_t n,
                      double *latency_us) {
  if (!s || !reqs || !arrival_s || !latency_us || n < 0) return set_error(CCT_EINVAL, "null argument");
  std::vector<uint64_t> tickets(n, 0);
  std::vector<int> status(n, CCT_OK);
  const Clock::time_point t0 = Clock::now();
  std::thread client([&] {
    for (int32_t i = 0; i < n; ++i) {
      const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
      while (Clock::now() < due) {
        const auto left = due - Clock::now();
        if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left - std::chrono::microseconds(100));
      }
      status[i] = cct_server_submit(s, &reqs[i], &tickets[i]);
    }
  });
  client.join();
  int first = CCT_OK;
  for (int32_t i = 0; i < n; ++i) {
    latency_us[i] = -1.0;
    if (status[i]) {
      if (!first) first = status[i];
      continue;
    }
    const int rc = cct_server_wait(s, tickets[i], -1, &latency_us[i]);
    if (rc && !first) first = rc;
  }
  return first;
}

int cct_server_stats(const cct_server *s, uint64_t *completed, uint64_t *batches, uint64_t *solo,
                     uint64_t *peak_arena_bytes) {
  if (!s) return set_error(CCT_EINVAL, "null server");
  if (completed) *completed = s->completed.load();
  if (batches) *batches = s->batches.load();
  if (solo) *solo = s->solo.load();
  if (peak_arena_bytes) *peak_arena_bytes = s->pool.peak();
  return CCT_OK;
}

int cct_host_alloc(void **ptr, size_t bytes) {
  if (!ptr) return set_error(CCT_EINVAL, "null argument");
  return check_cuda(cudaMallocHost(ptr, bytes), "cudaMallocHost");
}

int cct_host_free(void *ptr) { return check_cuda(cudaFreeHost(ptr), "cudaFreeHost"); }

}  // extern "C"
