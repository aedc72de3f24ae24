// Checkpoint records of plans and graphs: what ComputeGraph.write /
// readFromFile (src/main/scala/cogx/runtime/ComputeGraph.scala:523-727) need
// to save and restore a kernel of this backend.  The reference saves an
// OpenCL device kernel as its generated source code plus work-group
// parameters (platform/opencl/OpenCLDeviceKernel.scala:219-229) and rebuilds
// it on restore (OpenCLRestoredDeviceKernel.scala:53-64).  A kernel here is
// fully determined by its descriptor and, for a constant filter, the filter's
// values, so the record holds exactly those (plus a graph's step count), and
// restoring rebuilds the plans.
//
// The record is an array of 32-bit words, so that the Scala side can store it
// with the saver's writeIntArray and read it back with readIntArray:
//   0  magic 0x4B544343        1  format version (1)
//   2  kind (1 plan, 2 graph)  3  layer count
//   4  step count, low word    5  step count, high word
//   per layer: the descriptor's field count (15), the 15 fields from
//   image_rows to flags in declaration order, the filter element count (low,
//   high; 0: no constant filter), then the filter values as IEEE-754 bits
//   last: FNV-1a 32-bit hash of the bytes of every preceding word (each
//   word little-endian)
#include <cstring>
#include <vector>

#include "cct_internal.h"

namespace cct {
namespace {

constexpr uint32_t kMagic = 0x4B544343u;
constexpr uint32_t kVersion = 1;
constexpr uint32_t kDescFields = 15;

uint32_t fnv1a(const uint32_t *w, size_t n) {
  uint32_t h = 2166136261u;
  for (size_t i = 0; i < n; ++i)
    for (int b = 0; b < 4; ++b) {
      h ^= (w[i] >> (8 * b)) & 0xFFu;
      h *= 16777619u;
    }
  return h;
}

void desc_to_words(const cct_conv_desc &d, uint32_t *w) {
  const int32_t f[kDescFields] = {d.image_rows, d.image_cols, d.image_planes, d.filter_rows, d.filter_cols,
                                  d.filter_planes, d.batch_size, d.border, d.orientation, d.sampling,
                                  d.step, d.vector_mode, d.precision, d.algo, (int32_t)d.flags};
  for (uint32_t i = 0; i < kDescFields; ++i) w[i] = (uint32_t)f[i];
}

void words_to_desc(const uint32_t *w, cct_conv_desc *d) {
  cct_conv_desc_init(d);
  d->image_rows = (int32_t)w[0];
  d->image_cols = (int32_t)w[1];
  d->image_planes = (int32_t)w[2];
  d->filter_rows = (int32_t)w[3];
  d->filter_cols = (int32_t)w[4];
  d->filter_planes = (int32_t)w[5];
  d->batch_size = (int32_t)w[6];
  d->border = (int32_t)w[7];
  d->orientation = (int32_t)w[8];
  d->sampling = (int32_t)w[9];
  d->step = (int32_t)w[10];
  d->vector_mode = (int32_t)w[11];
  d->precision = (int32_t)w[12];
  d->algo = (int32_t)w[13];
  d->flags = w[14];
}

}  // namespace

int record_plan_layer(const cct_conv_plan *p, RecordLayer *out) {
  const float *dev = nullptr;
  size_t elems = 0;
  int device = 0;
  int rc = plan_record_parts(p, &out->desc, &dev, &elems, &device);
  if (rc) return rc;
  out->filter.clear();
  if (!dev) return CCT_OK;
  out->filter.resize(elems);
  int cur = 0;
  rc = check_cuda(cudaGetDevice(&cur), "cudaGetDevice");
  if (rc) return rc;
  if (cur != device) {
    rc = check_cuda(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
  }
  rc = check_cuda(cudaMemcpy(out->filter.data(), dev, elems * sizeof(float), cudaMemcpyDeviceToHost),
                  "copy static filter for the record");
  if (cur != device) cudaSetDevice(cur);
  return rc;
}

int record_encode(int kind, int64_t time, const std::vector<RecordLayer> &layers, std::vector<uint32_t> *out) {
  std::vector<uint32_t> &w = *out;
  w.clear();
  w.push_back(kMagic);
  w.push_back(kVersion);
  w.push_back((uint32_t)kind);
  w.push_back((uint32_t)layers.size());
  w.push_back((uint32_t)((uint64_t)time & 0xFFFFFFFFu));
  w.push_back((uint32_t)((uint64_t)time >> 32));
  for (const RecordLayer &l : layers) {
    w.push_back(kDescFields);
    uint32_t f[kDescFields];
    desc_to_words(l.desc, f);
    w.insert(w.end(), f, f + kDescFields);
    const uint64_t n = l.filter.size();
    w.push_back((uint32_t)(n & 0xFFFFFFFFu));
    w.push_back((uint32_t)(n >> 32));
    const size_t at = w.size();
    w.resize(at + n);
    if (n) std::memcpy(&w[at], l.filter.data(), n * sizeof(float));
  }
  w.push_back(fnv1a(w.data(), w.size()));
  return CCT_OK;
}

int record_decode(const uint32_t *w, size_t n, int *kind, int64_t *time, std::vector<RecordLayer> *layers) {
  if (!w) return set_error(CCT_EINVAL, "null record");
  if (n < 7) return set_error(CCT_EINVAL, "record too short (%zu words)", n);
  if (w[0] != kMagic) return set_error(CCT_EINVAL, "not a libcctconv record (magic 0x%08x)", w[0]);
  if (w[1] != kVersion) return set_error(CCT_EINVAL, "record format version %u is not supported", w[1]);
  if (fnv1a(w, n - 1) != w[n - 1]) return set_error(CCT_EINVAL, "record checksum mismatch (corrupted record)");
  if (w[2] != 1 && w[2] != 2) return set_error(CCT_EINVAL, "unknown record kind %u", w[2]);
  *kind = (int)w[2];
  const uint32_t count = w[3];
  if (count < 1 || (w[2] == 1 && count != 1)) return set_error(CCT_EINVAL, "bad layer count %u", count);
  *time = (int64_t)((uint64_t)w[4] | ((uint64_t)w[5] << 32));
  layers->clear();
  size_t at = 6;
  for (uint32_t i = 0; i < count; ++i) {
    if (at + 1 + kDescFields + 2 > n - 1) return set_error(CCT_EINVAL, "record truncated in layer %u", i + 1);
    if (w[at] != kDescFields) return set_error(CCT_EINVAL, "layer %u: %u descriptor fields", i + 1, w[at]);
    RecordLayer l;
    words_to_desc(w + at + 1, &l.desc);
    at += 1 + kDescFields;
    const uint64_t elems = (uint64_t)w[at] | ((uint64_t)w[at + 1] << 32);
    at += 2;
    if (elems > (uint64_t)(n - 1 - at)) return set_error(CCT_EINVAL, "record truncated in layer %u's filter", i + 1);
    l.filter.resize((size_t)elems);
    if (elems) std::memcpy(l.filter.data(), w + at, (size_t)elems * sizeof(float));
    at += (size_t)elems;
    layers->push_back(std::move(l));
  }
  if (at != n - 1) return set_error(CCT_EINVAL, "record has %zu unexpected trailing words", n - 1 - at);
  return CCT_OK;
}

int record_store(const std::vector<uint32_t> &words, uint32_t *out, size_t capacity, size_t *n_words) {
  if (n_words) *n_words = words.size();
  if (!out) return CCT_OK;  // size query
  if (capacity < words.size())
    return set_error(CCT_EINVAL, "the record needs %zu words, the buffer holds %zu", words.size(), capacity);
  std::memcpy(out, words.data(), words.size() * sizeof(uint32_t));
  return CCT_OK;
}

}  // namespace cct

using namespace cct;

extern "C" {

int cct_conv_plan_save(const cct_conv_plan *plan, uint32_t *words, size_t capacity, size_t *n_words) {
  if (!plan) return set_error(CCT_EINVAL, "null plan");
  std::vector<RecordLayer> layers(1);
  int rc = record_plan_layer(plan, &layers[0]);
  if (rc) return rc;
  std::vector<uint32_t> w;
  record_encode(1, 0, layers, &w);
  return record_store(w, words, capacity, n_words);
}

int cct_conv_plan_restore(const uint32_t *words, size_t n_words, cct_conv_plan **plan) {
  if (!plan) return set_error(CCT_EINVAL, "null plan output");
  *plan = nullptr;
  int kind = 0;
  int64_t time = 0;
  std::vector<RecordLayer> layers;
  int rc = record_decode(words, n_words, &kind, &time, &layers);
  if (rc) return rc;
  if (kind != 1) return set_error(CCT_EINVAL, "the record holds a graph, not a plan");
  cct_conv_plan *p = nullptr;
  rc = cct_conv_plan_create(&layers[0].desc, &p);
  if (rc) return rc;
  if (!layers[0].filter.empty()) {
    size_t need = 0;
    rc = plan_filter_elems(p, &need);
    if (!rc && need != layers[0].filter.size())
      rc = set_error(CCT_EINVAL, "record filter has %zu values, the plan needs %zu", layers[0].filter.size(), need);
    if (!rc) rc = cct_conv_plan_set_static_filter(p, layers[0].filter.data());
    if (rc) {
      cct_conv_plan_destroy(p);
      return rc;
    }
  }
  *plan = p;
  return CCT_OK;
}

int cct_record_describe(const uint32_t *words, size_t n_words, int32_t *kind, int32_t *n_layers, int64_t *time,
                        cct_conv_desc *descs, int32_t max_descs) {
  int k = 0;
  int64_t t = 0;
  std::vector<RecordLayer> layers;
  int rc = record_decode(words, n_words, &k, &t, &layers);
  if (rc) return rc;
  if (kind) *kind = k;
  if (n_layers) *n_layers = (int32_t)layers.size();
  if (time) *time = t;
  for (int32_t i = 0; descs && i < max_descs && i < (int32_t)layers.size(); ++i) descs[i] = layers[i].desc;
  return CCT_OK;
}

}  // extern "C"
