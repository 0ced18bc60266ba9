// Host side of the batching form: mixed-shape, mixed-direction batches in one persistent
// launch (k_ragged), and the per-array launch loop it is compared against.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/bridct_b200.h"
#include "bridct_internal.h"
#include "ragged.cuh"

struct bridct_ragged {
  int device = 0;
  bridct::DeviceCtx* dev = nullptr;
  std::vector<bridct_ragged_item> items;
  std::vector<bridct::RaggedArray> arrays;
  std::vector<bridct::RaggedUnit> units;
  bridct::RaggedArray* d_arrays = nullptr;
  bridct::RaggedUnit* d_units = nullptr;
  unsigned int* d_counters = nullptr;   // [0] queue head, [1..n] strips done per array
  int* d_err = nullptr;
  size_t span = 0;                      // floats covered by the batch (max offset + size)
  int grid = 0;
  bridct_ragged_tuning tuning{};
  std::map<int, bridct_plan*> plans;    // per-array launch loop: one plan per shape
};

namespace bridct {
namespace {

int lg(int n) {
  int k = 0;
  while ((8 << k) < n) ++k;
  return k;
}

// Four-step lines of length n are processed LPW = 1024/n at a time by one warp, so a unit must
// hold a multiple of that many lines (1 for register lines).
int lines_per_warp(int n) { return n >= 128 ? 1024 / n : 1; }

int pow2_floor(int v) {
  int p = 1;
  while (p * 2 <= v) p *= 2;
  return p;
}

// Columns per strip: a power of two dividing w, >= 4 (float4 rows), >= the four-step group,
// and h * columns <= budget unless the minimum forces more.
int strip_cols(int h, int w, int budget) {
  const int want = pow2_floor(std::max(1, std::min(w, budget / h)));
  return std::min(w, std::max(want, std::max(4, lines_per_warp(h))));
}

// Rows per row block: a power of two dividing h, >= the four-step group.
int block_rows(int h, int w, int budget) {
  const int want = pow2_floor(std::max(1, std::min(h, budget / w)));
  return std::min(h, std::max(want, lines_per_warp(w)));
}

void build_units(bridct_ragged* r) {
  const bridct_ragged_tuning& t = r->tuning;
  std::vector<int> big, small;
  r->arrays.clear();
  for (size_t i = 0; i < r->items.size(); ++i) {
    const bridct_ragged_item& it = r->items[i];
    RaggedArray a{(long long)it.offset, it.height, it.width, it.mode, 0};
    const long long e = (long long)it.height * it.width;
    if (e <= t.tile_floats) {
      small.push_back((int)i);
    } else {
      a.nstrips = it.width / strip_cols(it.height, it.width, t.strip_floats);
      big.push_back((int)i);
    }
    r->arrays.push_back(a);
  }
  auto size_desc = [&](int a, int b) {
    const long long ea = (long long)r->items[a].height * r->items[a].width;
    const long long eb = (long long)r->items[b].height * r->items[b].width;
    return ea != eb ? ea > eb : a < b;
  };
  std::stable_sort(big.begin(), big.end(), size_desc);
  std::stable_sort(small.begin(), small.end(), size_desc);
  r->units.clear();
  auto cols = [&](int i) {
    const RaggedArray& a = r->arrays[i];
    const int tc = a.w / a.nstrips;
    for (int s = 0; s < a.nstrips; ++s) r->units.push_back(RaggedUnit{i, UNIT_COLSTRIP, s * tc, tc});
  };
  auto rows = [&](int i) {
    const RaggedArray& a = r->arrays[i];
    const int rb = block_rows(a.h, a.w, t.row_floats);
    for (int r0 = 0; r0 < a.h; r0 += rb) r->units.push_back(RaggedUnit{i, UNIT_ROWBLOCK, r0, rb});
  };
  // Column strips of array k+lookahead are queued ahead of the row blocks of array k, so a
  // row block usually finds its strips finished; small arrays fill the tail.
  const int la = std::max(1, t.lookahead);
  for (size_t k = 0; k < big.size() + la; ++k) {
    if (k < big.size()) cols(big[k]);
    if (k >= (size_t)la) rows(big[k - la]);
  }
  for (int i : small) r->units.push_back(RaggedUnit{i, UNIT_TILE, 0, 0});
}

int upload(bridct_ragged* r) {
  cudaFree(r->d_arrays);
  cudaFree(r->d_units);
  r->d_arrays = nullptr;
  r->d_units = nullptr;
  cudaError_t e = cudaMalloc((void**)&r->d_arrays, r->arrays.size() * sizeof(RaggedArray));
  if (e == cudaSuccess) e = cudaMalloc((void**)&r->d_units, std::max<size_t>(1, r->units.size()) * sizeof(RaggedUnit));
  if (e == cudaSuccess)
    e = cudaMemcpy(r->d_arrays, r->arrays.data(), r->arrays.size() * sizeof(RaggedArray), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !r->units.empty())
    e = cudaMemcpy(r->d_units, r->units.data(), r->units.size() * sizeof(RaggedUnit), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "ragged upload");
}

}  // namespace
}  // namespace bridct

using namespace bridct;

extern "C" {

BRIDCT_API void bridct_ragged_default_tuning(bridct_ragged_tuning* t) {
  if (!t) return;
  t->tile_floats = 16384;
  t->strip_floats = 16384;
  t->row_floats = 16384;
  t->lookahead = 2;
}

BRIDCT_API bridct_ragged* bridct_ragged_create(const bridct_ragged_item* items, size_t count) {
  bridct_ragged_tuning t;
  bridct_ragged_default_tuning(&t);
  return bridct_ragged_create_tuned(items, count, &t);
}

BRIDCT_API bridct_ragged* bridct_ragged_create_tuned(const bridct_ragged_item* items, size_t count,
                                                     const bridct_ragged_tuning* tuning) {
  if (!items || count == 0 || count > 0x7FFFFFFF || !tuning) {
    set_error("bridct_ragged_create: empty or NULL item list");
    return nullptr;
  }
  const bridct_ragged_tuning& t = *tuning;
  if (t.tile_floats < 64 || t.tile_floats > 16384 || t.strip_floats < 64 || t.strip_floats > 16384 ||
      t.row_floats < 64 || t.row_floats > 16384 || t.lookahead < 1 || t.lookahead > 64) {
    set_error("bridct_ragged_create: tuning out of range");
    return nullptr;
  }
  std::vector<std::pair<size_t, size_t>> spans;
  size_t span = 0;
  for (size_t i = 0; i < count; ++i) {
    const bridct_ragged_item& it = items[i];
    if (!bridct_supported(it.height, it.width) || it.mode < 0 || it.mode > 2 || it.offset % 4) {
      set_error("bridct_ragged_create: item " + std::to_string(i) +
                " has an unsupported shape, mode, or an offset that is not a multiple of 4 floats");
      return nullptr;
    }
    const size_t e = (size_t)it.height * it.width;
    spans.push_back({it.offset, it.offset + e});
    span = std::max(span, it.offset + e);
  }
  std::sort(spans.begin(), spans.end());
  for (size_t i = 1; i < spans.size(); ++i)
    if (spans[i].first < spans[i - 1].second) {
      set_error("bridct_ragged_create: arrays overlap");
      return nullptr;
    }
  int dev = 0;
  if (current_device(&dev) != BRIDCT_OK) return nullptr;
  DeviceCtx* d = device_ctx(dev);
  if (!d) return nullptr;
  bridct_ragged* r = new bridct_ragged();
  r->device = dev;
  r->dev = d;
  r->items.assign(items, items + count);
  r->span = span;
  r->tuning = t;
  build_units(r);
  cudaError_t e = cudaMalloc((void**)&r->d_counters, (count + 1) * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&r->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(r->d_err, 0, sizeof(int));
  if (e != cudaSuccess || upload(r) != BRIDCT_OK) {
    if (e != cudaSuccess) cuda_fail(e, "bridct_ragged_create");
    bridct_ragged_destroy(r);
    return nullptr;
  }
  static int bps = [] {
    if (cudaFuncSetAttribute(k_ragged, cudaFuncAttributeMaxDynamicSharedMemorySize, kRaggedSmem) != cudaSuccess)
      return 0;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_ragged, kRaggedThreads, kRaggedSmem) != cudaSuccess) return 0;
    return b;
  }();
  if (bps <= 0) {
    cuda_fail(cudaErrorInvalidConfiguration, "k_ragged occupancy");
    bridct_ragged_destroy(r);
    return nullptr;
  }
  r->grid = std::min<long long>((long long)d->sm_count * bps, std::max<size_t>(1, r->units.size()));
  return r;
}

BRIDCT_API void bridct_ragged_destroy(bridct_ragged* r) {
  if (!r) return;
  cudaFree(r->d_arrays);
  cudaFree(r->d_units);
  cudaFree(r->d_counters);
  cudaFree(r->d_err);
  for (auto& kv : r->plans) bridct_plan_destroy(kv.second);
  delete r;
}

BRIDCT_API size_t bridct_ragged_units(const bridct_ragged* r) { return r ? r->units.size() : 0; }

BRIDCT_API int bridct_ragged_apply_device(bridct_ragged* r, const float* x, float* y, void* stream) {
  if (!r || !x || !y) return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = r->span * sizeof(float);
  const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
  if ((a <= b ? b - a : a - b) < bytes) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((a | b) % 16) return BRIDCT_BAD_ALIGNMENT;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(r->d_counters, 0, (r->items.size() + 1) * sizeof(unsigned int), st);
  if (e != cudaSuccess) return cuda_fail(e, "ragged reset");
  RaggedArgs args;
  args.x = x;
  args.y = y;
  args.arrays = r->d_arrays;
  args.units = r->d_units;
  args.nunits = (int)r->units.size();
  args.next = r->d_counters;
  args.done = r->d_counters + 1;
  args.err = r->d_err;
  for (int i = 0; i < 4; ++i) args.tab[i] = r->dev->fourstep[i];
  k_ragged<<<r->grid, kRaggedThreads, kRaggedSmem, st>>>(args);
  e = cudaGetLastError();
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_ragged launch");
}

BRIDCT_API int bridct_ragged_timeout_flag(bridct_ragged* r) {
  if (!r) return 0;
  int v = 0;
  cudaMemcpy(&v, r->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (v) cudaMemset(r->d_err, 0, sizeof(int));
  return v;
}

BRIDCT_API int bridct_ragged_apply_loop_device(bridct_ragged* r, const float* x, float* y, void* stream) {
  if (!r || !x || !y) return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = r->span * sizeof(float);
  const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
  if ((a <= b ? b - a : a - b) < bytes) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((a | b) % 16) return BRIDCT_BAD_ALIGNMENT;
  // one launch per array, grouped by shape so consecutive launches reuse kernels
  std::vector<int> order(r->items.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    const int kp = lg(r->items[p].height) * 8 + lg(r->items[p].width);
    const int kq = lg(r->items[q].height) * 8 + lg(r->items[q].width);
    return kp < kq;
  });
  for (int i : order) {
    const bridct_ragged_item& it = r->items[i];
    const int key = lg(it.height) * 8 + lg(it.width);
    bridct_plan*& p = r->plans[key];
    if (!p) {
      p = bridct_plan_create(it.height, it.width);
      if (!p) return BRIDCT_DEVICE_ERROR;
    }
    int s = launch_plain_form(p, it.mode, x + it.offset, y + it.offset, 1, (cudaStream_t)stream);
    if (s) return s;
  }
  return BRIDCT_OK;
}

}  // extern "C"
