// Host side of the batching form: mixed-shape, mixed-direction batches in one persistent
// launch (k_ragged), and the per-array launch loop it is compared against.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/bridct_b200.h"
#include "bridct_internal.h"
#include "ragged.cuh"

// One shape class of a ragged batch: every array of one (height, width, mode), with the device
// table of their offsets and the schedule that runs them.
struct RaggedClass {
  int h = 0, w = 0, mode = 0;
  std::vector<int> arrays;            // indices into the item list
  long long* d_offs = nullptr;        // offsets (floats) of those arrays
  size_t floats = 0;                  // elements of the class
  int schedule = BRIDCT_RAGGED_QUEUE;
};

constexpr int kRaggedMaxStreams = 8;

// A merged pass: every column strip (col) or row block of the MERGED classes that share one column
// length (or row length) and mode, as one launch over a device table of units.
struct MergedPass {
  int len = 0, mode = 0;
  bool col = true;
  bridct::PassUnit* d_units = nullptr;
  long long n = 0;
  size_t floats = 0;
};

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
  unsigned spin_limit = bridct::kRaggedSpin;
  bridct_ragged_tuning tuning{};
  std::map<int, bridct_plan*> plans;    // per-array launch loop: one plan per shape
  // shape classes, in decreasing size; classes scheduled as their own launches run on `streams`
  // side streams forked from and joined back into the caller's stream
  std::vector<RaggedClass> classes;
  std::vector<MergedPass> merged;       // column passes first, then row passes
  int streams = 4;
  cudaStream_t aux[kRaggedMaxStreams] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kRaggedMaxStreams] = {};
  cudaEvent_t mid_ev[kRaggedMaxStreams] = {}, mid_fork = nullptr;   // between merged column and row passes
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
  std::vector<char> queued(r->items.size(), 1);
  for (const RaggedClass& c : r->classes)
    if (c.schedule != BRIDCT_RAGGED_QUEUE)
      for (int i : c.arrays) queued[i] = 0;
  r->arrays.clear();
  for (size_t i = 0; i < r->items.size(); ++i) {
    const bridct_ragged_item& it = r->items[i];
    RaggedArray a{(long long)it.offset, it.height, it.width, it.mode, 0};
    const long long e = (long long)it.height * it.width;
    if (!queued[i]) {
      // run by its class's own launch: not in the queue
    } else if (e <= t.tile_floats) {
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

// Groups the items into shape classes (height, width, mode), largest first, and uploads each
// class's offset table.
int build_classes(bridct_ragged* r) {
  std::map<std::tuple<int, int, int>, size_t> index;
  for (size_t i = 0; i < r->items.size(); ++i) {
    const bridct_ragged_item& it = r->items[i];
    const auto key = std::make_tuple(it.height, it.width, it.mode);
    auto f = index.find(key);
    if (f == index.end()) {
      f = index.emplace(key, r->classes.size()).first;
      RaggedClass c;
      c.h = it.height;
      c.w = it.width;
      c.mode = it.mode;
      r->classes.push_back(c);
    }
    RaggedClass& c = r->classes[f->second];
    c.arrays.push_back((int)i);
    c.floats += (size_t)it.height * it.width;
  }
  std::stable_sort(r->classes.begin(), r->classes.end(),
                   [](const RaggedClass& a, const RaggedClass& b) { return a.floats > b.floats; });
  for (RaggedClass& c : r->classes) {
    std::vector<long long> offs;
    for (int i : c.arrays) offs.push_back((long long)r->items[i].offset);
    cudaError_t e = cudaMalloc((void**)&c.d_offs, offs.size() * sizeof(long long));
    if (e == cudaSuccess) e = cudaMemcpy(c.d_offs, offs.data(), offs.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "ragged class tables");
  }
  cudaError_t e = cudaEventCreateWithFlags(&r->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->mid_fork, cudaEventDisableTiming);
  for (int i = 0; e == cudaSuccess && i < kRaggedMaxStreams; ++i) {
    e = cudaStreamCreateWithFlags(&r->aux[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->join_ev[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->mid_ev[i], cudaEventDisableTiming);
  }
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "ragged streams");
}

void free_merged(bridct_ragged* r) {
  for (MergedPass& m : r->merged) cudaFree(m.d_units);
  r->merged.clear();
}

// Unit tables of the merged passes: column strips of the MERGED classes grouped by (column length,
// mode), row blocks grouped by (row length, mode), each group largest first.
int build_merged(bridct_ragged* r) {
  free_merged(r);
  std::map<std::pair<int, int>, std::vector<PassUnit>> cols, rows;
  std::map<std::pair<int, int>, size_t> cfl, rfl;
  for (const RaggedClass& c : r->classes) {
    if (c.schedule != BRIDCT_RAGGED_MERGED) continue;
    const int tc = merged_strip_cols(c.h), rb = merged_block_rows(c.w);
    for (int i : c.arrays) {
      const long long off = (long long)r->items[i].offset;
      for (int s0 = 0; s0 < c.w; s0 += tc) cols[{c.h, c.mode}].push_back(PassUnit{off + s0, c.w});
      for (int r0 = 0; r0 < c.h; r0 += rb) rows[{c.w, c.mode}].push_back(PassUnit{off + (long long)r0 * c.w, c.w});
      cfl[{c.h, c.mode}] += (size_t)c.h * c.w;
      rfl[{c.w, c.mode}] += (size_t)c.h * c.w;
    }
  }
  for (int pass = 0; pass < 2; ++pass) {
    auto& groups = pass == 0 ? cols : rows;
    auto& fl = pass == 0 ? cfl : rfl;
    std::vector<MergedPass> list;
    for (auto& kv : groups) {
      MergedPass m;
      m.len = kv.first.first;
      m.mode = kv.first.second;
      m.col = pass == 0;
      m.n = (long long)kv.second.size();
      m.floats = fl[kv.first];
      cudaError_t e = cudaMalloc((void**)&m.d_units, kv.second.size() * sizeof(PassUnit));
      if (e == cudaSuccess)
        e = cudaMemcpy(m.d_units, kv.second.data(), kv.second.size() * sizeof(PassUnit), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        cudaFree(m.d_units);
        free_merged(r);
        return cuda_fail(e, "merged pass tables");
      }
      list.push_back(m);
    }
    std::stable_sort(list.begin(), list.end(), [](const MergedPass& a, const MergedPass& b) { return a.floats > b.floats; });
    r->merged.insert(r->merged.end(), list.begin(), list.end());
  }
  return BRIDCT_OK;
}

int launch_merged(bridct_ragged* r, const MergedPass& m, const float* x, float* y, cudaStream_t st) {
  const int li = lg(m.len);
  UnitLauncher fn = m.col ? r->dev->col_units[li][m.mode] : r->dev->row_units[li][m.mode];
  if (!fn) {
    set_error("ragged: no merged pass for this length");
    return BRIDCT_INVALID_ARGUMENT;
  }
  // the line tables of the pass's own axis (the other axis's are not read)
  LineTables tab{r->dev->tables(m.len), r->dev->tables(m.len)};
  // column passes read x and write y; row passes transform y in place
  cudaError_t e = fn(m.col ? x : y, y, m.d_units, m.n, st, tab, r->dev->launch);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "merged pass launch");
}

// One class as its own plain-form launch over the class's offset table.
int launch_class(bridct_ragged* r, const RaggedClass& c, int schedule, const float* x, float* y, cudaStream_t st) {
  BatchLayout l;
  l.offs = c.d_offs;
  l.ld = c.w;
  l.small_units = schedule == BRIDCT_RAGGED_CLASS_LAUNCH_SMALL;
  return launch_plain_layout(r->dev, c.h, c.w, c.mode, x, y, (long long)c.arrays.size(), &l, &l, st);
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
  t->lookahead = 32;   // measured on the 4096-array mixed batch: 2 -> 16 -> 32 = 2.65 -> 2.26 -> 2.24 ms
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
  if (build_classes(r) != BRIDCT_OK) {
    bridct_ragged_destroy(r);
    return nullptr;
  }
  build_units(r);
  cudaError_t e = cudaMalloc((void**)&r->d_counters, (count + 1) * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&r->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(r->d_err, 0, sizeof(int));
  if (e != cudaSuccess || upload(r) != BRIDCT_OK) {
    if (e != cudaSuccess) cuda_fail(e, "bridct_ragged_create");
    bridct_ragged_destroy(r);
    return nullptr;
  }
  const int bps = kernel_setup(reinterpret_cast<const void*>(k_ragged), kRaggedSmem, kRaggedThreads);
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
  for (RaggedClass& c : r->classes) cudaFree(c.d_offs);
  free_merged(r);
  for (int i = 0; i < kRaggedMaxStreams; ++i) {
    if (r->aux[i]) cudaStreamDestroy(r->aux[i]);
    if (r->join_ev[i]) cudaEventDestroy(r->join_ev[i]);
    if (r->mid_ev[i]) cudaEventDestroy(r->mid_ev[i]);
  }
  if (r->fork_ev) cudaEventDestroy(r->fork_ev);
  if (r->mid_fork) cudaEventDestroy(r->mid_fork);
  delete r;
}

BRIDCT_API size_t bridct_ragged_units(const bridct_ragged* r) { return r ? r->units.size() : 0; }

BRIDCT_API int bridct_ragged_apply_device(bridct_ragged* r, const float* x, float* y, void* stream) {
  if (!r || !x || !y) return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = r->span * sizeof(float);
  const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
  if ((a <= b ? b - a : a - b) < bytes) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((a | b) % 16) return BRIDCT_BAD_ALIGNMENT;
  DeviceGuard guard(r->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(batch device)");
  cudaStream_t st = (cudaStream_t)stream;
  // Classes with their own launches run on side streams forked from the caller's stream (largest
  // class first, round robin) and joined back into it; the queue's persistent kernel runs on the
  // caller's stream meanwhile.  Capturable: the fork and join are events on captured streams.
  // MERGED classes run as merged column passes, then (after every column pass has finished) merged
  // row passes, spread over the side streams; classes with their own launches follow on the same
  // streams.
  std::vector<const RaggedClass*> own;
  for (const RaggedClass& c : r->classes)
    if (c.schedule == BRIDCT_RAGGED_CLASS_LAUNCH || c.schedule == BRIDCT_RAGGED_CLASS_LAUNCH_SMALL) own.push_back(&c);
  size_t ncol = 0;
  for (const MergedPass& m : r->merged) ncol += m.col ? 1 : 0;
  const size_t nrow = r->merged.size() - ncol;
  const size_t widest = std::max(own.size(), std::max(ncol, nrow));
  cudaError_t e = cudaSuccess;
  const int nst = std::max(1, std::min(r->streams, (int)widest));
  const bool fork = !own.empty() || !r->merged.empty();
  if (fork) {
    e = cudaEventRecord(r->fork_ev, st);
    for (int i = 0; e == cudaSuccess && i < nst; ++i) e = cudaStreamWaitEvent(r->aux[i], r->fork_ev, 0);
    if (e != cudaSuccess) return cuda_fail(e, "ragged fork");
  }
  if (!r->merged.empty()) {
    for (size_t k = 0; k < ncol; ++k) {
      const int s = launch_merged(r, r->merged[k], x, y, r->aux[k % nst]);
      if (s) return s;
    }
    // every row block needs its array's column strips: all side streams meet here
    for (int i = 1; e == cudaSuccess && i < nst; ++i) {
      e = cudaEventRecord(r->mid_ev[i], r->aux[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(r->aux[0], r->mid_ev[i], 0);
    }
    if (e == cudaSuccess) e = cudaEventRecord(r->mid_fork, r->aux[0]);
    for (int i = 1; e == cudaSuccess && i < nst; ++i) e = cudaStreamWaitEvent(r->aux[i], r->mid_fork, 0);
    if (e != cudaSuccess) return cuda_fail(e, "ragged merged barrier");
    for (size_t k = 0; k < nrow; ++k) {
      const int s = launch_merged(r, r->merged[ncol + k], x, y, r->aux[k % nst]);
      if (s) return s;
    }
  }
  for (size_t k = 0; k < own.size(); ++k) {
    const int s = launch_class(r, *own[k], own[k]->schedule, x, y, r->aux[k % nst]);
    if (s) return s;
  }
  if (!r->units.empty()) {
    e = cudaMemsetAsync(r->d_counters, 0, (r->items.size() + 1) * sizeof(unsigned int), st);
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
    args.spin_limit = r->spin_limit;
    for (int i = 0; i < 4; ++i) args.tab[i] = r->dev->fourstep[i];
    k_ragged<<<r->grid, kRaggedThreads, kRaggedSmem, st>>>(args);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_ragged launch");
  }
  for (int i = 0; fork && i < nst; ++i) {
    e = cudaEventRecord(r->join_ev[i], r->aux[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, r->join_ev[i], 0);
    if (e != cudaSuccess) return cuda_fail(e, "ragged join");
  }
  return BRIDCT_OK;
}

BRIDCT_API size_t bridct_ragged_class_count(const bridct_ragged* r) { return r ? r->classes.size() : 0; }

BRIDCT_API size_t bridct_ragged_launch_count(const bridct_ragged* r) {
  if (!r) return 0;
  size_t n = r->merged.size() + (r->units.empty() ? 0 : 1);
  for (const RaggedClass& c : r->classes)
    if (c.schedule == BRIDCT_RAGGED_CLASS_LAUNCH || c.schedule == BRIDCT_RAGGED_CLASS_LAUNCH_SMALL)
      n += c.h * c.w <= 16384 || whole_array_route(c.h, c.w, c.mode) ? 1 : 2;
  return n;
}

BRIDCT_API int bridct_ragged_class_info(const bridct_ragged* r, size_t cls, int* height, int* width, int* mode,
                                        size_t* arrays, int* schedule) {
  if (!r || cls >= r->classes.size()) return BRIDCT_INVALID_ARGUMENT;
  const RaggedClass& c = r->classes[cls];
  if (height) *height = c.h;
  if (width) *width = c.w;
  if (mode) *mode = c.mode;
  if (arrays) *arrays = c.arrays.size();
  if (schedule) *schedule = c.schedule;
  return BRIDCT_OK;
}

BRIDCT_API int bridct_ragged_set_schedule(bridct_ragged* r, const int* schedules, size_t count, int streams) {
  if (!r || count != r->classes.size() || (count && !schedules) || streams < 1 || streams > kRaggedMaxStreams)
    return BRIDCT_INVALID_ARGUMENT;
  for (size_t i = 0; i < count; ++i) {
    if (schedules[i] < BRIDCT_RAGGED_QUEUE || schedules[i] > BRIDCT_RAGGED_MERGED) {
      set_error("bridct_ragged_set_schedule: unknown schedule " + std::to_string(schedules[i]));
      return BRIDCT_INVALID_ARGUMENT;
    }
    const RaggedClass& c = r->classes[i];
    if (schedules[i] == BRIDCT_RAGGED_MERGED && !two_pass_route(c.h, c.w, c.mode)) {
      set_error("bridct_ragged_set_schedule: class " + std::to_string(i) + " is not a two-pass shape");
      return BRIDCT_INVALID_ARGUMENT;
    }
  }
  DeviceGuard guard(r->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(batch device)");
  cudaError_t e = cudaDeviceSynchronize();   // the old queue may still be in use
  if (e != cudaSuccess) return cuda_fail(e, "bridct_ragged_set_schedule");
  for (size_t i = 0; i < count; ++i) r->classes[i].schedule = schedules[i];
  r->streams = streams;
  build_units(r);
  int s = upload(r);
  if (!s) s = build_merged(r);
  if (s) return s;
  const int bps = kernel_setup(reinterpret_cast<const void*>(k_ragged), kRaggedSmem, kRaggedThreads);
  r->grid = (int)std::min<long long>((long long)r->dev->sm_count * std::max(1, bps),
                                     std::max<size_t>(1, r->units.size()));
  return BRIDCT_OK;
}

BRIDCT_API int bridct_ragged_apply_class_device(bridct_ragged* r, size_t cls, int schedule, const float* x, float* y,
                                                void* stream) {
  if (!r || !x || !y || cls >= r->classes.size() ||
      (schedule != BRIDCT_RAGGED_CLASS_LAUNCH && schedule != BRIDCT_RAGGED_CLASS_LAUNCH_SMALL))
    return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = r->span * sizeof(float);
  const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
  if ((a <= b ? b - a : a - b) < bytes) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((a | b) % 16) return BRIDCT_BAD_ALIGNMENT;
  DeviceGuard guard(r->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(batch device)");
  return launch_class(r, r->classes[cls], schedule, x, y, (cudaStream_t)stream);
}

BRIDCT_API int bridct_ragged_set_wait_limit(bridct_ragged* r, unsigned polls) {
  if (!r) return BRIDCT_INVALID_ARGUMENT;
  r->spin_limit = polls;
  return BRIDCT_OK;
}

BRIDCT_API int bridct_ragged_timeout_flag(bridct_ragged* r) {
  if (!r) return 0;
  DeviceGuard guard(r->device);
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
  DeviceGuard guard(r->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(batch device)");
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

// ---- Ragged batch without any allocation ---------------------------------------------------
//
// Some callers cannot let a library allocate device memory: a framework whose caching
// allocator owns every byte of the GPU (any cudaMalloc outside it can fail or fragment its
// pool), a latency-bound loop where cudaMalloc/cudaFree's implicit device synchronisation is
// not acceptable, or an embedding that fixes the process's device footprint at start-up.
// bridct_ragged_apply_noalloc serves them: the caller passes the item list and the input and
// output buffers, and everything else the persistent kernel needs (work queue, per-array
// counters, error word, four-step tables) lives in one statically sized __device__ array below,
// which every GPU that loads this library holds until the process exits.  The host side builds
// the queue in static buffers as well, so a successful call allocates nothing.
namespace {

constexpr int kNaMaxArrays = 4096;    // items per call
constexpr int kNaMaxUnits = 49152;    // work units per call (default unit geometry)
constexpr int kNaTw = 17 * (4 + 8 + 16 + 32);     // float2 twiddles, N = 128..1024
constexpr int kNaPost = 17 * (4 + 8 + 16 + 32);   // float4 post coefficients, N = 128..1024

struct NaOff {
  static constexpr size_t arrays = 0;
  static constexpr size_t units = arrays + sizeof(bridct::RaggedArray) * kNaMaxArrays;
  static constexpr size_t counters = units + sizeof(bridct::RaggedUnit) * kNaMaxUnits;
  static constexpr size_t err = counters + sizeof(unsigned int) * (kNaMaxArrays + 1);
  static constexpr size_t tw = (err + sizeof(int) + 255) / 256 * 256;
  static constexpr size_t post = tw + sizeof(float2) * kNaTw;
  static constexpr size_t bytes = post + sizeof(float4) * kNaPost;
};
static_assert(NaOff::post % 16 == 0, "post table alignment");

}  // namespace

// About 0.9 MB: queue (arrays, units), counters, error word, four-step tables.  Host code must
// not use this name as a device address; the entry point resolves it per device below.
static __device__ __align__(256) unsigned char g_ragged_scratch[NaOff::bytes];

namespace {

std::mutex g_na_mutex;                                  // one call at a time (shared scratch)
bridct::RaggedArray g_na_arrays[kNaMaxArrays];
bridct::RaggedUnit g_na_units[kNaMaxUnits];
int g_na_big[kNaMaxArrays];
int g_na_small[kNaMaxArrays];
int g_na_order[kNaMaxArrays];
float2 g_na_tw[kNaTw];
float4 g_na_post[kNaPost];
bool g_na_tables = false;
unsigned char* g_na_addr[64] = {};                      // scratch address per device

int na_segment(int i) { return 17 * ((4 << i) - 4); }  // first entry of N = 128 << i

}  // namespace

extern "C" BRIDCT_API int bridct_ragged_apply_noalloc(const bridct_ragged_item* items, size_t count,
                                                      const float* input, float* output, void* stream) {
  using namespace bridct;
  if (!items || !input || !output || count == 0) return BRIDCT_INVALID_ARGUMENT;
  if (count > (size_t)kNaMaxArrays) {
    set_error("bridct_ragged_apply_noalloc: at most 4096 arrays per call");
    return BRIDCT_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  // validation (as bridct_ragged_create): shapes, modes, 16-byte aligned offsets, no overlap
  size_t span = 0;
  for (size_t i = 0; i < count; ++i) {
    const bridct_ragged_item& it = items[i];
    if (!bridct_supported(it.height, it.width) || it.mode < 0 || it.mode > 2 || it.offset % 4) {
      set_error("bridct_ragged_apply_noalloc: unsupported shape or mode, or misaligned offset");
      return BRIDCT_INVALID_ARGUMENT;
    }
    span = std::max(span, it.offset + (size_t)it.height * it.width);
    g_na_order[i] = (int)i;
  }
  std::sort(g_na_order, g_na_order + count, [&](int a, int b) {
    return items[a].offset != items[b].offset ? items[a].offset < items[b].offset : a < b;
  });
  for (size_t i = 1; i < count; ++i) {
    const bridct_ragged_item& p = items[g_na_order[i - 1]];
    if (items[g_na_order[i]].offset < p.offset + (size_t)p.height * p.width) {
      set_error("bridct_ragged_apply_noalloc: arrays overlap");
      return BRIDCT_INVALID_ARGUMENT;
    }
  }
  const uintptr_t xa = (uintptr_t)input, ya = (uintptr_t)output;
  if ((xa <= ya ? ya - xa : xa - ya) < span * sizeof(float)) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((xa | ya) % 16) return BRIDCT_BAD_ALIGNMENT;

  // work queue with the default unit geometry (same units as bridct_ragged_create)
  bridct_ragged_tuning t;
  bridct_ragged_default_tuning(&t);
  int nbig = 0, nsmall = 0;
  for (size_t i = 0; i < count; ++i) {
    const bridct_ragged_item& it = items[i];
    RaggedArray a{(long long)it.offset, it.height, it.width, it.mode, 0};
    if ((long long)it.height * it.width <= t.tile_floats) {
      g_na_small[nsmall++] = (int)i;
    } else {
      a.nstrips = it.width / strip_cols(it.height, it.width, t.strip_floats);
      g_na_big[nbig++] = (int)i;
    }
    g_na_arrays[i] = a;
  }
  auto size_desc = [&](int a, int b) {
    const long long ea = (long long)items[a].height * items[a].width;
    const long long eb = (long long)items[b].height * items[b].width;
    return ea != eb ? ea > eb : a < b;
  };
  std::sort(g_na_big, g_na_big + nbig, size_desc);
  std::sort(g_na_small, g_na_small + nsmall, size_desc);
  int nunits = 0;
  bool full = false;
  auto push = [&](RaggedUnit u) {
    if (nunits == kNaMaxUnits) full = true;
    else g_na_units[nunits++] = u;
  };
  for (int k = 0; k < nbig + t.lookahead; ++k) {
    if (k < nbig) {
      const RaggedArray& a = g_na_arrays[g_na_big[k]];
      const int tc = a.w / a.nstrips;
      for (int s = 0; s < a.nstrips; ++s) push(RaggedUnit{g_na_big[k], UNIT_COLSTRIP, s * tc, tc});
    }
    if (k >= t.lookahead) {
      const int i = g_na_big[k - t.lookahead];
      const RaggedArray& a = g_na_arrays[i];
      const int rb = block_rows(a.h, a.w, t.row_floats);
      for (int r0 = 0; r0 < a.h; r0 += rb) push(RaggedUnit{i, UNIT_ROWBLOCK, r0, rb});
    }
  }
  for (int k = 0; k < nsmall; ++k) push(RaggedUnit{g_na_small[k], UNIT_TILE, 0, 0});
  if (full) {
    set_error("bridct_ragged_apply_noalloc: the batch needs more than 49152 work units");
    return BRIDCT_INVALID_ARGUMENT;
  }

  // set-up, once per device, with that device current: resolve the scratch array's device
  // address (the host-side name is only a stand-in) and upload the four-step tables into it
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) {
    set_error("bridct_ragged_apply_noalloc: device index beyond 63");
    return BRIDCT_INVALID_ARGUMENT;
  }
  if (!g_na_tables) {
    for (int i = 0; i < 4; ++i) fill_fourstep_tables(128 << i, g_na_tw + na_segment(i), g_na_post + na_segment(i));
    g_na_tables = true;
  }
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ragged_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_ragged_scratch)");
    unsigned char* base = static_cast<unsigned char*>(p);
    e = cudaMemcpy(base + NaOff::tw, g_na_tw, sizeof(g_na_tw), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + NaOff::post, g_na_post, sizeof(g_na_post), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "scratch tables");
    g_na_addr[dev] = base;
  }
  const int bps = kernel_setup(reinterpret_cast<const void*>(k_ragged), kRaggedSmem, kRaggedThreads);
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess || bps <= 0) return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidConfiguration, "k_ragged");
  unsigned char* base = g_na_addr[dev];
  cudaStream_t st = (cudaStream_t)stream;
  // The scratch keeps the previous call's contents: queue tables are overwritten, and the
  // counters and error word are cleared before the launch.
  e = cudaMemcpyAsync(base + NaOff::arrays, g_na_arrays, count * sizeof(RaggedArray), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + NaOff::units, g_na_units, (size_t)nunits * sizeof(RaggedUnit), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + NaOff::counters, 0, (count + 1) * sizeof(unsigned int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + NaOff::err, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "scratch upload");
  RaggedArgs args;
  args.x = input;
  args.y = output;
  args.arrays = reinterpret_cast<const RaggedArray*>(base + NaOff::arrays);
  args.units = reinterpret_cast<const RaggedUnit*>(base + NaOff::units);
  args.nunits = nunits;
  args.next = reinterpret_cast<unsigned int*>(base + NaOff::counters);
  args.done = args.next + 1;
  args.err = reinterpret_cast<int*>(base + NaOff::err);
  args.spin_limit = kRaggedSpin;
  for (int i = 0; i < 4; ++i) {
    args.tab[i].tw = reinterpret_cast<const float2*>(base + NaOff::tw) + na_segment(i);
    args.tab[i].post = reinterpret_cast<const float4*>(base + NaOff::post) + na_segment(i);
  }
  const int grid = (int)std::min<long long>((long long)sms * bps, nunits);
  k_ragged<<<grid, kRaggedThreads, kRaggedSmem, st>>>(args);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "k_ragged launch");
  // Synchronous: the shared scratch is free again when the call returns.
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "bridct_ragged_apply_noalloc");
  int flag = 0;
  e = cudaMemcpy(&flag, base + NaOff::err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "error word");
  return flag ? BRIDCT_TIMEOUT : BRIDCT_OK;
}
