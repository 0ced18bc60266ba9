// Batching form: one persistent launch over a mixed-shape, mixed-direction batch.
//
// The host turns the batch into a queue of work units:
//   TILE      one array with h*w <= 16384: both passes in shared memory (as k_full)
//   COLSTRIP  h rows x TC columns of a larger array: its column lines, x -> y
//   ROWBLOCK  RB full rows of a larger array: its row lines, y -> y in place
// CTAs are persistent (one launch, grid = SMs x resident CTAs) and take units in queue order
// from an atomic counter.  A ROWBLOCK of array i needs every COLSTRIP of array i finished: each
// strip adds 1 to done[i] after a __threadfence, and the row block spins on done[i] with a
// bounded budget (nanosleep back-off).  Column strips never wait, and every unit that a waiting
// row block depends on was dequeued earlier by a running CTA, so the wait always ends; on budget
// expiry the unit is skipped and the error flag set instead (the host reports BRIDCT_TIMEOUT).
// Line lengths and modes vary per unit and are dispatched at run time to the same generated
// straight-line SJ programs and four-step lines as the fixed-shape kernels.
#pragma once
#include "sj_kernels.cuh"

namespace bridct {

enum UnitType { UNIT_TILE = 0, UNIT_COLSTRIP = 1, UNIT_ROWBLOCK = 2 };

struct RaggedArray {
  long long offset;   // first float of the array in x and y
  int h, w, mode;
  int nstrips;        // column strips of a two-pass array (0 for tile arrays)
};

struct RaggedUnit {
  int array;
  int type;
  int first;          // first column (COLSTRIP) or first row (ROWBLOCK)
  int count;          // columns or rows covered
};

struct RaggedArgs {
  const float* x;
  float* y;
  const RaggedArray* arrays;
  const RaggedUnit* units;
  int nunits;
  unsigned int* next;       // queue head (zeroed before the launch)
  unsigned int* done;       // finished column strips per array (zeroed before the launch)
  int* err;
  unsigned spin_limit;      // polls of a row block's dependency wait before it gives up
  FourStepTables tab[4];    // N = 128, 256, 512, 1024
};

constexpr int kRaggedThreads = 256;                                 // 2 CTAs per SM at <= 128 registers
// Exchange floats per warp, worst case over the four-step widths G = 4..32 (G = 4 and 8 need
// most: 8 slots of 84 or 4 slots of 168 floats, re and im).
constexpr int kXbufPerWarp = cmax(cmax(FourStepSizes<4>::FLOATS, FourStepSizes<8>::FLOATS),
                                  cmax(FourStepSizes<16>::FLOATS, FourStepSizes<32>::FLOATS));
constexpr int kRaggedXbuf = (kRaggedThreads / 32) * kXbufPerWarp;
constexpr int kRaggedTile = 16384 + 1024;                           // worst-case tile floats (odd pitch)
constexpr int kRaggedSmem = (kRaggedTile + kRaggedXbuf) * 4;
constexpr unsigned kRaggedSpin = 1u << 22;                          // x ~256 ns back-off

// Line l of a unit starts at tile + l * s (s = 1 for columns, the pitch for rows).
struct StrideOff {
  int s;
  __device__ __forceinline__ int operator()(int l) const { return l * s; }
};

__device__ __forceinline__ FourStepTables pick_tables(const RaggedArgs& a, int n) {
  return n >= 1024 ? a.tab[3] : n >= 512 ? a.tab[2] : n >= 256 ? a.tab[1] : a.tab[0];
}

// Runtime dispatch of run_lines over the line length and mode.
__device__ __forceinline__ void lines_dyn(int n, int mode, float* tile, int nlines, int es, StrideOff off,
                                       float* xbuf, FourStepTables t) {
#define BRIDCT_LINES_N(N)                                                          \
  case N:                                                                          \
    if (mode == LM_FWD) run_lines<N, LM_FWD>(tile, nlines, es, off, xbuf, t);      \
    else if (mode == LM_INV) run_lines<N, LM_INV>(tile, nlines, es, off, xbuf, t); \
    else run_lines<N, LM_RT>(tile, nlines, es, off, xbuf, t);                      \
    break;
  switch (n) {
    BRIDCT_LINES_N(8)
    BRIDCT_LINES_N(16)
    BRIDCT_LINES_N(32)
    BRIDCT_LINES_N(64)
    BRIDCT_LINES_N(128)
    BRIDCT_LINES_N(256)
    BRIDCT_LINES_N(512)
    BRIDCT_LINES_N(1024)
    default: break;
  }
#undef BRIDCT_LINES_N
}

// Shared-memory pitch of a unit's block (rows x cols): aligned (cols + 4, float4 staging)
// unless a column pass of 512- or 1024-point lines runs on it (their four-step groups put
// every lane in one bank at an aligned pitch) or the aligned block would not fit the tile.
__device__ __forceinline__ int ragged_pitch(int rows, int cols, bool column_pass, int h) {
  if ((column_pass && h >= 512) || rows * (cols + 4) > kRaggedTile) return cols + 1;
  return cols + 4;
}

// Loads rows x cols floats (row pitch gp in global) into shared memory (pitch P).  The copies are
// asynchronous (cp.async), so a thread has all of its share of the block in flight at once; the
// caller's __syncthreads after this call publishes the block.  An odd-pitch block copies 4-byte
// elements (its rows are not 16-byte aligned), except when it must bypass L1 (row blocks read data
// that other CTAs wrote in this launch; 4-byte cp.async always goes through L1), where it loads
// through L2 synchronously.
__device__ __forceinline__ void load_block(const float* g, long long gp, int rows, int cols, float* s, int P,
                                           bool bypass_l1) {
  const int q = cols >> 2;
  const bool vec = (P & 3) == 0;
  if (vec || !bypass_l1) {
    for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
      const int r = i / q, c = (i % q) * 4;
      const float* src = g + r * gp + c;
      float* d = s + r * P + c;
      if (vec) {
        cp_async16(d, src);
      } else {
        cp_async4(d, src);
        cp_async4(d + 1, src + 1);
        cp_async4(d + 2, src + 2);
        cp_async4(d + 3, src + 3);
      }
    }
    cp_async_wait_all();
    return;
  }
  for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
    const int r = i / q, c = (i % q) * 4;
    const float4* p = reinterpret_cast<const float4*>(g + r * gp + c);
    const float4 v = bypass_l1 ? __ldcg(p) : __ldg(p);
    float* d = s + r * P + c;
    if (vec) {
      *reinterpret_cast<float4*>(d) = v;
    } else {
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
  }
}

__device__ __forceinline__ void store_block(float* g, long long gp, int rows, int cols, const float* s, int P) {
  const int q = cols >> 2;
  const bool vec = (P & 3) == 0;
  for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
    const int r = i / q, c = (i % q) * 4;
    const float* v = s + r * P + c;
    *reinterpret_cast<float4*>(g + r * gp + c) =
        vec ? *reinterpret_cast<const float4*>(v) : make_float4(v[0], v[1], v[2], v[3]);
  }
}

__global__ void __launch_bounds__(kRaggedThreads, 2) k_ragged(RaggedArgs a) {
  extern __shared__ float smem[];
  float* tile = smem;
  float* xbuf = smem + kRaggedTile;
  __shared__ int s_unit;
  __shared__ int s_ok;
  for (;;) {
    if (threadIdx.x == 0) s_unit = (int)atomicAdd(a.next, 1u);
    __syncthreads();
    const int u = s_unit;
    if (u >= a.nunits) break;
    const RaggedUnit unit = a.units[u];
    const RaggedArray arr = a.arrays[unit.array];
    const int h = arr.h, w = arr.w, mode = arr.mode;
    const float* xa = a.x + arr.offset;
    float* ya = a.y + arr.offset;
    if (unit.type == UNIT_TILE) {
      const int P = ragged_pitch(h, w, true, h);
      load_block(xa, w, h, w, tile, P, false);
      __syncthreads();
      lines_dyn(h, mode, tile, w, P, StrideOff{1}, xbuf, pick_tables(a, h));
      __syncthreads();
      lines_dyn(w, mode, tile, h, 1, StrideOff{P}, xbuf, pick_tables(a, w));
      __syncthreads();
      store_block(ya, w, h, w, tile, P);
    } else if (unit.type == UNIT_COLSTRIP) {
      const int tc = unit.count, P = ragged_pitch(h, tc, true, h);
      load_block(xa + unit.first, w, h, tc, tile, P, false);
      __syncthreads();
      lines_dyn(h, mode, tile, tc, P, StrideOff{1}, xbuf, pick_tables(a, h));
      __syncthreads();
      store_block(ya + unit.first, w, h, tc, tile, P);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicAdd(a.done + unit.array, 1u);
    } else {
      if (threadIdx.x == 0) {
        int ok = 0;
        for (unsigned i = 0; i < a.spin_limit; ++i) {
          if (atomicAdd(a.done + unit.array, 0u) >= (unsigned)arr.nstrips) {
            ok = 1;
            break;
          }
          __nanosleep(256);
        }
        if (!ok) atomicExch(a.err, 2);
        __threadfence();
        s_ok = ok;
      }
      __syncthreads();
      if (s_ok) {
        const int rb = unit.count, P = ragged_pitch(rb, w, false, 0);
        float* ga = ya + (long long)unit.first * w;
        load_block(ga, w, rb, w, tile, P, true);
        __syncthreads();
        lines_dyn(w, mode, tile, rb, 1, StrideOff{P}, xbuf, pick_tables(a, w));
        __syncthreads();
        store_block(ga, w, rb, w, tile, P);
      }
    }
    __syncthreads();
  }
}

}  // namespace bridct
