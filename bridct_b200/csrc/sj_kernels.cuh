// 2D kernels of the plain (Shao-Johnson FP32) form.
//
// Shape classes (h, w powers of two in [8, 1024]):
//   h*w <= 16384  "tile"    k_full<..., DO_COL=1, DO_ROW=1>: a CTA loads A whole arrays
//                           (A*h*w ~ 8192 floats) into shared memory with coalesced float4
//                           loads, runs every column line, then every row line, and stores.
//                           One HBM read and one HBM write per element.
//   h*w >  16384  "2-pass"  k_colstrip (h rows x TC columns per CTA, column lines, x -> y)
//                           then k_full<DO_COL=0> (TR full rows per CTA, row lines, y -> y in
//                           place), one launch each over the whole batch.  The intermediate
//                           lives in y (the reference's rect route does the same pair of
//                           passes, vertical then bands, src/generated/rect.c:5-23).
//                           A 32768-float array runs as one whole-array tile instead (one CTA
//                           per SM) in the modes where that measured faster (plain_launch.cuh).
// Shared-memory rows are padded (pitch_of, strip_pitch, rowblock_pitch) so that the line walks
// of both passes stay free of most bank conflicts.
#pragma once
#include "sj_lines.cuh"

namespace bridct {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileFloats = 8192;   // target floats per CTA tile for small arrays
// Longest line run as one thread's straight-line program for a pass of N-point lines whose
// array has `other` points on the other axis.  128-point register lines (168 registers, no
// spills) measured +12-59% over the four-step on 128x128, the two-pass shapes and forward /
// inverse tiles with a short other axis, and -6..-28% on tiles mixing them with 64-point lines
// in forward / inverse.  Round trips of tiles with a 128-point axis take them too, in 128-thread
// CTAs (launch_plain): +3..30% over the four-step (128x8 alone -3%).
__host__ __device__ constexpr int reg_line_max(int N, int other, int mode, bool two_pass) {
  return N == 128 && (two_pass || other >= 128 || mode == LM_RT || other <= 32) ? 128 : 64;
}

struct LineTables {
  FourStepTables col;   // for line length h (used when h >= 128)
  FourStepTables row;   // for line length w (used when w >= 128)
};

// Where the arrays of a launch live in a general layout (kernels instantiated with GEN): array b
// starts at offs[b] when an offset table is given (the shape classes of a ragged batch), else at
// b * bs (a strided batch), and its rows are ld floats apart.  Array starts and ld are multiples of
// 4 floats, so every row is 16-byte aligned.  Contiguous batches (array b at b*h*w, rows w apart)
// use the kernels' fixed addressing instead.
struct BatchLayout {
  const long long* offs = nullptr;
  long long bs = 0;
  long long ld = 0;
  int small_units = 0;   // two-pass shapes: force the few-array geometry (one line group per warp)
};

// One unit of a merged launch (UNITS kernels): a column strip or a row block of some array of a
// ragged batch, starting `off` floats into both x and y, rows `ld` floats apart.  A merged column
// launch covers strips of arrays that share the column length but not the width; a merged row
// launch covers row blocks of arrays that share the row length but not the height.
struct PassUnit {
  long long off;
  long long ld;
};

struct TileArgs {
  const float* x;
  float* y;
  long long ntiles;
  long long rows_total;   // rows of the (batch*h) x w matrix covered by this launch
  LineTables tab;
  BatchLayout lx, ly;     // layouts of x and y (GEN kernels only)
  const PassUnit* units = nullptr;   // UNITS kernels: one unit per tile
};

// Offset (floats) of row g of the (batch*H) x W row matrix in a general layout.
template <int H>
__device__ __forceinline__ long long layout_row(const BatchLayout& l, long long g) {
  const long long b = g / H;
  const int r = (int)(g % H);
  return (l.offs ? __ldg(l.offs + b) : b * l.bs) + (long long)r * l.ld;
}

template <int N> struct ExchangeFloats { static constexpr int value = 0; };
template <> struct ExchangeFloats<128> { static constexpr int value = FourStepSizes<4>::FLOATS; };
template <> struct ExchangeFloats<256> { static constexpr int value = FourStepSizes<8>::FLOATS; };
template <> struct ExchangeFloats<512> { static constexpr int value = FourStepSizes<16>::FLOATS; };
template <> struct ExchangeFloats<1024> { static constexpr int value = FourStepSizes<32>::FLOATS; };

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int round4(int a) { return (a + 3) & ~3; }

// Floats of one line length's four-step tables in shared memory (post first: float4 aligned).
template <int N> struct TableFloats {
  static constexpr int G = N / 32;
  static constexpr int value = N >= 128 ? 17 * G * 4 + round4(17 * G * 2) : 0;
};

// Copies the four-step tables of line length N into shared memory at s (16-byte aligned);
// returns tables that point there.  The caller synchronizes before first use.
template <int N>
__device__ __forceinline__ FourStepTables stage_tables(FourStepTables g, float* s) {
  if constexpr (N < 128) {
    return g;
  } else {
    constexpr int G = N / 32;
    float4* post = reinterpret_cast<float4*>(s);
    float2* tw = reinterpret_cast<float2*>(s + 17 * G * 4);
    for (int i = threadIdx.x; i < 17 * G; i += blockDim.x) {
      post[i] = __ldg(g.post + i);
      tw[i] = __ldg(g.tw + i);
    }
    return FourStepTables{tw, post};
  }
}

// Shared-memory row pitch (floats).  A 16-byte aligned pitch (w + 4) lets the tile be staged
// with 128-bit accesses and costs no extra bank conflicts in the line walks, except for column
// four-step lines with G >= 16 (h >= 512), whose stage-1 reads need an odd pitch (w + 1).
__host__ __device__ constexpr bool odd_pitch(int h, bool has_col) { return has_col && h >= 512; }
__host__ __device__ constexpr int pitch_of(int h, int w, bool has_col) { return odd_pitch(h, has_col) ? w + 1 : w + 4; }
// Pitches of the two-pass kernels, whose long lines all run the four-step.  Chosen with a bank
// model of the four-step's shared-memory accesses (Makhoul gather, post-rotation stores, exchange):
// a column strip of 256-point lines with pitch tc + 2 (= 2 mod 4) and row blocks of 256- and
// 512-point lines with pitch w + 8 (= 8 mod 32) and w + 16 (= 16 mod 32) need 20%, 23% and 14%
// fewer wavefronts per line than with pitch + 4; tc + 2 rows are staged with 64-bit accesses.
// 32-column strips of 512-point lines take pitch 34: as few wavefronts as the odd pitch 33, and an
// even pitch lets tile_load copy asynchronously.
__host__ __device__ constexpr int strip_pitch(int h, int tc) {
  return h == 256 || (h == 512 && tc == 32) ? tc + 2 : pitch_of(h, tc, true);
}
__host__ __device__ constexpr int rowblock_pitch(int w) { return w == 256 ? w + 8 : w == 512 ? w + 16 : w + 4; }
// Row pitch of a whole-array tile.  Where one axis runs the four-step and the other register lines,
// the four-step axis takes the two-pass kernels' bank-model pitch: 256-point columns w + 2, 256- and
// 512-point rows w + 8 and w + 16 (per line group 142, 174 and 190 wavefronts against 206, 270 and
// 222 at w + 4; tests/test_bank_model.py).  Shapes with four-step lines on both axes (256 x 128,
// 128 x 256) keep w + 4, which the model counts as good or better for the two walks together.
__host__ __device__ constexpr int tile_pitch(int h, int w) {
  return h == 256 && w <= 64 ? w + 2 : w == 256 && h <= 64 ? w + 8 : w == 512 && h <= 64 ? w + 16 : pitch_of(h, w, true);
}
// Array pitch in a whole-array tile.  With pitch w + 4, h * (w + 4) is a multiple of 32 floats for
// every shape, so the register-line column walks of the 4 (w = 8) or 2 (w = 16) arrays that a
// warp's 32 lines span share banks (4- and 2-way conflicts; the tile kernel of 32 x 8 arrays spent
// most of its time in mio_throttle stalls).  Arrays of 8 columns up to 128 high and of 16 columns
// up to 64 high are padded to 8 and 16 (mod 32) floats apart instead: 16..64 x 8 +16..26%,
// 128 x 8 +8..12%, 8..32 x 16 +5..11%, 64 x 16 +4% (same-box A/B, all modes).  128 x 16 (-5%
// forward) and the taller four-step shapes (-1..2%) keep the plain layout.
__host__ __device__ constexpr int tile_array_pitch(int h, int w, int p) {
  return w == 8 && h <= 128 ? h * p + (40 - (h * p) % 32) % 32
                            : w == 16 && h <= 64 ? h * p + (48 - (h * p) % 32) % 32 : h * p;
}
// Shared-memory offset of row r of a tile whose rows come in groups of AH (one array each), AP
// floats apart, and P floats apart within a group (AH = 1, AP = P: every row P apart).
template <int P, int AH, int AP>
__device__ __forceinline__ int tile_row(int r) {
  return AH == 1 ? r * AP : (r / AH) * AP + (r % AH) * P;
}

// Asynchronous global -> shared copies (cp.async; 16 bytes through L2 only, 8 and 4 bytes through
// L1).  The issuing thread waits with cp_async_wait_all; a barrier then publishes the data.
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Moves rows x cols floats between global memory (row pitch gp) and the tile (pitch P).  Rows
// from valid_rows on are zero-filled.  With an even pitch the load is asynchronous (cp.async of 16
// or 8 bytes): a thread has its whole share of the tile in flight at once, which measured +4..22%
// on tiles of short lines and +6..12% on 1024-point row passes.  An odd pitch (column passes of
// 512- and 1024-point lines) would need four 4-byte copies per float4, which measured 6-14% slower
// than the synchronous float4 load it keeps.
template <int P, int AH = 1, int AP = P>
__device__ __forceinline__ void tile_load(const float* g, long long gp, int rows, int cols, float* tile,
                                          int valid_rows) {
  const int q = cols / 4;
  for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
    const int r = i / q, c = (i % q) * 4;
    float* d = tile + tile_row<P, AH, AP>(r) + c;
    if constexpr (P % 2 == 0) {
      if (r < valid_rows) {
        const float* src = g + r * gp + c;
        if constexpr (P % 4 == 0) {
          cp_async16(d, src);
        } else {
          cp_async8(d, src);
          cp_async8(d + 2, src + 2);
        }
      } else {
        d[0] = 0.f; d[1] = 0.f; d[2] = 0.f; d[3] = 0.f;
      }
    } else {
      const float4 v = r < valid_rows ? __ldg(reinterpret_cast<const float4*>(g + r * gp + c))
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
  }
  if constexpr (P % 2 == 0) cp_async_wait_all();
}

// A tile held in registers between its global load and its shared-memory store, so that the
// next tile's loads are in flight while the current tile is transformed (ROWS x COLS floats,
// row pitch P in shared memory; element i of the tile's float4 sequence goes to thread
// i % THREADS).
template <int P, int ROWS, int COLS, int THREADS = kThreads, int AH = 1, int AP = P>
struct TileRegs {
  static constexpr int Q = COLS / 4;
  static constexpr int N = (ROWS * Q + THREADS - 1) / THREADS;
  float4 v[N];
  __device__ __forceinline__ void load(const float* g, long long gp, int valid_rows) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int i = threadIdx.x + k * THREADS;
      if (ROWS * Q % THREADS == 0 || i < ROWS * Q) {
        const int r = i / Q, c = (i % Q) * 4;
        v[k] = r < valid_rows ? __ldg(reinterpret_cast<const float4*>(g + r * gp + c))
                              : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
  // As load, with row r of the tile at rp(r).
  template <typename RowPtr>
  __device__ __forceinline__ void load_rows(const RowPtr& rp, int valid_rows) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int i = threadIdx.x + k * THREADS;
      if (ROWS * Q % THREADS == 0 || i < ROWS * Q) {
        const int r = i / Q, c = (i % Q) * 4;
        v[k] = r < valid_rows ? __ldg(reinterpret_cast<const float4*>(rp(r) + c))
                              : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
  __device__ __forceinline__ void put(float* tile) const {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int i = threadIdx.x + k * THREADS;
      if (ROWS * Q % THREADS == 0 || i < ROWS * Q) {
        const int r = i / Q, c = (i % Q) * 4;
        float* d = tile + tile_row<P, AH, AP>(r) + c;
        if constexpr (P % 4 == 0) {
          *reinterpret_cast<float4*>(d) = v[k];
        } else if constexpr (P % 2 == 0) {
          reinterpret_cast<float2*>(d)[0] = make_float2(v[k].x, v[k].y);
          reinterpret_cast<float2*>(d)[1] = make_float2(v[k].z, v[k].w);
        } else {
          d[0] = v[k].x; d[1] = v[k].y; d[2] = v[k].z; d[3] = v[k].w;
        }
      }
    }
  }
};

// tile_load for tiles whose rows lie anywhere (row r at rp(r), 16-byte aligned).
template <int P, int AH = 1, int AP = P, typename RowPtr>
__device__ __forceinline__ void tile_load_rows(const RowPtr& rp, int rows, int cols, float* tile, int valid_rows) {
  const int q = cols / 4;
  for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
    const int r = i / q, c = (i % q) * 4;
    float* d = tile + tile_row<P, AH, AP>(r) + c;
    if constexpr (P % 2 == 0) {
      if (r < valid_rows) {
        const float* src = rp(r) + c;
        if constexpr (P % 4 == 0) {
          cp_async16(d, src);
        } else {
          cp_async8(d, src);
          cp_async8(d + 2, src + 2);
        }
      } else {
        d[0] = 0.f; d[1] = 0.f; d[2] = 0.f; d[3] = 0.f;
      }
    } else {
      const float4 v = r < valid_rows ? __ldg(reinterpret_cast<const float4*>(rp(r) + c))
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
  }
  if constexpr (P % 2 == 0) cp_async_wait_all();
}

// tile_store for tiles whose rows lie anywhere; rows from valid_rows on are not stored.
template <int P, int AH = 1, int AP = P, typename RowPtr>
__device__ __forceinline__ void tile_store_rows(const RowPtr& rp, int rows, int cols, const float* tile) {
  const int q = cols / 4;
  for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
    const int r = i / q, c = (i % q) * 4;
    const float* sp = tile + tile_row<P, AH, AP>(r) + c;
    float4 v;
    if constexpr (P % 4 == 0) {
      v = *reinterpret_cast<const float4*>(sp);
    } else if constexpr (P % 2 == 0) {
      const float2 lo = reinterpret_cast<const float2*>(sp)[0], hi = reinterpret_cast<const float2*>(sp)[1];
      v = make_float4(lo.x, lo.y, hi.x, hi.y);
    } else {
      v = make_float4(sp[0], sp[1], sp[2], sp[3]);
    }
    *reinterpret_cast<float4*>(rp(r) + c) = v;
  }
}

template <int P, int AH = 1, int AP = P>
__device__ __forceinline__ void tile_store(float* g, long long gp, int rows, int cols, const float* tile) {
  const int q = cols / 4;
  for (int i = threadIdx.x; i < rows * q; i += blockDim.x) {
    const int r = i / q, c = (i % q) * 4;
    const float* sp = tile + tile_row<P, AH, AP>(r) + c;
    float4 v;
    if constexpr (P % 4 == 0) {
      v = *reinterpret_cast<const float4*>(sp);
    } else if constexpr (P % 2 == 0) {
      const float2 lo = reinterpret_cast<const float2*>(sp)[0], hi = reinterpret_cast<const float2*>(sp)[1];
      v = make_float4(lo.x, lo.y, hi.x, hi.y);
    } else {
      v = make_float4(sp[0], sp[1], sp[2], sp[3]);
    }
    *reinterpret_cast<float4*>(g + r * gp + c) = v;
  }
}

// Runs all lines of length N in a set of `nlines` lines; line l starts at tile + off(l),
// elements at stride es.  Register lines (one thread per line) for N <= REG_MAX, warp
// four-step lines above.
// PAIRS: rows (es = 1) at 8-byte aligned starts; the four-step moves them in 64-bit pairs.
template <int N, int MODE, int REG_MAX = 64, bool PAIRS = false, typename Off>
__device__ __forceinline__ void run_lines(float* tile, int nlines, int es, const Off& off,
                                          float* xbuf, FourStepTables tab) {
  if constexpr (N <= REG_MAX) {
    for (int l = threadIdx.x; l < nlines; l += blockDim.x) reg_line<N, MODE>(tile + off(l), es);
  } else {
    constexpr int G = N / 32;
    constexpr int LPW = 32 / G;
    const int warp = threadIdx.x >> 5;
    float* xb = xbuf + warp * FourStepSizes<G>::FLOATS;
    for (int g = warp; g * LPW < nlines; g += blockDim.x >> 5) {
      auto ptr = [&](int j) { return tile + off(g * LPW + j); };
      fs_line<G, MODE, PAIRS>(ptr, es, xb, tab);
    }
  }
}

// Full-width tiles: TR consecutive rows (of width W) of the batch viewed as a (B*H) x W
// matrix.  With DO_COL the tile holds TR/H whole arrays.
template <int H, int W, int TR, bool DO_COL, bool DO_ROW, int MODE, int THREADS = kThreads, bool GEN = false,
          bool UNITS = false>
__global__ void __launch_bounds__(THREADS) k_full(TileArgs a) {
  static_assert(!UNITS || !DO_COL, "merged units are row blocks");
  constexpr int P = DO_COL ? tile_pitch(H, W) : rowblock_pitch(W);
  // whole-array tiles: arrays of H rows, AP floats apart (tile_array_pitch); row blocks: rows P apart
  constexpr int AH = DO_COL ? H : 1;
  constexpr int AP = DO_COL ? tile_array_pitch(H, W, P) : P;
  // Only four-step lines use the exchange buffer and the staged tables; register lines (N up to
  // the pass's reg_line_max) need neither, and the tile launches size shared memory the same way
  // (Geometry::tile_smem).
  constexpr bool kFsCol = DO_COL && H > reg_line_max(H, W, MODE, false);
  constexpr bool kFsRow = DO_ROW && W > reg_line_max(W, H, MODE, !DO_COL);
  constexpr int XB = (THREADS / 32) * cmax(kFsCol ? ExchangeFloats<H>::value : 0, kFsRow ? ExchangeFloats<W>::value : 0);
  extern __shared__ float smem[];
  float* tile = smem;
  float* xbuf = smem + round4((TR / AH) * AP);
  float* tabs = xbuf + round4(XB);
  griddep_wait();
  const FourStepTables tcol = kFsCol ? stage_tables<H>(a.tab.col, tabs) : a.tab.col;
  const FourStepTables trow = kFsRow ? stage_tables<W>(a.tab.row, tabs + (kFsCol ? TableFloats<H>::value : 0))
                                     : a.tab.row;
  // The last tile of a launch may hold fewer than TR rows; it is zero-filled.
  auto rows_of = [&](long long t) {
    const long long left = a.rows_total - t * (long long)TR;
    return left >= TR ? TR : (int)left;
  };
  // Whole-array tiles with a 128..1024-point axis and row passes of 128-point lines prefetch the
  // next tile into registers during the transform (measured +10-50% on such shapes).  Full
  // 16384-float tiles whose rows are the long axis (64x256, 32x512, 16x1024, 64 prefetch floats a
  // thread) and row passes of 256..1024-point lines load with cp.async instead: measured +3-27%
  // and +1-11% over the register prefetch there.  Short-line tiles keep their occupancy, and
  // 128-thread CTAs and whole 32768-float tiles have no registers to spare for it.
  constexpr bool kPrefetch = THREADS == kThreads && TR * W <= 16384 &&
                             (DO_COL ? DO_ROW && (H >= 128 || W >= 128) && !(W >= 256 && TR * W >= 16384)
                                     : (DO_ROW && W == 128));
  // General layouts (GEN): row r of tile t is row t * TR + r of the batch's row matrix.  Merged
  // row blocks (UNITS): row r of tile t is row r of unit t.
  auto xrow = [&](long long t) {
    return [&a, t](int r) {
      return UNITS ? a.x + a.units[t].off + r * a.units[t].ld : a.x + layout_row<H>(a.lx, t * TR + r);
    };
  };
  auto yrow = [&](long long t) {
    return [&a, t](int r) {
      return UNITS ? a.y + a.units[t].off + r * a.units[t].ld : a.y + layout_row<H>(a.ly, t * TR + r);
    };
  };
  constexpr bool kRows = GEN || UNITS;   // per-row addressing
  TileRegs<P, kPrefetch ? TR : 4, kPrefetch ? W : 4, THREADS, AH, AP> next;
  if (kPrefetch && blockIdx.x < a.ntiles) {
    if constexpr (kRows) next.load_rows(xrow(blockIdx.x), rows_of(blockIdx.x));
    else next.load(a.x + blockIdx.x * (long long)TR * W, W, rows_of(blockIdx.x));
  }
  for (long long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    if (t + gridDim.x >= a.ntiles) griddep_trigger();   // this CTA's last tile
    const int rows = rows_of(t);
    if constexpr (kPrefetch) {
      next.put(tile);
      __syncthreads();
      if (t + gridDim.x < a.ntiles) {
        if constexpr (kRows) next.load_rows(xrow(t + gridDim.x), rows_of(t + gridDim.x));
        else next.load(a.x + (t + gridDim.x) * (long long)TR * W, W, rows_of(t + gridDim.x));
      }
    } else {
      if constexpr (kRows) tile_load_rows<P, AH, AP>(xrow(t), TR, W, tile, rows);
      else tile_load<P, AH, AP>(a.x + t * (long long)TR * W, W, TR, W, tile, rows);
      __syncthreads();
    }
    if constexpr (DO_COL) {
      static_assert(TR % H == 0, "column pass needs whole arrays");
      run_lines<H, MODE, reg_line_max(H, W, MODE, false)>(tile, (TR / H) * W, P,
                         [](int l) { return (l / W) * AP + (l % W); }, xbuf, tcol);
      __syncthreads();
    }
    if constexpr (DO_ROW) {
      // Paired 64-bit gathers for 512- and 1024-point rows only: they remove the stride-2 bank
      // conflicts there, while 256-point rows (no fewer wavefronts at their pitch, plus the
      // shuffles) measured 7-12% slower with them.
      run_lines<W, MODE, reg_line_max(W, H, MODE, !DO_COL), P % 2 == 0 && W >= 512>(
          tile, TR, 1, [](int l) { return tile_row<P, AH, AP>(l); }, xbuf, trow);
      __syncthreads();
    }
    if constexpr (kRows) tile_store_rows<P, AH, AP>(yrow(t), rows, W, tile);
    else tile_store<P, AH, AP>(a.y + t * (long long)TR * W, W, rows, W, tile);
    __syncthreads();
  }
}

// Column strips: H rows x TC columns of one array (row pitch W in global memory; ld of the
// layouts with GEN).
// Strips of 1024-point columns (16 wide; 8 wide for calls on a few arrays) and 512-point columns
// (32 wide) are staged transposed: column c of the strip is row c of the tile (pitch
// transposed_pitch), so the column lines run the row-line code instead of a stride-pitch walk down
// the tile, whose stride-2 Makhoul gather is 2-way bank-conflicted at any pitch.  1024: pitch 1026
// (16 wide) or 1028 (8 wide) with 64-bit paired gathers; a warp holds one 1024-point line, so the
// pitch only matters to the staging.  Sizing the 16-wide strip as transposed (114.6 KB, two CTAs
// per SM) rather than at the column walk's pitch measured +1.4..4.6% on every 1024-high two-pass
// shape over 8 wide strips (64-byte row segments instead of 32).  512: pitch 529 (= 17 mod 32); the
// bank model (tests/test_bank_model.py) counts 158 wavefronts per warp for 512-point rows at that
// pitch against 190 for the 34-pitch column walk, and the scalar gathers of a warp's two lines fall
// into even and odd banks.  Narrower 512-point strips (8 wide, 128-thread CTAs, five per SM)
// measured 20-25% slower: 32-byte row segments.  The transposing scalar stores of the staging are
// conflict-free at these pitches: a warp covers 32 / (TC / 4) rows of TC / 4 float4 groups, and
// group q's stores land 4 q * pitch = q * 128 / TC (mod 32) banks apart.
__host__ __device__ constexpr bool is_transposed_strip(int h, int tc) {
  return (h == 1024 && (tc == 8 || tc == 16)) || (h == 512 && tc == 32);
}
template <int H, int TC> __host__ __device__ constexpr bool transposed_strip() { return is_transposed_strip(H, TC); }
__host__ __device__ constexpr int transposed_pitch(int h, int tc) {
  return h == 1024 ? (tc == 16 ? 1026 : 1028) : tc == 32 ? h + 17 : h + 4;
}

template <int H, int W, int TC, int MODE, int THREADS = kThreads, bool GEN = false, bool UNITS = false>
__global__ void __launch_bounds__(THREADS) k_colstrip(TileArgs a) {
  constexpr bool kT = transposed_strip<H, TC>();
  constexpr int P = kT ? transposed_pitch(H, TC) : strip_pitch(H, TC);
  constexpr int STRIPS = W / TC;
  extern __shared__ float smem[];
  float* tile = smem;
  float* xbuf = smem + round4(kT ? TC * P : H * P);
  griddep_wait();
  // register lines (128-point columns of the two-pass shapes) need no exchange buffer or tables
  constexpr bool kFs = H > reg_line_max(H, W, MODE, true);
  const FourStepTables tcol =
      kFs ? stage_tables<H>(a.tab.col, xbuf + round4((THREADS / 32) * ExchangeFloats<H>::value)) : a.tab.col;
  // Strips of 128- and 256-point columns prefetch the next strip into registers during the
  // transform; longer columns keep their occupancy.  (256-point strips of 16 columns in 128-thread
  // CTAs, five per SM but without the prefetch, measured 20-25% slower.)
  constexpr bool kPrefetch = THREADS == kThreads && (H == 128 || H == 256);
  // Strip t: its first element in x and y and the row pitch of its array.  Contiguous batches:
  // strip t % STRIPS of array t / STRIPS; GEN: the same through the layouts; UNITS: unit t.
  auto xarr = [&](long long arr) { return GEN ? a.x + layout_row<H>(a.lx, arr * H) : a.x + arr * (long long)H * W; };
  auto yarr = [&](long long arr) { return GEN ? a.y + layout_row<H>(a.ly, arr * H) : a.y + arr * (long long)H * W; };
  auto src = [&](long long t) -> const float* {
    return UNITS ? a.x + a.units[t].off : xarr(t / STRIPS) + (t % STRIPS) * TC;
  };
  auto dst = [&](long long t) -> float* {
    return UNITS ? a.y + a.units[t].off : yarr(t / STRIPS) + (t % STRIPS) * TC;
  };
  auto xpitch = [&](long long t) -> long long { return UNITS ? a.units[t].ld : GEN ? a.lx.ld : W; };
  auto ypitch = [&](long long t) -> long long { return UNITS ? a.units[t].ld : GEN ? a.ly.ld : W; };
  TileRegs<P, kPrefetch ? H : 4, kPrefetch ? TC : 4, THREADS> next;
  if (kPrefetch && blockIdx.x < a.ntiles) next.load(src(blockIdx.x), xpitch(blockIdx.x), H);
  for (long long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    if (t + gridDim.x >= a.ntiles) griddep_trigger();   // this CTA's last strip
    const long long xp = xpitch(t), yp = ypitch(t);
    if constexpr (kPrefetch) {
      next.put(tile);
      __syncthreads();
      if (t + gridDim.x < a.ntiles) next.load(src(t + gridDim.x), xpitch(t + gridDim.x), H);
    } else if constexpr (kT) {
      // eight float4 loads in flight per thread before their transposing stores
      const float* g = src(t);
      constexpr int Q = TC / 4, kPer = H * Q / THREADS, kBatch = kPer < 8 ? kPer : 8;
      static_assert(kPer % kBatch == 0, "strip staging batches");
#pragma unroll 1
      for (int k0 = 0; k0 < kPer; k0 += kBatch) {
        float4 v[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
          const int i = threadIdx.x + (k0 + k) * THREADS, r = i / Q, c = (i % Q) * 4;
          v[k] = __ldg(reinterpret_cast<const float4*>(g + r * xp + c));
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
          const int i = threadIdx.x + (k0 + k) * THREADS, r = i / Q, c = (i % Q) * 4;
          tile[c * P + r] = v[k].x;
          tile[(c + 1) * P + r] = v[k].y;
          tile[(c + 2) * P + r] = v[k].z;
          tile[(c + 3) * P + r] = v[k].w;
        }
      }
      __syncthreads();
    } else {
      tile_load<P>(src(t), xp, H, TC, tile, H);
      __syncthreads();
    }
    if constexpr (kT) {
      run_lines<H, MODE, reg_line_max(H, W, MODE, true), P % 2 == 0>(tile, TC, 1, [](int l) { return l * P; },
                                                                    xbuf, tcol);
    } else {
      run_lines<H, MODE, reg_line_max(H, W, MODE, true)>(tile, TC, P, [](int l) { return l; }, xbuf, tcol);
    }
    __syncthreads();
    if constexpr (kT) {
      float* g = dst(t);
      constexpr int Q = TC / 4;
      for (int i = threadIdx.x; i < H * Q; i += THREADS) {
        const int r = i / Q, c = (i % Q) * 4;
        *reinterpret_cast<float4*>(g + r * yp + c) =
            make_float4(tile[c * P + r], tile[(c + 1) * P + r], tile[(c + 2) * P + r], tile[(c + 3) * P + r]);
      }
    } else {
      tile_store<P>(dst(t), yp, H, TC, tile);
    }
    __syncthreads();
  }
}

// Compile-time launch geometry of one (H, W) shape.  Shared-memory sizes are kept at or below
// kSmemTwoPerSM so that two CTAs share an SM: tile rows (whole arrays), strip widths and row
// blocks are halved from their targets until they fit.
constexpr int kSmemTwoPerSM = 115712;

template <int N> __host__ __device__ constexpr int lines_per_warp() { return N >= 128 ? 1024 / N : 1; }

template <int H, int W>
struct Geometry {
  static constexpr bool kTile = H * W <= 16384;
  // tile class
  static constexpr int kXbufFull = kWarps * cmax(ExchangeFloats<H>::value, ExchangeFloats<W>::value);
  static constexpr int full_smem(int arrays) {
    return (round4(arrays * tile_array_pitch(H, W, tile_pitch(H, W))) + round4(kXbufFull) + TableFloats<H>::value +
            TableFloats<W>::value) * 4;
  }
  // Shared memory of a whole-array tile kernel (k_full<H, W, arrays * H, 1, 1, MODE, THREADS>):
  // the tile, and for the axes whose lines run the four-step their exchange buffer and tables.
  template <int MODE, int THREADS>
  static constexpr int tile_smem(int arrays) {
    constexpr bool fc = H > reg_line_max(H, W, MODE, false), fr = W > reg_line_max(W, H, MODE, false);
    return (round4(arrays * tile_array_pitch(H, W, tile_pitch(H, W))) +
            round4((THREADS / 32) * cmax(fc ? ExchangeFloats<H>::value : 0, fr ? ExchangeFloats<W>::value : 0)) +
            (fc ? TableFloats<H>::value : 0) + (fr ? TableFloats<W>::value : 0)) * 4;
  }
  static constexpr int pick_arrays(int target, int cap = kSmemTwoPerSM) {
    int a = cmax(1, target / (H * W));
    while (a > 1 && full_smem(a) > cap) a /= 2;
    return a;
  }
  static constexpr int kArrays = pick_arrays(kTileFloats);
  static constexpr int kTR = kTile ? kArrays * H : 1;
  static constexpr int kSmemFull = full_smem(kArrays);
  // Tiles of twice the target, for the shapes where they measured faster (see launch_plain).
  static constexpr int kArraysBig = pick_arrays(2 * kTileFloats);
  static constexpr int kTRBig = kTile ? kArraysBig * H : 1;
  static constexpr int kSmemFullBig = full_smem(kArraysBig);
  // Tiles of twice the target for kernels that hold one CTA per SM anyway (128-point register
  // lines, 227 registers): sized against one CTA's shared memory instead of two.
  static constexpr int kArraysWide = pick_arrays(2 * kTileFloats, 2 * kSmemTwoPerSM);
  static constexpr int kTRWide = kTile ? kArraysWide * H : 1;
  static constexpr int kSmemFullWide = full_smem(kArraysWide);
  // Tiles of a quarter of the target for small batches, so that a batch of a few MiB spreads over
  // several CTAs per SM instead of one uneven wave (see launch_plain).
  static constexpr int kArraysSmall = pick_arrays(kTileFloats / 2);
  static constexpr int kTRSmall = kTile ? kArraysSmall * H : 1;
  static constexpr int kSmemFullSmall = full_smem(kArraysSmall);
  // One whole array of 32768 floats per tile (one CTA per SM, 178-184 KB of shared memory), for
  // the two-pass shapes and modes where it measured faster than the two passes (launch_plain).
  static constexpr int kSmemWhole = full_smem(1);
  // 2-pass class
  static constexpr int strip_tile(int tc) {
    return is_transposed_strip(H, tc) ? tc * transposed_pitch(H, tc) : H * strip_pitch(H, tc);
  }
  static constexpr int strip_smem(int tc) {
    return (round4(strip_tile(tc)) + round4(kWarps * ExchangeFloats<H>::value) + TableFloats<H>::value) * 4;
  }
  // The strip width is sized with pitch tc + 4 even where the strip uses tc + 2: 256-point strips
  // widened to 64 columns by the smaller pitch measured 4-11% slower.
  static constexpr int sizing_smem(int tc) {
    return (round4(H * pitch_of(H, tc, true)) + round4(kWarps * ExchangeFloats<H>::value) + TableFloats<H>::value) * 4;
  }
  static constexpr int pick_tc() {
    int tc = (16384 / H) < W ? (16384 / H) : W;
    while (tc > cmax(4, lines_per_warp<H>()) &&
           (is_transposed_strip(H, tc) ? strip_smem(tc) : sizing_smem(tc)) > kSmemTwoPerSM)
      tc /= 2;
    return tc;
  }
  static constexpr int kTC = pick_tc();
  static constexpr int kSmemStrip = strip_smem(kTC);
  static constexpr int rows_smem(int rb) {
    return (round4(rb * rowblock_pitch(W)) + round4(kWarps * ExchangeFloats<W>::value) + TableFloats<W>::value) * 4;
  }
  // What the two-pass kernels of one mode and thread count use: the exchange buffer and tables only
  // where the pass's lines run the four-step (strip_smem / rows_smem size the geometry).
  template <int MODE, int THREADS>
  static constexpr int strip_smem_used(int tc) {
    constexpr bool fs = H > reg_line_max(H, W, MODE, true);
    return (round4(strip_tile(tc)) + (fs ? round4((THREADS / 32) * ExchangeFloats<H>::value) + TableFloats<H>::value : 0)) * 4;
  }
  template <int MODE, int THREADS>
  static constexpr int rows_smem_used(int rb) {
    constexpr bool fs = W > reg_line_max(W, H, MODE, true);
    return (round4(rb * rowblock_pitch(W)) + (fs ? round4((THREADS / 32) * ExchangeFloats<W>::value) + TableFloats<W>::value : 0)) * 4;
  }
  static constexpr int pick_rb() {
    int rb = cmax(1, 16384 / W);
    while (rb > lines_per_warp<W>() && rows_smem(rb) > kSmemTwoPerSM) rb /= 2;
    return rb;
  }
  static constexpr int kRB = pick_rb();
  static constexpr int kSmemRows = rows_smem(kRB);
  // Few-array variant: one four-step line group per warp, so that a call on one or a few arrays
  // spreads over more SMs (a single 1024x1024 array: 128 strips instead of 64).
  static constexpr int kTCs = H >= 128 ? cmin(kTC, cmax(4, kWarps * lines_per_warp<H>())) : kTC;
  static constexpr int kSmemStripS = strip_smem(kTCs);
  static constexpr int kRBs = W >= 128 ? cmin(kRB, kWarps * lines_per_warp<W>()) : kRB;
  static constexpr int kSmemRowsS = rows_smem(kRBs);
  // Row passes of 256- and 512-point lines in 128-thread CTAs: one line group per warp (16 or 8
  // rows) and four warps' exchange buffers, 42-43 KB, so five CTAs (20 warps) share an SM where
  // 256-thread CTAs of 64 or 32 rows fit two (16 warps).
  static constexpr bool kNarrowRows = W == 256 || W == 512;
  static constexpr int kRBn = lines_per_warp<W>() * 4;
  static constexpr int kSmemRowsN =
      (round4(kRBn * rowblock_pitch(W)) + round4(4 * ExchangeFloats<W>::value) + TableFloats<W>::value) * 4;
};

}  // namespace bridct
