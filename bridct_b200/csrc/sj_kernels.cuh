// 2D kernels of the plain (Shao-Johnson FP32) form.
//
// Shape classes (h, w powers of two in [8, 1024]):
//   h*w <= 16384  "tile"    k_full<..., DO_COL=1, DO_ROW=1>: a CTA loads A whole arrays
//                           (A*h*w ~ 8192 floats) into shared memory with coalesced float4
//                           loads, runs every column line, then every row line, and stores.
//                           One HBM read and one HBM write per element.
//   h*w >  16384  "2-pass"  k_colstrip (h rows x TC columns per CTA, column lines, x -> y)
//                           then k_full<DO_COL=0> (TR full rows per CTA, row lines, y -> y in
//                           place).  The intermediate lives in y and is re-read while it is
//                           still L2-resident: the host walks large batches in chunks sized
//                           for L2 (the reference's rect route does the same pair of passes,
//                           vertical then bands, src/generated/rect.c:5-23).
// Shared-memory rows use an odd pitch (w + 1 floats) so that a thread-per-row line walk and a
// thread-per-column line walk are both bank-conflict free.
#pragma once
#include "sj_lines.cuh"

namespace bridct {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileFloats = 8192;   // target floats per CTA tile for small arrays

struct LineTables {
  FourStepTables col;   // for line length h (used when h >= 128)
  FourStepTables row;   // for line length w (used when w >= 128)
};

struct TileArgs {
  const float* x;
  float* y;
  long long ntiles;
  long long rows_total;   // rows of the (batch*h) x w matrix covered by this launch
  LineTables tab;
};

template <int N> struct ExchangeFloats { static constexpr int value = 0; };
template <> struct ExchangeFloats<128> { static constexpr int value = FourStepSizes<4>::FLOATS; };
template <> struct ExchangeFloats<256> { static constexpr int value = FourStepSizes<8>::FLOATS; };
template <> struct ExchangeFloats<512> { static constexpr int value = FourStepSizes<16>::FLOATS; };
template <> struct ExchangeFloats<1024> { static constexpr int value = FourStepSizes<32>::FLOATS; };

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Runs all lines of length N in a set of `nlines` lines; line l starts at tile + off(l),
// elements at stride es.  Register lines for N <= 64, warp four-step lines above.
template <int N, int MODE, typename Off>
__device__ __forceinline__ void run_lines(float* tile, int nlines, int es, const Off& off,
                                          float* xbuf, FourStepTables tab) {
  if constexpr (N <= 64) {
    for (int l = threadIdx.x; l < nlines; l += blockDim.x) reg_line<N, MODE>(tile + off(l), es);
  } else {
    constexpr int G = N / 32;
    constexpr int LPW = 32 / G;
    const int warp = threadIdx.x >> 5;
    float* xb = xbuf + warp * FourStepSizes<G>::FLOATS;
    for (int g = warp; g * LPW < nlines; g += blockDim.x >> 5) {
      auto ptr = [&](int j) { return tile + off(g * LPW + j); };
      fs_line<G, MODE>(ptr, es, xb, tab);
    }
  }
}

// Full-width tiles: TR consecutive rows (of width W) of the batch viewed as a (B*H) x W
// matrix.  With DO_COL the tile holds TR/H whole arrays.
template <int H, int W, int TR, bool DO_COL, bool DO_ROW, int MODE>
__global__ void __launch_bounds__(kThreads) k_full(TileArgs a) {
  constexpr int P = W + 1;
  extern __shared__ float smem[];
  float* tile = smem;
  float* xbuf = smem + TR * P;
  constexpr int N4 = TR * W / 4;
  for (long long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const float4* src = reinterpret_cast<const float4*>(a.x + t * (long long)TR * W);
    // The last tile of a launch may hold fewer than TR rows; it is zero-filled.
    const long long left = a.rows_total - t * (long long)TR;
    const int n4 = left >= TR ? N4 : (int)left * (W / 4);
#pragma unroll 4
    for (int i = threadIdx.x; i < N4; i += kThreads) {
      const float4 v = i < n4 ? __ldg(src + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      const int r = (4 * i) / W, c = (4 * i) % W;
      float* d = tile + r * P + c;
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
    __syncthreads();
    if constexpr (DO_COL) {
      static_assert(TR % H == 0, "column pass needs whole arrays");
      run_lines<H, MODE>(tile, (TR / H) * W, P,
                         [](int l) { return (l / W) * H * P + (l % W); }, xbuf, a.tab.col);
      __syncthreads();
    }
    if constexpr (DO_ROW) {
      run_lines<W, MODE>(tile, TR, 1, [](int l) { return l * P; }, xbuf, a.tab.row);
      __syncthreads();
    }
    float4* dst = reinterpret_cast<float4*>(a.y + t * (long long)TR * W);
#pragma unroll 4
    for (int i = threadIdx.x; i < n4; i += kThreads) {
      const int r = (4 * i) / W, c = (4 * i) % W;
      const float* s = tile + r * P + c;
      dst[i] = make_float4(s[0], s[1], s[2], s[3]);
    }
    __syncthreads();
  }
}

// Column strips: H rows x TC columns of one array (row pitch W in global memory).
template <int H, int W, int TC, int MODE>
__global__ void __launch_bounds__(kThreads) k_colstrip(TileArgs a) {
  constexpr int P = TC + 1;
  constexpr int STRIPS = W / TC;
  constexpr int Q = TC / 4;   // float4 per strip row
  extern __shared__ float smem[];
  float* tile = smem;
  float* xbuf = smem + H * P;
  for (long long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const long long arr = t / STRIPS;
    const int s = (int)(t % STRIPS);
    const float* base = a.x + arr * (long long)H * W + s * TC;
#pragma unroll 4
    for (int i = threadIdx.x; i < H * Q; i += kThreads) {
      const int r = i / Q, c = (i % Q) * 4;
      const float4 v = __ldg(reinterpret_cast<const float4*>(base + (long long)r * W + c));
      float* d = tile + r * P + c;
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
    __syncthreads();
    run_lines<H, MODE>(tile, TC, P, [](int l) { return l; }, xbuf, a.tab.col);
    __syncthreads();
    float* obase = a.y + arr * (long long)H * W + s * TC;
#pragma unroll 4
    for (int i = threadIdx.x; i < H * Q; i += kThreads) {
      const int r = i / Q, c = (i % Q) * 4;
      const float* sp = tile + r * P + c;
      *reinterpret_cast<float4*>(obase + (long long)r * W + c) = make_float4(sp[0], sp[1], sp[2], sp[3]);
    }
    __syncthreads();
  }
}

// Compile-time launch geometry of one (H, W) shape.
template <int H, int W>
struct Geometry {
  static constexpr bool kTile = H * W <= 16384;
  // tile class
  static constexpr int kArrays = cmax(1, kTileFloats / (H * W));
  static constexpr int kTR = kTile ? kArrays * H : 1;
  static constexpr int kXbufFull = kWarps * cmax(ExchangeFloats<H>::value, ExchangeFloats<W>::value);
  static constexpr int kSmemFull = (kTR * (W + 1) + kXbufFull) * 4;
  // 2-pass class
  static constexpr int kTC = (16384 / H) < W ? (16384 / H) : W;
  static constexpr int kSmemStrip = (H * (kTC + 1) + kWarps * ExchangeFloats<H>::value) * 4;
  static constexpr int kRB = cmax(1, 16384 / W);
  static constexpr int kSmemRows = (kRB * (W + 1) + kWarps * ExchangeFloats<W>::value) * 4;
};

}  // namespace bridct
