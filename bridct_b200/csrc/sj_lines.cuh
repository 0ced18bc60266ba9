// Line operations of the plain (Shao-Johnson, FP32 CUDA-core) form.
//
// A "line" is one row or one column of an h x w array, held in shared memory with an
// element stride.  Three line operations exist, one per reference mode (include/bridct.h:24-28):
//   FWD: y = Q x        orthonormal DCT-II      (reference: col_fN then x norm, rect.c:8-15)
//   INV: y = Q^T x      orthonormal DCT-III     (x norm then col_tN)
//   RT : y = Q^T Q x    normalized round trip   (col_fN, x corr, col_tN)
// The 2D transform is a column pass then a row pass; the per-axis factors of the reference's
// normalization table (src/plan.c:92-107, norm[r,c] = s_h(r) s_w(c)) are separable, so each pass
// folds its own factor into its line operation instead of reading an h*w table.
//
// N <= 64: one thread owns the whole line in registers and runs the generated straight-line
//          SJ program (sj_generated.cuh).
// N >= 128: N = 32 * G; G lanes of one warp cooperate ("four-step" split of the SJ real FFT):
//   stage 1  lane b runs the SJ scaled real FFT of length 32 on v[G a + b], a = 0..31
//            (v = Makhoul reorder of x, as the reference's idx tables);
//   twiddle  T_b(c) = W_b(c) * w_N^{bc} * s(32, c)  (the leaf's SJ scale folded in);
//   exchange through shared memory (same warp: __syncwarp only);
//   stage 2  for each column c = 0..16, an SJ scaled complex FFT of length G over b gives
//            V_{c + 32 d} / s(G, d);
//   post     y[k] and y[N-k] from V_k (Makhoul: C[k] = Re(e^{-i pi k/2N} V_k),
//            C[N-k] = -Im(...)), with s(G, d) and the orthonormal factor folded into one table.
// The inverse runs the transposed stages in reverse order.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "sj_generated.cuh"

namespace bridct {

enum LineMode { LM_FWD = 0, LM_INV = 1, LM_RT = 2 };

// ---------------------------------------------------------------------------------------
// Register lines (N <= 64)
// ---------------------------------------------------------------------------------------
template <int N> struct RegLine;
#define BRIDCT_REGLINE(N)                                                                  \
  template <> struct RegLine<N> {                                                          \
    static __device__ __forceinline__ void fwd(float (&v)[N]) { sj_line_fwd_##N(v); }      \
    static __device__ __forceinline__ void inv(float (&v)[N]) { sj_line_inv_##N(v); }      \
    static __device__ __forceinline__ void rt(float (&v)[N]) { sj_line_rt_##N(v); }        \
  };
BRIDCT_REGLINE(8)
BRIDCT_REGLINE(16)
BRIDCT_REGLINE(32)
BRIDCT_REGLINE(64)
#undef BRIDCT_REGLINE

template <int N, int MODE>
__device__ __forceinline__ void reg_line_apply(float (&v)[N]) {
  if (MODE == LM_FWD) RegLine<N>::fwd(v);
  else if (MODE == LM_INV) RegLine<N>::inv(v);
  else RegLine<N>::rt(v);
}

// One thread, one line: load, transform, store (shared memory, element stride es).
template <int N, int MODE>
__device__ __forceinline__ void reg_line(float* line, int es) {
  float v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = line[i * es];
  reg_line_apply<N, MODE>(v);
#pragma unroll
  for (int i = 0; i < N; ++i) line[i * es] = v[i];
}

// ---------------------------------------------------------------------------------------
// Four-step lines (N = 32 G, G in {4, 8, 16, 32})
// ---------------------------------------------------------------------------------------
template <int G> struct CFFT;
#define BRIDCT_CFFT(G)                                                                     \
  template <> struct CFFT<G> {                                                             \
    static __device__ __forceinline__ void fwd(float (&z)[2 * G]) { sj_cfft_##G(z); }      \
    static __device__ __forceinline__ void tr(float (&z)[2 * G]) { sj_cfft_##G##_t(z); }   \
  };
BRIDCT_CFFT(4)
BRIDCT_CFFT(8)
BRIDCT_CFFT(16)
BRIDCT_CFFT(32)
#undef BRIDCT_CFFT

// Tables of one line length N (device memory, built on the host in float64):
//   tw[b * 17 + c]   = w_N^{b c} s(32, c)                     (float2)
//   post[c * G + d]  = (A, B, C, D) for k = c + 32 d          (float4)
//     y[k] = A Vr + B Vi,  y[N-k] = C Vr + D Vi,  V = stage-2 output (scaled).
struct FourStepTables {
  const float2* tw;
  const float4* post;
};

// Exchange buffer floats needed per warp for a given G (re and im planes).
template <int G>
struct FourStepSizes {
  static constexpr int LPW = 32 / G;           // lines per warp
  static constexpr int PITCH = G + 1;          // odd pitch: conflict-free column reads
  static constexpr int PLANE = LPW * 17 * PITCH;
  static constexpr int FLOATS = 2 * PLANE;
};

__device__ __forceinline__ int makhoul_src(int n, int N) {
  return n < N / 2 ? 2 * n : 2 * N - 1 - 2 * n;
}

// Forward four-step on the LPW lines owned by this warp.  line_ptr(j) returns the base of
// the warp's j-th line (j < LPW); es = element stride.  xb = this warp's exchange buffer.
template <int G, typename LinePtr>
__device__ __forceinline__ void fs_forward(const LinePtr& line_ptr, int es, float* xb,
                                           FourStepTables tab) {
  constexpr int N = 32 * G;
  using SZ = FourStepSizes<G>;
  const int lane = threadIdx.x & 31;
  const int grp = lane / G, b = lane % G;
  {
    float* line = line_ptr(grp);
    float xin[32], w[32];
#pragma unroll
    for (int a = 0; a < 32; ++a) xin[a] = line[makhoul_src(G * a + b, N) * es];
    sj_rfft_32(xin, w);
    float* re = xb + grp * 17 * SZ::PITCH + b;
    float* im = re + SZ::PLANE;
    re[0] = w[0];
    im[0] = 0.0f;
#pragma unroll
    for (int c = 1; c < 16; ++c) {
      const float2 t = __ldg(&tab.tw[b * 17 + c]);
      const float wr = w[c], wi = w[16 + c];
      re[c * SZ::PITCH] = wr * t.x - wi * t.y;
      im[c * SZ::PITCH] = wr * t.y + wi * t.x;
    }
    {
      const float2 t = __ldg(&tab.tw[b * 17 + 16]);
      re[16 * SZ::PITCH] = w[16] * t.x;
      im[16 * SZ::PITCH] = w[16] * t.y;
    }
  }
  __syncwarp();
  for (int task = lane; task < SZ::LPW * 17; task += 32) {
    const int g2 = task / 17, c = task % 17;
    const float* re = xb + task * SZ::PITCH;
    const float* im = re + SZ::PLANE;
    float z[2 * G];
#pragma unroll
    for (int q = 0; q < G; ++q) {
      z[2 * q] = re[q];
      z[2 * q + 1] = im[q];
    }
    CFFT<G>::fwd(z);
    float* line = line_ptr(g2);
    const int dmax = (c == 0) ? G / 2 : (c == 16 ? G / 2 - 1 : G - 1);
#pragma unroll
    for (int d = 0; d < G; ++d) {
      if (d > dmax) break;
      const int k = c + 32 * d;
      const float4 p = __ldg(&tab.post[c * G + d]);
      const float vr = z[2 * d], vi = z[2 * d + 1];
      if (k == 0) {
        line[0] = p.x * vr;
      } else {
        line[k * es] = p.x * vr + p.y * vi;
        if (2 * k != N) line[(N - k) * es] = p.z * vr + p.w * vi;
      }
    }
  }
  __syncwarp();
}

// Transpose of fs_forward: orthonormal DCT-III on the warp's lines.
template <int G, typename LinePtr>
__device__ __forceinline__ void fs_inverse(const LinePtr& line_ptr, int es, float* xb,
                                           FourStepTables tab) {
  constexpr int N = 32 * G;
  using SZ = FourStepSizes<G>;
  const int lane = threadIdx.x & 31;
  for (int task = lane; task < SZ::LPW * 17; task += 32) {
    const int g2 = task / 17, c = task % 17;
    const float* line = line_ptr(g2);
    const int dmax = (c == 0) ? G / 2 : (c == 16 ? G / 2 - 1 : G - 1);
    float z[2 * G];
#pragma unroll
    for (int d = 0; d < G; ++d) {
      float zr = 0.0f, zi = 0.0f;
      if (d <= dmax) {
        const int k = c + 32 * d;
        const float4 p = __ldg(&tab.post[c * G + d]);
        if (k == 0) {
          zr = p.x * line[0];
        } else {
          const float yk = line[k * es];
          zr = p.x * yk;
          zi = p.y * yk;
          if (2 * k != N) {
            const float ynk = line[(N - k) * es];
            zr += p.z * ynk;
            zi += p.w * ynk;
          }
        }
      }
      z[2 * d] = zr;
      z[2 * d + 1] = zi;
    }
    CFFT<G>::tr(z);
    float* re = xb + task * SZ::PITCH;
    float* im = re + SZ::PLANE;
#pragma unroll
    for (int q = 0; q < G; ++q) {
      re[q] = z[2 * q];
      im[q] = z[2 * q + 1];
    }
  }
  __syncwarp();
  {
    const int grp = lane / G, b = lane % G;
    const float* re = xb + grp * 17 * SZ::PITCH + b;
    const float* im = re + SZ::PLANE;
    float w[32], xo[32];
    w[0] = re[0];
#pragma unroll
    for (int c = 1; c < 16; ++c) {
      const float2 t = __ldg(&tab.tw[b * 17 + c]);
      const float tr = re[c * SZ::PITCH], ti = im[c * SZ::PITCH];
      w[c] = tr * t.x + ti * t.y;
      w[16 + c] = ti * t.x - tr * t.y;
    }
    {
      const float2 t = __ldg(&tab.tw[b * 17 + 16]);
      w[16] = re[16 * SZ::PITCH] * t.x + im[16 * SZ::PITCH] * t.y;
    }
    sj_rfft_32_t(w, xo);
    float* line = line_ptr(grp);
#pragma unroll
    for (int a = 0; a < 32; ++a) line[makhoul_src(G * a + b, N) * es] = xo[a];
  }
  __syncwarp();
}

template <int G, int MODE, typename LinePtr>
__device__ __forceinline__ void fs_line(const LinePtr& line_ptr, int es, float* xb,
                                        FourStepTables tab) {
  if (MODE == LM_FWD) {
    fs_forward<G>(line_ptr, es, xb, tab);
  } else if (MODE == LM_INV) {
    fs_inverse<G>(line_ptr, es, xb, tab);
  } else {
    fs_forward<G>(line_ptr, es, xb, tab);
    fs_inverse<G>(line_ptr, es, xb, tab);
  }
}

}  // namespace bridct
