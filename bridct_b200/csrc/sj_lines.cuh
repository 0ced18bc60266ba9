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

// Programmatic dependent launch: the plain kernels are launched with programmatic stream
// serialization, so a kernel's CTAs may be scheduled while the previous kernel in the stream is
// still finishing.  griddep_wait() blocks until every prerequisite grid has completed and its
// memory is visible; each kernel calls it before its first global access, so results are exactly
// those of a serialized launch (without a prerequisite it returns at once).  griddep_trigger()
// lets the next kernel's CTAs be scheduled once every CTA of this one has reached it.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------------------------------
// Register lines (N <= 128; the fixed-shape kernels use them for N = 128, the ragged kernel
// only up to 64)
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
BRIDCT_REGLINE(128)
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

// Tables of one line length N (built on the host in float64; the fixed-shape kernels copy them
// into shared memory at start):
//   tw[b * 17 + c]   = w_N^{b c} s(32, c)  for c = 1..15 (c = 0 and 16 need none:
//                       s(32, 0) = s(32, 16) = 1 and column 16's rotation is inside sj_col16)
//   post[d * 17 + c] = (A, B, C, D) for k = c + 32 d (d-major, so the lanes of a stage-2 round,
//                       which hold consecutive columns c, read consecutive float4s):
//     y[k] = A Vr + B Vi,  y[N-k] = C Vr + D Vi, with V the stage-2 output of column c, whose
//     SJ scale (s(G,d); s(16,d>>1) for the split G = 32 columns; 1 for columns 0 and 16, which
//     use an unscaled cooperative DFT) and the orthonormal factor are folded in.
struct FourStepTables {
  const float2* tw;
  const float4* post;
};

// Position of post coefficient (d, c) in the table of lines of N = 32 G points: [d][c] (17 per d)
// for G < 32.  For G = 32 the table is [d / 2][c][d % 2]: the 30 stage-2 lanes of one step, lane
// (c, h) reading d = 2 m + h, then read 30 consecutive float4s (a [d][c] table put lanes (c, 0) and
// (c, 1) 17 float4s apart: 2-way bank conflicts on every read).  Host and device use this function.
__host__ __device__ constexpr int post_index(int G, int d, int c) {
  return G == 32 ? (d >> 1) * 34 + 2 * c + (d & 1) : d * 17 + c;
}

// Exchange buffer floats needed per warp for a given G (re and im planes).
template <int G>
struct FourStepSizes {
  static constexpr int LPW = 32 / G;           // lines per warp
  static constexpr int PITCH = G + 1;          // odd pitch: conflict-free column reads
  // per-line (slot) stride: the LPW slots' stage-1 writes hit disjoint banks (stride = G * odd
  // mod 32), and for G = 4, 8 slots LPW/2 apart lie 16 banks apart (stride * LPW/2 = 16 mod 32)
  static constexpr int LINE = G == 4 ? 84 : G == 8 ? 168 : G == 16 ? 304 : 17 * PITCH;
  static constexpr int PLANE = LPW * LINE;
  static constexpr int FLOATS = 2 * PLANE;
};

// Exchange slot of the warp's line j, and the stage-2 task (line g2, column c) of a lane in
// round r.  For G = 4 and 8 (LPW = 8 or 4 lines per warp) each of the LPW/2 rounds takes the 15
// columns of two lines whose slots lie LPW/2 apart, i.e. 16 banks apart, so a round's exchange
// accesses are conflict-free.  Rows pair lines r and r + LPW/2 (at a row pitch of 4 mod 8 for
// G = 4, 8 mod 32 for G = 8 their post-rotation stores are 16 banks apart too); columns pair the
// adjacent columns 2r and 2r + 1, which the slot permutation puts LPW/2 slots apart.  Other G:
// slot = line and task = lane + 32 r.
template <int G>
__device__ __forceinline__ int fs_slot(int j, bool rows) {
  constexpr int HALF = FourStepSizes<G>::LPW / 2;
  return ((G == 4 || G == 8) && !rows) ? (j >> 1) + HALF * (j & 1) : j;
}
template <int G>
struct FsTasks {
  static constexpr bool PAIRED = G == 4 || G == 8;
  static constexpr int ROUNDS = PAIRED ? FourStepSizes<G>::LPW / 2 : (FourStepSizes<G>::LPW * 15 + 31) / 32;
  static __device__ __forceinline__ bool get(int lane, int r, bool rows, int& g2, int& c) {
    if constexpr (PAIRED) {
      if (lane >= 30) return false;
      const int hi = lane >= 15 ? 1 : 0;
      c = 1 + lane - 15 * hi;
      g2 = rows ? r + (FourStepSizes<G>::LPW / 2) * hi : 2 * r + hi;
      return true;
    } else {
      const int task = lane + 32 * r;
      if (task >= FourStepSizes<G>::LPW * 15) return false;
      g2 = task / 15;
      c = 1 + task % 15;
      return true;
    }
  }
};

__device__ __forceinline__ int makhoul_src(int n, int N) {
  return n < N / 2 ? 2 * n : 2 * N - 1 - 2 * n;
}

// Cooperative DFT of length G across the G lanes of one line group (lane b holds element b):
// radix-2 decimation in frequency with shuffles; on return lane b holds X(bitrev(b)).  The
// twiddle w_G^m is tw[2m * 17 + 16] = w_N^{32 m} (table entry of column 16).
template <int G>
__device__ __forceinline__ void coop_dft(float& re, float& im, int b, const float2* tw) {
#pragma unroll
  for (int s = G / 2; s >= 1; s >>= 1) {
    const float pr = __shfl_xor_sync(0xFFFFFFFFu, re, s, G);
    const float pi = __shfl_xor_sync(0xFFFFFFFFu, im, s, G);
    if (b & s) {
      const float2 w = tw[(2 * (b & (s - 1)) * (G / (2 * s))) * 17 + 16];
      const float dr = pr - re, di = pi - im;
      re = dr * w.x - di * w.y;
      im = dr * w.y + di * w.x;
    } else {
      re += pr;
      im += pi;
    }
  }
}

// Transpose of coop_dft: lane b holds the adjoint of X(bitrev(b)) on entry and of x_b on return.
template <int G>
__device__ __forceinline__ void coop_dft_t(float& re, float& im, int b, const float2* tw) {
#pragma unroll
  for (int s = 1; s <= G / 2; s <<= 1) {
    const float pr = __shfl_xor_sync(0xFFFFFFFFu, re, s, G);
    const float pi = __shfl_xor_sync(0xFFFFFFFFu, im, s, G);
    const float2 w = tw[(2 * (b & (s - 1)) * (G / (2 * s))) * 17 + 16];
    if (b & s) {                      // x_{j+s} = top - conj(w) * bottom
      const float nr = pr - (re * w.x + im * w.y);
      const float ni = pi - (im * w.x - re * w.y);
      re = nr;
      im = ni;
    } else {                          // x_j = top + conj(w) * bottom
      re = re + (pr * w.x + pi * w.y);
      im = im + (pi * w.x - pr * w.y);
    }
  }
}

template <int G>
__device__ __forceinline__ int bitrev(int b) {
  return (int)(__brev((unsigned)b) >> (32 - __ffs(G) + 1));
}

// Post rotation of one stage-2 output V(d) of column c into the line (and its transpose).
__device__ __forceinline__ void post_store(float* line, int es, int N, int k, float4 p, float vr, float vi) {
  if (k == 0) {
    line[0] = p.x * vr;
  } else {
    line[k * es] = p.x * vr + p.y * vi;
    if (2 * k != N) line[(N - k) * es] = p.z * vr + p.w * vi;
  }
}
__device__ __forceinline__ void post_load(const float* line, int es, int N, int k, float4 p, float& vr, float& vi) {
  if (k == 0) {
    vr = p.x * line[0];
    vi = 0.0f;
  } else {
    const float yk = line[k * es];
    vr = p.x * yk;
    vi = p.y * yk;
    if (2 * k != N) {
      const float ynk = line[(N - k) * es];
      vr += p.z * ynk;
      vi += p.w * ynk;
    }
  }
}

// Forward four-step on the LPW lines owned by this warp.  line_ptr(j) returns the base of
// the warp's j-th line (j < LPW); es = element stride.  xb = this warp's exchange buffer.
//   stage 1   lane b: SJ real FFT of length 32 of v[G a + b]; columns c = 1..15 twiddled into
//             the exchange buffer; columns 0 and 16 stay in registers
//   special   columns 0 and 16: cooperative shuffle DFT over the line's G lanes (column 16
//             pre-rotated by w_N^{16 b}); lane b stores V(bitrev(b)) where that index is needed
//   stage 2   columns 1..15: generated SJ complex FFT of length G per task (G = 32: each column
//             split into its two radix-2 halves, so 30 lanes do equal work)
// PAIRS: the lines are rows (es = 1) starting 8-byte aligned.  Makhoul's v[n] = x[2n] and
// v[N-1-n] = x[2n+1] (n < N/2) then come from one 64-bit load: lane b keeps x[2n] (n = G a + b,
// a < 16) and passes x[2n+1] = v[N-1-n] = v[G (31 - a) + (G-1-b)] to lane G-1-b, whose element
// 31 - a it is.  Half the load instructions, and no 2-way bank conflict of the stride-2 scalar
// gather.
template <int G, bool PAIRS = false, typename LinePtr>
__device__ __forceinline__ void fs_forward(const LinePtr& line_ptr, int es, float* xb,
                                           FourStepTables tab) {
  constexpr int N = 32 * G;
  using SZ = FourStepSizes<G>;
  const int lane = threadIdx.x & 31;
  const int grp = lane / G, b = lane % G;
  float w0, w16;
  {
    float* line = line_ptr(grp);
    float xin[32], w[32];
    if constexpr (PAIRS) {
#pragma unroll
      for (int a = 0; a < 16; ++a) {
        const float2 p = *reinterpret_cast<const float2*>(line + 2 * (G * a + b));
        xin[a] = p.x;
        xin[31 - a] = __shfl_xor_sync(0xFFFFFFFFu, p.y, G - 1);
      }
    } else {
#pragma unroll
      for (int a = 0; a < 32; ++a) xin[a] = line[makhoul_src(G * a + b, N) * es];
    }
    sj_rfft_32(xin, w);
    float* re = xb + fs_slot<G>(grp, es == 1) * SZ::LINE + b;
    float* im = re + SZ::PLANE;
#pragma unroll
    for (int c = 1; c < 16; ++c) {
      const float2 t = tab.tw[b * 17 + c];
      const float wr = w[c], wi = w[16 + c];
      re[c * SZ::PITCH] = wr * t.x - wi * t.y;
      im[c * SZ::PITCH] = wr * t.y + wi * t.x;
    }
    w0 = w[0];
    w16 = w[16];
  }
  // columns 0 and 16 (all lanes, registers and shuffles)
  float ar = w0, ai = 0.0f;
  coop_dft<G>(ar, ai, b, tab.tw);
  const float2 rot = tab.tw[b * 17 + 16];
  float cr = w16 * rot.x, ci = w16 * rot.y;
  coop_dft<G>(cr, ci, b, tab.tw);
  __syncwarp();                                  // every lane has read its stage-1 inputs
  {
    float* line = line_ptr(grp);
    const int d = bitrev<G>(b);
    if (d <= G / 2) post_store(line, es, N, 32 * d, tab.post[post_index(G, d, 0)], ar, (d == 0 || d == G / 2) ? 0.0f : ai);
    if (d < G / 2) post_store(line, es, N, 16 + 32 * d, tab.post[post_index(G, d, 16)], cr, ci);
  }
  if constexpr (G == 32) {
    if (lane < 30) {
      float* line = line_ptr(0);
      const float* re = xb;
      const float* im = xb + SZ::PLANE;
      const int c = 1 + (lane >> 1), h = lane & 1;
      float z[64], o[32];
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        z[2 * q] = re[c * SZ::PITCH + q];
        z[2 * q + 1] = im[c * SZ::PITCH + q];
      }
      if (h) sj_cfft_32_half1(z, o);
      else sj_cfft_32_half0(z, o);
      // Lanes (c, 0) and (c, 1) would store y[k] and y[k + 32] (one bank) at once: lane h = 1
      // stores its y[N - k] first instead (bank -k, disjoint from the h = 0 lanes' banks k, for
      // rows and for the odd pitches of 512/1024-point column strips alike).
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const int dd = 2 * m + h, k = c + 32 * dd;
        const float4 pc = tab.post[post_index(G, dd, c)];
        const float vr = o[2 * m], vi = o[2 * m + 1];
        const float yk = pc.x * vr + pc.y * vi, ynk = pc.z * vr + pc.w * vi;
        line[(h ? N - k : k) * es] = h ? ynk : yk;
        line[(h ? k : N - k) * es] = h ? yk : ynk;
      }
    }
  } else {
#pragma unroll 1
    for (int r = 0; r < FsTasks<G>::ROUNDS; ++r) {
      int g2, c;
      if (!FsTasks<G>::get(lane, r, es == 1, g2, c)) continue;
      float* line = line_ptr(g2);
      const float* re = xb + fs_slot<G>(g2, es == 1) * SZ::LINE + c * SZ::PITCH;
      const float* im = re + SZ::PLANE;
      float z[2 * G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        z[2 * q] = re[q];
        z[2 * q + 1] = im[q];
      }
      CFFT<G>::fwd(z);
#pragma unroll
      for (int dd = 0; dd < G; ++dd)
        post_store(line, es, N, c + 32 * dd, tab.post[post_index(G, dd, c)], z[2 * dd], z[2 * dd + 1]);
    }
  }
  __syncwarp();
}

// Transpose of fs_forward: orthonormal DCT-III on the warp's lines (PAIRS: 64-bit stores of
// x[2n], x[2n+1], the odd element taken from lane G-1-b).
template <int G, bool PAIRS = false, typename LinePtr>
__device__ __forceinline__ void fs_inverse(const LinePtr& line_ptr, int es, float* xb,
                                           FourStepTables tab) {
  constexpr int N = 32 * G;
  using SZ = FourStepSizes<G>;
  const int lane = threadIdx.x & 31;
  const int grp = lane / G, b = lane % G;
  // columns 0 and 16: adjoints of V(bitrev(b)), then the transposed cooperative DFTs
  float ar = 0.0f, ai = 0.0f, cr = 0.0f, ci = 0.0f;
  {
    const float* line = line_ptr(grp);
    const int d = bitrev<G>(b);
    if (d <= G / 2) {
      post_load(line, es, N, 32 * d, tab.post[post_index(G, d, 0)], ar, ai);
      if (d == 0 || d == G / 2) ai = 0.0f;
    }
    if (d < G / 2) post_load(line, es, N, 16 + 32 * d, tab.post[post_index(G, d, 16)], cr, ci);
  }
  coop_dft_t<G>(ar, ai, b, tab.tw);
  coop_dft_t<G>(cr, ci, b, tab.tw);
  const float2 rot = tab.tw[b * 17 + 16];
  const float w0 = ar;                           // real part: the forward input was real
  const float w16 = cr * rot.x + ci * rot.y;     // Re(conj(rotation) * adjoint)
  if constexpr (G == 32) {
    if (lane < 30) {
      const float* line = line_ptr(0);
      float* re = xb;
      float* im = xb + SZ::PLANE;
      const int c = 1 + (lane >> 1), h = lane & 1;
      float o[32], z[64];
#pragma unroll
      for (int m = 0; m < 16; ++m) {       // loads in the bank-disjoint order of the forward's stores
        const int dd = 2 * m + h, k = c + 32 * dd;
        const float4 pc = tab.post[post_index(G, dd, c)];
        const float first = line[(h ? N - k : k) * es];
        const float second = line[(h ? k : N - k) * es];
        const float yk = h ? second : first, ynk = h ? first : second;
        float vr = pc.x * yk, vi = pc.y * yk;   // the arithmetic of post_load
        vr += pc.z * ynk;
        vi += pc.w * ynk;
        o[2 * m] = vr;
        o[2 * m + 1] = vi;
      }
      if (h) sj_cfft_32_half1_t(o, z);
      else sj_cfft_32_half0_t(o, z);
      // both halves feed every b: each lane sums one half of the b range with its partner
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const float send = h ? z[q] : z[32 + q];
        const float recv = __shfl_xor_sync(0x3FFFFFFFu, send, 1);
        const float sum = (h ? z[32 + q] : z[q]) + recv;
        const int bb = (h ? 16 : 0) + (q >> 1);
        ((q & 1) ? im : re)[c * SZ::PITCH + bb] = sum;
      }
    }
  } else {
#pragma unroll 1
    for (int r = 0; r < FsTasks<G>::ROUNDS; ++r) {
      int g2, c;
      if (!FsTasks<G>::get(lane, r, es == 1, g2, c)) continue;
      const float* line = line_ptr(g2);
      float* re = xb + fs_slot<G>(g2, es == 1) * SZ::LINE + c * SZ::PITCH;
      float* im = re + SZ::PLANE;
      float z[2 * G];
#pragma unroll
      for (int dd = 0; dd < G; ++dd)
        post_load(line, es, N, c + 32 * dd, tab.post[post_index(G, dd, c)], z[2 * dd], z[2 * dd + 1]);
      CFFT<G>::tr(z);
#pragma unroll
      for (int q = 0; q < G; ++q) {
        re[q] = z[2 * q];
        im[q] = z[2 * q + 1];
      }
    }
  }
  __syncwarp();
  {
    const float* re = xb + fs_slot<G>(grp, es == 1) * SZ::LINE + b;
    const float* im = re + SZ::PLANE;
    float w[32], xo[32];
    w[0] = w0;
#pragma unroll
    for (int c = 1; c < 16; ++c) {
      const float2 t = tab.tw[b * 17 + c];
      const float tr = re[c * SZ::PITCH], ti = im[c * SZ::PITCH];
      w[c] = tr * t.x + ti * t.y;
      w[16 + c] = ti * t.x - tr * t.y;
    }
    w[16] = w16;
    sj_rfft_32_t(w, xo);
    float* line = line_ptr(grp);
    if constexpr (PAIRS) {
#pragma unroll
      for (int a = 0; a < 16; ++a) {
        const float odd = __shfl_xor_sync(0xFFFFFFFFu, xo[31 - a], G - 1);
        *reinterpret_cast<float2*>(line + 2 * (G * a + b)) = make_float2(xo[a], odd);
      }
    } else {
#pragma unroll
      for (int a = 0; a < 32; ++a) line[makhoul_src(G * a + b, N) * es] = xo[a];
    }
  }
  __syncwarp();
}

template <int G, int MODE, bool PAIRS = false, typename LinePtr>
__device__ __forceinline__ void fs_line(const LinePtr& line_ptr, int es, float* xb,
                                        FourStepTables tab) {
  if (MODE == LM_FWD) {
    fs_forward<G, PAIRS>(line_ptr, es, xb, tab);
  } else if (MODE == LM_INV) {
    fs_inverse<G, PAIRS>(line_ptr, es, xb, tab);
  } else {
    fs_forward<G, PAIRS>(line_ptr, es, xb, tab);
    fs_inverse<G, PAIRS>(line_ptr, es, xb, tab);
  }
}

}  // namespace bridct
