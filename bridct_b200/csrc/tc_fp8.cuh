// FP8 (E4M3) tensor-core form with per-32x32-tile scaling, for axes of 128 and 256.
//
// A 2D transform is two row passes, as in the split-precision forms, but the operands are
// quantized instead of split: every 32x32 tile of the data gets its own scale
// s = max|tile| / 448 (the largest finite E4M3 value) and is stored as E4M3 codes, and C (or
// C^T) is quantized the same way on the host.  A row of length L spans L/32 K-tiles with
// different scales, so each K-tile's product (one kind::f8f6f4 MMA, K = 32) accumulates in its
// own TMEM block and the epilogue forms sum_t sX(row band, t) * sC(column band, t) * acc_t in
// FP32.  One refinement step on the host side of the form recovers accuracy:
//     Y = Y8 + FP8(X - DCT-III_fp32(Y8)),  with the residual taken in FP32 by the plain form.
//
// k_quant8: one warp per 32x32 tile (lane = tile row): warp max of |x|, scale, E4M3 codes.
// k_fp8pass<L> (256 threads): warp 0 TMA producer (E4M3 rows, 128-byte boxes), warp 1 MMA
// issuer, warp 2 TMEM allocator, warps 4-7 epilogue (scales, sum, transposed stores).
#pragma once
#include <cuda_fp8.h>

#include "tc_blocks8.cuh"

namespace bridct {
namespace tc {

constexpr float kE4M3Max = 448.0f;

// rows: nrows x L FP32 (arrays of R rows); q: E4M3 codes, same layout; scales: per array
// [R/32][L/32].  ntiles = nrows/32 * L/32.
__global__ void __launch_bounds__(256) k_quant8(const float* __restrict__ rows, uint8_t* __restrict__ q,
                                                float* __restrict__ scales, long long ntiles, int L) {
  const int lane = threadIdx.x & 31;
  const long long t = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (t >= ntiles) return;
  const int tiles_per_band = L / 32;
  const long long band = t / tiles_per_band;      // 32-row band of the row matrix
  const int kt = (int)(t % tiles_per_band);
  const long long row = band * 32 + lane;
  const float4* src = reinterpret_cast<const float4*>(rows + row * L + kt * 32);
  float v[32];
  float amax = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float4 a = __ldg(src + i);
    v[4 * i] = a.x; v[4 * i + 1] = a.y; v[4 * i + 2] = a.z; v[4 * i + 3] = a.w;
    amax = fmaxf(amax, fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(a.w))));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xFFFFFFFFu, amax, o));
  const float s = amax > 0.0f ? amax / kE4M3Max : 1.0f;
  const float inv = 1.0f / s;
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const __nv_fp8x2_storage_t lo = __nv_cvt_float2_to_fp8x2(make_float2(v[4 * i] * inv, v[4 * i + 1] * inv),
                                                             __NV_SATFINITE, __NV_E4M3);
    const __nv_fp8x2_storage_t hi = __nv_cvt_float2_to_fp8x2(make_float2(v[4 * i + 2] * inv, v[4 * i + 3] * inv),
                                                             __NV_SATFINITE, __NV_E4M3);
    w[i] = (uint32_t)lo | ((uint32_t)hi << 16);
  }
  uint4* dst = reinterpret_cast<uint4*>(q + row * L + kt * 32);
  dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
  dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
  if (lane == 0) scales[t] = s;
}

// y = x - y (elementwise, n multiple of 4)
__global__ void k_residual(const float4* __restrict__ x, float4* __restrict__ y, long long n4) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 a = x[i], b = y[i];
    y[i] = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
  }
}

// y += d (elementwise, n multiple of 4)
__global__ void k_accumulate(float4* __restrict__ y, const float4* __restrict__ d, long long n4) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 a = y[i], b = d[i];
    y[i] = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
  }
}

template <int L>
struct Fp8Layout {
  static constexpr int kThreads = 256;
  static constexpr int kKT = L / 32;                  // K-tiles (one MMA and one accumulator each)
  static constexpr int kAtoms = L / 128;              // 128-byte K atoms per row
  static constexpr int kStageBytes = kAtoms * 16384;  // 128 rows x L codes
  static constexpr int kBBytes = kAtoms * 8192;       // 64 rows x L codes
  static constexpr int kSets = 2 * kKT * 64 <= 512 ? 2 : 1;   // TMEM accumulator sets
  static constexpr int kTmemAlloc = kSets * kKT * 64 <= 256 ? 256 : 512;
  static constexpr int kStages = 4;
  static constexpr int kBOff = kStages * kStageBytes;
  static constexpr int kScOff = kBOff + kBBytes;       // sC of this CTA's two column bands
  static constexpr int kBarOff = kScOff + 2 * kKT * 4 + 64;
  static constexpr int kDynamic = ((kBarOff + 255) / 256) * 256 + 256 + 1024;
  static_assert(kDynamic <= 232448, "shared memory budget");
};

__device__ __forceinline__ void umma_fp8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, 0, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc));
}

// Instruction descriptor for kind::f8f6f4: D FP32, A and B E4M3 (format 0), K-major, M=128, N=64.
constexpr uint32_t kFp8Idesc = (1u << 4) | ((64u >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);

// xmap: (nrows x L) E4M3 rows (box 128 x 128 bytes, SWIZZLE_128B); sx: their tile scales
// ([array][R/32][L/32]); bimage: kBlocks slices of 64 rows x L codes; sc: C's tile scales
// [L/32 column bands][L/32 K-tiles]; out: FP32 arrays written transposed (R = 1 << rshift).
template <int L>
__global__ void __launch_bounds__(256, 1)
    k_fp8pass(const __grid_constant__ CUtensorMap xmap, const float* __restrict__ sx, float* __restrict__ out,
              const uint4* __restrict__ bimage, const float* __restrict__ sc, long long nrows, int rshift,
              int* __restrict__ err) {
  using F = Fp8Layout<L>;
  constexpr int kBlocks = L / 64;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(base);
  const uint32_t bar = sbase + F::kBarOff;
  const uint32_t stage_full = bar, stage_free = bar + 8 * F::kStages, acc_full = bar + 16 * F::kStages,
                 acc_free = acc_full + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + F::kBarOff + 16 * F::kStages + 32);
  float* s_sc = reinterpret_cast<float*>(base + F::kScOff);
  __shared__ volatile int s_abort;
  __shared__ volatile int s_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nblk = blockIdx.x % kBlocks;
  const long long slot = blockIdx.x / kBlocks, nslots = gridDim.x / kBlocks;
  const long long mtiles = (nrows + kRows - 1) / kRows;
  const long long nlocal = slot < mtiles ? (mtiles - 1 - slot) / nslots + 1 : 0;

  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < F::kStages; ++i) {
      mbar_init(stage_full + 8 * i, 1);
      mbar_init(stage_free + 8 * i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(acc_full + 8 * i, 1);
      mbar_init(acc_free + 8 * i, 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(F::kTmemAlloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  {
    const uint4* src = bimage + (size_t)nblk * (F::kBBytes / 16);
    uint4* dst = reinterpret_cast<uint4*>(base + F::kBOff);
    for (int i = tid; i < F::kBBytes / 16; i += F::kThreads) dst[i] = __ldg(src + i);
    for (int i = tid; i < 2 * F::kKT; i += F::kThreads) s_sc[i] = __ldg(sc + (size_t)(2 * nblk) * F::kKT + i);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  bool ok = true;

  if (warp == 0 && lane == 0) {
    for (long long j = 0; j < nlocal && ok && !s_abort; ++j) {
      const int s = (int)(j % F::kStages);
      ok = mbar_wait(stage_free + 8 * s, ((uint32_t)(j / F::kStages) & 1u) ^ 1u);
      if (!ok) break;
      const int row0 = (int)((slot + j * nslots) * kRows);
      const uint32_t dst = sbase + s * F::kStageBytes;
      mbar_expect_tx(stage_full + 8 * s, F::kStageBytes);
#pragma unroll
      for (int a = 0; a < F::kAtoms; ++a) tma_load_2d(dst + a * 16384u, &xmap, a * 128, row0, stage_full + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    for (long long j = 0; j < nlocal && ok && !s_abort; ++j) {
      const int s = (int)(j % F::kStages), t = F::kSets == 2 ? (int)(j & 1) : 0;
      const uint32_t ph_set = F::kSets == 2 ? (uint32_t)(j >> 1) & 1u : (uint32_t)j & 1u;
      ok = mbar_wait(stage_full + 8 * s, (uint32_t)(j / F::kStages) & 1u);
      if (ok) ok = mbar_wait(acc_free + 8 * t, ph_set ^ 1u);
      if (!ok) break;
      tc_fence_after();
      const uint32_t st = sbase + s * F::kStageBytes, sb = sbase + F::kBOff;
      const uint32_t acc = tmem_base + (uint32_t)(t * F::kKT * 64);
#pragma unroll
      for (int kt = 0; kt < F::kKT; ++kt) {   // 32 E4M3 (32 bytes) per MMA, its own accumulator
        const uint32_t ka = (kt >> 2) * 16384u + (kt & 3) * 32u, kb = (kt >> 2) * 8192u + (kt & 3) * 32u;
        umma_fp8(acc + kt * 64, sw128_desc(st + ka), sw128_desc(sb + kb), kFp8Idesc);
      }
      umma_commit(stage_free + 8 * s);
      umma_commit(acc_full + 8 * t);
    }
    if (ok && nlocal > 0) {
      const long long j = nlocal - 1;
      const int s = (int)(j % F::kStages);
      ok = mbar_wait(stage_free + 8 * s, (uint32_t)(j / F::kStages) & 1u);
    }
  } else if (warp >= 4) {
    const uint32_t r = tid - 128;
    const uint32_t quarter = (uint32_t)(warp & 3) * 32u;
    const long long rmask = (1ll << rshift) - 1;
    const int bands = (int)((1ll << rshift) / 32);
    for (long long j = 0; j < nlocal; ++j) {
      const int t = F::kSets == 2 ? (int)(j & 1) : 0;
      const uint32_t ph_set = F::kSets == 2 ? (uint32_t)(j >> 1) & 1u : (uint32_t)j & 1u;
      if (r == 0) s_ok = (!s_abort && mbar_wait(acc_full + 8 * t, ph_set)) ? 1 : 0;
      named_sync(1, 128);
      if (!s_ok) {
        ok = r != 0;
        break;
      }
      tc_fence_after();
      const long long g = (slot + j * nslots) * kRows + r;
      const bool live = g < nrows;
      const long long b = g >> rshift, h = g & rmask;
      float rs[F::kKT];
#pragma unroll
      for (int kt = 0; kt < F::kKT; ++kt)
        rs[kt] = live ? __ldg(sx + (b * bands + (h >> 5)) * F::kKT + kt) : 0.0f;
      float v[64];
      const uint32_t taddr = tmem_base + (uint32_t)(t * F::kKT * 64) + (quarter << 16);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float acc[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[i] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < F::kKT; ++kt) {
          float w[16];
          tmem_ld16(taddr + kt * 64 + q * 16, w);
          tmem_wait_ld();
          const float f = rs[kt] * s_sc[(q >> 1) * F::kKT + kt];
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = fmaf(f, w[i], acc[i]);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) v[q * 16 + i] = acc[i];
      }
      tc_fence_before();
      named_sync(1, 128);
      if (r == 0) mbar_arrive(acc_free + 8 * t);
      if (live) {
        float* dst = out + ((b * L + (long long)nblk * 64) << rshift) + h;
#pragma unroll
        for (int c = 0; c < 64; ++c) dst[(long long)c << rshift] = v[c];
      }
    }
  }
  if (!ok) {
    s_abort = 1;
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 2) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(F::kTmemAlloc));
  }
}

}  // namespace tc
}  // namespace bridct
