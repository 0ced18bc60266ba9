// FP8 (E4M3) tensor-core form with per-tile scaling, for every axis from 8 to 1024.
//
// A 2D transform is two row passes, as in the split-precision forms, but the operands are
// quantized instead of split: every tile of min(R, 32) rows x min(L, 32) columns of an array
// (32 x 32 where both axes allow) gets its own scale s = max|tile| / 448 (the largest finite E4M3
// value) and is stored as E4M3 codes, and C (or C^T) is quantized the same way on the host.
// A row of length L spans L/32 K-tiles with different scales, so each K-tile's product (one
// kind::f8f6f4 MMA, K = 32) accumulates in its own TMEM block and the epilogue forms
// sum_t sX(row band, t) * sC(column band, t) * acc_t in FP32.  One refinement step on the host
// side of the form recovers accuracy:
//     Y = Y8 + FP8(X - DCT-III_fp32(Y8)),  with the residual taken in FP32 by the plain form.
//
// Rows shorter than 128 codes run as super-rows of LS = 128 codes (SUB = 128 / L consecutive
// rows) against a block-diagonal B of SUB copies of C_L; a K-tile of a super-row then holds
// 32 / L whole rows (L < 32) or a 32-column band of one row, of one scale tile either way.
//
// k_quant8: one warp per scale tile: warp max of |x|, scale, E4M3 codes.
// k_fp8pass<LS, SUB, UKT> (256 threads): warp 0 TMA producer (E4M3 super-rows, 128-byte boxes),
// warp 1 MMA issuer, warp 2 TMEM allocator, warps 4-7 epilogue (scales, sum, transposed stores).
// The pipeline unit is one M-tile's UKT K-tiles (UKT * 32 codes of 128 super-rows): 128- and
// 256-code rows take a whole row per unit, 512- and 1024-code rows stream 4 K-tiles per unit
// through two TMEM accumulator sets while the epilogue sums the units of a tile in registers.
#pragma once
#include <cuda_fp8.h>

#include "tc_blocks8.cuh"

namespace bridct {
namespace tc {

constexpr float kE4M3Max = 448.0f;

// rows: nrows x L FP32 (arrays of R rows); q: E4M3 codes, same layout; scales: one per tile of
// TR = 1 << tr_shift rows (TR = min(R, 32)) and TL = min(L, 32) columns, tile index
// (row / TR) * (L / TL) + column / TL.  ntiles = nrows / TR * L / TL.  A tile's 16..256 float4
// groups go to 32 lanes, or to 16 when it has only 16 (8 x 8 tiles: two tiles per warp).  Block 0
// also zeroes the `pad` bytes after the codes, the tail of the pass's last (partial) super-row.
__host__ __device__ constexpr int quant8_tiles_per_warp(int tr_shift, int L) {
  return tr_shift + (L < 32 ? (L == 8 ? 1 : 2) : 3) < 5 ? 2 : 1;
}

__global__ void __launch_bounds__(256) k_quant8(const float* __restrict__ rows, uint8_t* __restrict__ q,
                                                float* __restrict__ scales, long long ntiles, int L, int tr_shift,
                                                int pad) {
  const int lane = threadIdx.x & 31;
  const int tl_shift = L == 8 ? 3 : L == 16 ? 4 : 5;          // TL = min(L, 32)
  const int ql = tl_shift - 2;                                  // float4 groups of a tile row
  const int n4_shift = tr_shift + ql;                           // float4 groups of a tile (16..256)
  const int lpt_shift = n4_shift < 5 ? n4_shift : 5;            // lanes per tile
  const int bands_shift = (31 - __clz(L)) - tl_shift;           // tiles across a row
  const long long total = ntiles << (tr_shift + tl_shift);
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i < pad; i += blockDim.x) q[total + i] = 0;
  const long long t = ((((long long)blockIdx.x << 3) + (threadIdx.x >> 5)) << (5 - lpt_shift)) + (lane >> lpt_shift);
  const int sl = lane & ((1 << lpt_shift) - 1);
  const bool live = t < ntiles;
  const long long row0 = (t >> bands_shift) << tr_shift;
  const int col0 = (int)(t & ((1 << bands_shift) - 1)) << tl_shift;
  const int n4 = live ? 1 << n4_shift : 0;
  float4 v[8];
  float amax = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int i = sl + (k << lpt_shift);
    v[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (i < n4) {
      v[k] = __ldg(reinterpret_cast<const float4*>(rows + (row0 + (i >> ql)) * L + col0 + ((i & ((1 << ql) - 1)) << 2)));
      amax = fmaxf(amax, fmaxf(fmaxf(fabsf(v[k].x), fabsf(v[k].y)), fmaxf(fabsf(v[k].z), fabsf(v[k].w))));
    }
  }
  for (int o = (1 << lpt_shift) >> 1; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xFFFFFFFFu, amax, o));
  const float s = amax > 0.0f ? amax / kE4M3Max : 1.0f;
  const float inv = 1.0f / s;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int i = sl + (k << lpt_shift);
    if (i < n4) {
      const __nv_fp8x2_storage_t lo =
          __nv_cvt_float2_to_fp8x2(make_float2(v[k].x * inv, v[k].y * inv), __NV_SATFINITE, __NV_E4M3);
      const __nv_fp8x2_storage_t hi =
          __nv_cvt_float2_to_fp8x2(make_float2(v[k].z * inv, v[k].w * inv), __NV_SATFINITE, __NV_E4M3);
      *reinterpret_cast<uint32_t*>(q + (row0 + (i >> ql)) * L + col0 + ((i & ((1 << ql) - 1)) << 2)) =
          (uint32_t)lo | ((uint32_t)hi << 16);
    }
  }
  if (live && sl == 0) scales[t] = s;
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

template <int LS, int SUB, int UKT>
struct Fp8Layout {
  static constexpr int kThreads = 256;
  static constexpr int L = LS / SUB;                  // row length
  static constexpr int kKT = LS / 32;                 // K-tiles of a super-row (one MMA and accumulator each)
  static constexpr int kUnits = kKT / UKT;            // pipeline units per M-tile
  static constexpr int kStageBytes = (UKT / 4) * 16384;   // 128 super-rows x UKT * 32 codes
  static constexpr int kBBytes = (LS / 128) * 8192;   // 64 rows x LS codes
  static constexpr int kSets = 2 * UKT * 64 <= 512 ? 2 : 1;   // TMEM accumulator sets
  static constexpr int kTmemAlloc = kSets * UKT * 64 <= 256 ? 256 : 512;
  static constexpr int kStages = (196608 - kBBytes) / kStageBytes < 8 ? (196608 - kBBytes) / kStageBytes : 8;
  static constexpr int kBOff = kStages * kStageBytes;
  // rows shorter than 64 points: each epilogue warp's 64 x 32 outputs, staged for the stores
  static constexpr int kStoreOff = kBOff + kBBytes;
  static constexpr int kStoreBytes = L < 64 ? 4 * 64 * 33 * 4 : 0;
  static constexpr int kScOff = kStoreOff + kStoreBytes;   // sC of this CTA's two column bands
  static constexpr int kBarOff = kScOff + 2 * kKT * 4 + 64;
  static constexpr int kDynamic = ((kBarOff + 255) / 256) * 256 + 256 + 1024;
  static_assert(LS % 128 == 0 && kKT % UKT == 0 && UKT % 4 == 0, "FP8 pass geometry");
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

// xmap: (ceil(nrows / SUB) x LS) E4M3 super-rows (box 128 x 128 bytes, SWIZZLE_128B); sx: their
// scale tiles (k_quant8's layout, tr_shift = min(rshift, 5)); bimage: LS/64 slices of 64 rows x
// LS codes; sc: C's tile scales [LS/32 column bands][LS/32 K-tiles]; out: FP32 arrays written
// transposed (R = 1 << rshift rows of length L in, L rows of length R out).
template <int LS, int SUB, int UKT>
__global__ void __launch_bounds__(256, 1)
    k_fp8pass(const __grid_constant__ CUtensorMap xmap, const float* __restrict__ sx, float* __restrict__ out,
              const uint4* __restrict__ bimage, const float* __restrict__ sc, long long nrows, int rshift,
              int* __restrict__ err) {
  using F = Fp8Layout<LS, SUB, UKT>;
  constexpr int L = F::L;
  constexpr int kBlocks = LS / 64;
  constexpr int kSpan = L > 32 ? L : 32;             // codes whose K-tiles feed one output column
  constexpr int kBandsPerRow = L > 32 ? L / 32 : 1;  // scale tiles across a row
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(base);
  const uint32_t bar = sbase + F::kBarOff;
  const uint32_t stage_full = bar, stage_free = bar + 8 * F::kStages, acc_full = bar + 16 * F::kStages,
                 acc_free = acc_full + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + F::kBarOff + 16 * F::kStages + 32);
  float* s_sc = reinterpret_cast<float*>(base + F::kScOff);
  float* s_store = reinterpret_cast<float*>(base + F::kStoreOff);
  __shared__ volatile int s_abort;
  __shared__ volatile int s_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nblk = blockIdx.x % kBlocks;
  const long long slot = blockIdx.x / kBlocks, nslots = gridDim.x / kBlocks;
  const long long srows = (nrows + SUB - 1) / SUB;
  const long long mtiles = (srows + kRows - 1) / kRows;
  const long long nlocal = slot < mtiles ? (mtiles - 1 - slot) / nslots + 1 : 0;
  const long long nunits = nlocal * F::kUnits;

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
  // Launched with programmatic stream serialization: the prologue above (barriers, TMEM, the
  // coefficient image, which no kernel writes) overlaps the previous grid's tail; the data is
  // touched only after the wait.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  // Unit j: M-tile j / kUnits of this CTA, K-tiles (j % kUnits) * UKT ...; stage j % kStages,
  // accumulator set j % kSets.
  if (warp == 0 && lane == 0) {
    for (long long j = 0; j < nunits && ok && !s_abort; ++j) {
      const int s = (int)(j % F::kStages), u = (int)(j % F::kUnits);
      ok = mbar_wait(stage_free + 8 * s, ((uint32_t)(j / F::kStages) & 1u) ^ 1u);
      if (!ok) break;
      const int row0 = (int)((slot + (j / F::kUnits) * nslots) * kRows);
      const uint32_t dst = sbase + s * F::kStageBytes;
      mbar_expect_tx(stage_full + 8 * s, F::kStageBytes);
#pragma unroll
      for (int a = 0; a < UKT / 4; ++a)
        tma_load_2d(dst + a * 16384u, &xmap, (u * (UKT / 4) + a) * 128, row0, stage_full + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    for (long long j = 0; j < nunits && ok && !s_abort; ++j) {
      const int s = (int)(j % F::kStages), t = F::kSets == 2 ? (int)(j & 1) : 0, u = (int)(j % F::kUnits);
      const uint32_t ph_set = F::kSets == 2 ? (uint32_t)(j >> 1) & 1u : (uint32_t)j & 1u;
      ok = mbar_wait(stage_full + 8 * s, (uint32_t)(j / F::kStages) & 1u);
      if (ok) ok = mbar_wait(acc_free + 8 * t, ph_set ^ 1u);
      if (!ok) break;
      tc_fence_after();
      const uint32_t st = sbase + s * F::kStageBytes, sb = sbase + F::kBOff;
      const uint32_t acc = tmem_base + (uint32_t)(t * UKT * 64);
#pragma unroll
      for (int kt = 0; kt < UKT; ++kt) {   // 32 E4M3 (32 bytes) per MMA, its own accumulator
        const int kg = u * UKT + kt;
        const uint32_t ka = (kt >> 2) * 16384u + (kt & 3) * 32u, kb = (kg >> 2) * 8192u + (kg & 3) * 32u;
        umma_fp8(acc + kt * 64, sw128_desc(st + ka), sw128_desc(sb + kb), kFp8Idesc);
      }
      umma_commit(stage_free + 8 * s);
      umma_commit(acc_full + 8 * t);
    }
    if (ok && nunits > 0) {
      const long long j = nunits - 1;
      const int s = (int)(j % F::kStages);
      ok = mbar_wait(stage_free + 8 * s, (uint32_t)(j / F::kStages) & 1u);
    }
  } else if (warp >= 4) {
    const uint32_t r = tid - 128;
    const uint32_t quarter = (uint32_t)(warp & 3) * 32u;
    const long long rmask = (1ll << rshift) - 1;
    const int tr_shift = rshift < 5 ? rshift : 5;
    float v[64];
    for (long long j = 0; j < nunits; ++j) {
      const int t = F::kSets == 2 ? (int)(j & 1) : 0, u = (int)(j % F::kUnits);
      const uint32_t ph_set = F::kSets == 2 ? (uint32_t)(j >> 1) & 1u : (uint32_t)j & 1u;
      if (r == 0) s_ok = (!s_abort && mbar_wait(acc_full + 8 * t, ph_set)) ? 1 : 0;
      named_sync(1, 128);
      if (!s_ok) {
        ok = r != 0;
        break;
      }
      tc_fence_after();
      const long long gs = (slot + (j / F::kUnits) * nslots) * kRows + r;   // this thread's super-row
      // data scale of each of the unit's K-tiles: its first row and column band
      float rs[UKT];
#pragma unroll
      for (int kt = 0; kt < UKT; ++kt) {
        const int kg = u * UKT + kt;
        const long long g = gs * SUB + (kg * 32) / L;
        rs[kt] = g < nrows ? __ldg(sx + (g >> tr_shift) * kBandsPerRow + kg % kBandsPerRow) : 0.0f;
      }
      const uint32_t taddr = tmem_base + (uint32_t)(t * UKT * 64) + (quarter << 16);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        // K-tiles that feed output columns nblk * 64 + q * 16 ... + 15 (one row of the super-row,
        // or one 32-code group of rows): the others meet zeros of the block-diagonal B
        const int lo = ((nblk * 64 + q * 16) / kSpan) * (kSpan / 32), hi = lo + kSpan / 32;
        float acc[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[i] = u == 0 ? 0.0f : v[q * 16 + i];
#pragma unroll
        for (int kt = 0; kt < UKT; ++kt) {
          const int kg = u * UKT + kt;
          if (kg < lo || kg >= hi) continue;
          float w[16];
          tmem_ld16(taddr + kt * 64 + q * 16, w);
          tmem_wait_ld();
          const float f = rs[kt] * s_sc[(q >> 1) * F::kKT + kg];
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = fmaf(f, w[i], acc[i]);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) v[q * 16 + i] = acc[i];
      }
      tc_fence_before();
      named_sync(1, 128);
      if (r == 0) mbar_arrive(acc_free + 8 * t);
      if (u == F::kUnits - 1) {
        if constexpr (SUB == 1) {
          if (gs < nrows) {
            const long long b = gs >> rshift, h = gs & rmask;
            float* dst = out + ((b * L + (long long)nblk * 64) << rshift) + h;
#pragma unroll
            for (int c = 0; c < 64; ++c) dst[(long long)c << rshift] = v[c];
          }
        } else if constexpr (L == 64) {
#pragma unroll
          for (int c = 0; c < 64; ++c) {
            const long long g = gs * SUB + nblk;
            if (g < nrows) {
              const long long b = g >> rshift, h = g & rmask;
              out[((b * L + c) << rshift) + h] = v[c];
            }
          }
        } else {
          // The CTA's 64 columns are RUN = 64 / L whole sub-rows s0 + s of each super-row, so
          // rows g = gs * SUB + s0 + s of one output column k come in runs of RUN consecutive
          // rows: the warp stages its 32 super-rows x 64 columns (column-major, pitch 33) and
          // stores element e = (k * 32 + lane_src) * RUN + s, a run of RUN floats per super-row.
          constexpr int RUN = 64 / L;
          float* wb = s_store + (warp & 3) * (64 * 33);
          __syncwarp();
#pragma unroll
          for (int c = 0; c < 64; ++c) wb[c * 33 + lane] = v[c];
          __syncwarp();
          const long long gs0 = gs - lane;
#pragma unroll 8
          for (int e = lane; e < 64 * 32; e += 32) {
            const int s = e % RUN, src = (e / RUN) % 32, k = e / (RUN * 32);
            const long long g = (gs0 + src) * SUB + nblk * RUN + s;
            if (g < nrows) {
              const long long b = g >> rshift, h = g & rmask;
              out[((b * L + k) << rshift) + h] = wb[(s * L + k) * 33 + src];
            }
          }
        }
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
