// BF16x3 tensor-core form for batches of 64x64 arrays, both passes fused in one kernel.
//
// A tile is two arrays (128 rows of 64 FP32).  Pass 1 computes D1 = X C^T (rows (b,h), columns
// n) into TMEM; its epilogue splits every value exactly into three bf16 parts and writes them
// transposed, as rows (b,n) with K = h, straight into the shared-memory A operand of pass 2;
// pass 2 computes D2 = Z^T C^T, whose row (b,n) column k is Y_b[k][n] = (C X_b C^T)[k][n], and
// its epilogue stores Y.  The intermediate never leaves the SM: per tile, HBM sees 32 KB in
// and 32 KB out.  The inverse uses C^T in place of C for both passes.
//
// Both passes use the product grouping of the other tensor-core forms: Xh.[Ch|Cm|Cl] ->
// [big|small|smaller], Xm.[Ch|Cm] -> [small|smaller], Xl.Ch -> small (three MMAs per K step,
// M = 128, N = 192/128/64, K = 16), summed in FP32 by the epilogues.
//
// Warp roles (640 threads):
//   warp 0 lane 0   TMA producer: L2 prefetch of tile j+4, ring stage s <- X tile j
//   warp 1 lane 0   MMA issuer: pass 1 of tile j, then pass 2 of tile j-1
//   warp 2          TMEM allocator (512 columns: D1 at 0, D2 at 256, 192 each)
//   warps 4-7       split: stage s -> Xh, Xm in place + Xl into A buffer j%2
//   warps 8-15      epilogue 1: D1 -> registers (frees D1) -> Z^T splits into A2 buffer j%2;
//                   two warps per TMEM lane quarter, one per half of the 64 columns
//   warps 16-19     epilogue 2: D2 -> global stores of Y, 16 columns at a time (then frees D2)
// Every mbarrier wait is bounded; on expiry the CTA sets *err and all roles leave their loops.
#pragma once
#include "tc_blocks8.cuh"

namespace bridct {
namespace tc {

struct Fused64 {
  static constexpr int kThreads = 640;
  static constexpr int kStages = 2;
  static constexpr int kPrefetch = 4;            // tiles brought into L2 ahead of the ring
  static constexpr int kStageBytes = 32768;     // 128 rows x 64 FP32 (two SW128 boxes)
  static constexpr int kABufBytes = 16384;      // Xl (bf16)
  static constexpr int kA2Bytes = 3 * 16384;    // Zh | Zm | Zl (bf16, 128 rows x 64)
  static constexpr int kBBytes = 3 * 8192;      // [Ch; Cm; Cl], 64 rows each
  static constexpr int kAOff = kStages * kStageBytes;
  static constexpr int kA2Off = kAOff + 2 * kABufBytes;
  static constexpr int kBOff = kA2Off + 2 * kA2Bytes;
  static constexpr int kBarOff = kBOff + kBBytes;
  static constexpr int kDynamic = kBarOff + 256 + 1024;   // barriers, TMEM slot, alignment slack
  static constexpr uint32_t kD1 = 0, kD2 = 256;            // TMEM columns
  static constexpr int kTmemAlloc = 512;
  static_assert(kDynamic <= 232448, "shared memory budget");
};

struct Fused64Bars {
  uint32_t stage_full, stage_free, a_full, a_free, d1_full, d1_free, a2_full, a2_free, d2_full, d2_free;
  __device__ explicit Fused64Bars(uint32_t b)
      : stage_full(b), stage_free(b + 16), a_full(b + 32), a_free(b + 48), d1_full(b + 64), d1_free(b + 72),
        a2_full(b + 80), a2_free(b + 96), d2_full(b + 112), d2_free(b + 120) {}
  static constexpr int kSlotOff = 128;   // TMEM address slot
};

// One pass of the split products into the accumulator set at tmem (one thread).
// a0, a1, a2: shared addresses of the hi, mid and lo A parts; sb: the B image.
__device__ __forceinline__ void fused64_mmas(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t sb, uint32_t tmem) {
  constexpr uint32_t i192 = instr_desc(1, 192), i128 = instr_desc(1, 128), i64 = instr_desc(1, 64);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint64_t bd = sw128_desc(sb + k * 32u);
    umma(tmem, sw128_desc(a0 + k * 32u), bd, i192, k ? 1u : 0u, BF16X3);
    umma(tmem + 64, sw128_desc(a1 + k * 32u), bd, i128, 1u, BF16X3);
    umma(tmem + 64, sw128_desc(a2 + k * 32u), bd, i64, 1u, BF16X3);
  }
}

// xmap: the (batch*64 x 64) FP32 input rows (box 32 x 128, SWIZZLE_128B).  out: batch 64x64
// arrays.  bimage: [Ch; Cm; Cl] of C (forward) or C^T (inverse), 24 KB.
__global__ void __launch_bounds__(Fused64::kThreads, 1)
    k_tc64(const __grid_constant__ CUtensorMap xmap, float* __restrict__ out, const uint4* __restrict__ bimage,
           long long batch, int* __restrict__ err) {
  using F = Fused64;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(base);
  const Fused64Bars bars(sbase + F::kBarOff);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + F::kBarOff + Fused64Bars::kSlotOff);
  __shared__ volatile int s_abort;
  __shared__ volatile int s_group_ok[3];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long ntiles = (batch + 1) / 2;
  const long long nlocal = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < 2; ++i) {
      mbar_init(bars.stage_full + 8 * i, 1);
      mbar_init(bars.stage_free + 8 * i, 1);
      mbar_init(bars.a_full + 8 * i, 1);
      mbar_init(bars.a_free + 8 * i, 1);
      mbar_init(bars.a2_full + 8 * i, 1);
      mbar_init(bars.a2_free + 8 * i, 1);
    }
    mbar_init(bars.d1_full, 1);
    mbar_init(bars.d1_free, 1);
    mbar_init(bars.d2_full, 1);
    mbar_init(bars.d2_free, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(F::kTmemAlloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  {
    uint4* dst = reinterpret_cast<uint4*>(base + F::kBOff);
    for (int i = tid; i < F::kBBytes / 16; i += F::kThreads) dst[i] = __ldg(bimage + i);
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

  if (warp == 0 && lane == 0) {
    // The two-stage ring alone would expose a full DRAM latency per tile; tiles up to
    // kPrefetch ahead are brought into L2 first, so the ring's loads are served from L2.
    for (long long j = 0; j < nlocal && j < F::kPrefetch; ++j) {
      const int row0 = (int)((blockIdx.x + j * gridDim.x) * 128);
      tma_prefetch_2d(&xmap, 0, row0);
      tma_prefetch_2d(&xmap, 32, row0);
    }
    for (long long j = 0; j < nlocal && ok && !s_abort; ++j) {
      if (j + F::kPrefetch < nlocal) {
        const int rowp = (int)((blockIdx.x + (j + F::kPrefetch) * gridDim.x) * 128);
        tma_prefetch_2d(&xmap, 0, rowp);
        tma_prefetch_2d(&xmap, 32, rowp);
      }
      const int s = (int)(j % F::kStages);
      ok = mbar_wait(bars.stage_free + 8 * s, ((uint32_t)(j / F::kStages) & 1u) ^ 1u);
      if (!ok) break;
      const int row0 = (int)((blockIdx.x + j * gridDim.x) * 128);
      const uint32_t dst = sbase + s * F::kStageBytes;
      mbar_expect_tx(bars.stage_full + 8 * s, F::kStageBytes);
      tma_load_2d(dst, &xmap, 0, row0, bars.stage_full + 8 * s);
      tma_load_2d(dst + 16384u, &xmap, 32, row0, bars.stage_full + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    const uint32_t sb = sbase + F::kBOff, sa2 = sbase + F::kA2Off;
    for (long long j = 0; j <= nlocal && ok && !s_abort; ++j) {
      if (j < nlocal) {   // pass 1 of tile j
        const int s = (int)(j % F::kStages), a = (int)(j & 1);
        ok = mbar_wait(bars.a_full + 8 * a, (uint32_t)(j >> 1) & 1u);
        if (ok) ok = mbar_wait(bars.d1_free, ((uint32_t)j & 1u) ^ 1u);
        if (!ok) break;
        tc_fence_after();
        const uint32_t st = sbase + s * F::kStageBytes;
        fused64_mmas(st, st + 16384u, sbase + F::kAOff + a * F::kABufBytes, sb, tmem_base + F::kD1);
        umma_commit(bars.stage_free + 8 * s);
        umma_commit(bars.a_free + 8 * a);
        umma_commit(bars.d1_full);
      }
      if (j >= 1) {       // pass 2 of tile j - 1 from A2 buffer (j - 1) % 2
        const long long i = j - 1;
        const int q = (int)(i & 1);
        ok = mbar_wait(bars.a2_full + 8 * q, (uint32_t)(i >> 1) & 1u);
        if (ok) ok = mbar_wait(bars.d2_free, ((uint32_t)i & 1u) ^ 1u);
        if (!ok) break;
        tc_fence_after();
        const uint32_t a2 = sa2 + q * F::kA2Bytes;
        fused64_mmas(a2, a2 + 16384u, a2 + 32768u, sb, tmem_base + F::kD2);
        umma_commit(bars.a2_free + 8 * q);
        umma_commit(bars.d2_full);
      }
    }
    if (ok && nlocal > 0) {   // the last MMAs must finish before TMEM is freed
      const long long i = nlocal - 1;
      ok = mbar_wait(bars.a2_free + 8 * (int)(i & 1), (uint32_t)(i >> 1) & 1u);
    }
  } else if (warp >= 4 && warp < 8) {
    const uint32_t r = tid - 128;
    for (long long j = 0; j < nlocal; ++j) {
      const int s = (int)(j % F::kStages), a = (int)(j & 1);
      if (r == 0) {
        bool g = !s_abort && mbar_wait(bars.stage_full + 8 * s, (uint32_t)(j / F::kStages) & 1u);
        if (g) g = mbar_wait(bars.a_free + 8 * a, ((uint32_t)(j >> 1) & 1u) ^ 1u);
        s_group_ok[0] = g ? 1 : 0;
      }
      named_sync(1, 128);
      if (!s_group_ok[0]) {
        ok = r != 0;
        break;
      }
      split_tile<BF16X3>(base + s * F::kStageBytes, base + F::kAOff + a * F::kABufBytes, r);
      fence_async_smem();
      named_sync(1, 128);
      if (r == 0) mbar_arrive(bars.a_full + 8 * a);
    }
  } else if (warp >= 8 && warp < 16) {
    // epilogue 1: thread = TMEM lane = row (b = row / 64, h = row % 64) of the tile; warps 8-11
    // take columns n = 0..31, warps 12-15 columns 32..63
    const uint32_t r = tid - 256;                       // 0..255, leader r == 0
    const uint32_t quarter = (uint32_t)(warp & 3) * 32u;
    const uint32_t row = quarter + lane;
    const uint32_t ncol0 = (uint32_t)((warp - 8) >> 2) * 32u;
    const uint32_t b = row >> 6, h = row & 63u, odd = lane & 1u;
    for (long long j = 0; j < nlocal; ++j) {
      const int q = (int)(j & 1);
      if (r == 0) {
        bool g = !s_abort && mbar_wait(bars.d1_full, (uint32_t)j & 1u);
        if (g) g = mbar_wait(bars.a2_free + 8 * q, ((uint32_t)(j >> 1) & 1u) ^ 1u);
        s_group_ok[1] = g ? 1 : 0;
      }
      named_sync(2, 256);
      if (!s_group_ok[1]) {
        ok = r != 0;
        break;
      }
      tc_fence_after();
      float z[32];
      {
        const uint32_t taddr = tmem_base + F::kD1 + (quarter << 16) + ncol0;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          float big[16], sm[16], sm2[16];
          tmem_ld16(taddr + c * 16, big);
          tmem_ld16(taddr + 64 + c * 16, sm);
          tmem_ld16(taddr + 128 + c * 16, sm2);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) z[c * 16 + i] = big[i] + (sm[i] + sm2[i]);
        }
      }
      tc_fence_before();
      named_sync(2, 256);
      if (r == 0) mbar_arrive(bars.d1_free);
      // Z^T into A2: row (b, n), K = h.  Lanes h, h^1 exchange so that even lanes write the
      // bf16 pair (h, h+1) of row n0 and odd lanes the pair (h-1, h) of row n1 = n0 + 4 (rows
      // n0 and n0 + 4 differ in swizzle bit 2: the two half-warps hit disjoint banks).
      uint8_t* a2 = base + F::kA2Off + q * F::kA2Bytes;
#pragma unroll
      for (int g8 = 0; g8 < 4; ++g8)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int n0 = 8 * g8 + i, n1 = n0 + 4;
          const float send = odd ? z[n0] : z[n1];
          const float recv = __shfl_xor_sync(0xFFFFFFFFu, send, 1);
          const float x0 = odd ? recv : z[n0];
          const float x1 = odd ? z[n1] : recv;
          const uint32_t arow = b * 64u + ncol0 + (uint32_t)(odd ? n1 : n0);
          const uint32_t kw = h & ~1u;
          uint32_t hi, mid, lo;
          split_bf16x3_pair(x0, x1, hi, mid, lo);
          const uint32_t off = sw128(arow, kw >> 3) + (kw & 7u) * 2u;
          *reinterpret_cast<uint32_t*>(a2 + off) = hi;
          *reinterpret_cast<uint32_t*>(a2 + 16384u + off) = mid;
          *reinterpret_cast<uint32_t*>(a2 + 32768u + off) = lo;
        }
      fence_async_smem();
      named_sync(2, 256);
      if (r == 0) mbar_arrive(bars.a2_full + 8 * q);
    }
  } else if (warp >= 16) {
    // epilogue 2: thread r = TMEM lane = row (b, n); its columns k are Y_b[k][n]
    const uint32_t r = tid - 512;
    const uint32_t quarter = (uint32_t)(warp & 3) * 32u;
    for (long long j = 0; j < nlocal; ++j) {
      if (r == 0) s_group_ok[2] = (!s_abort && mbar_wait(bars.d2_full, (uint32_t)j & 1u)) ? 1 : 0;
      named_sync(3, 128);
      if (!s_group_ok[2]) {
        ok = r != 0;
        break;
      }
      tc_fence_after();
      const long long arr = (blockIdx.x + j * gridDim.x) * 2 + (r >> 6);
      float* dst = out + arr * 4096 + (r & 63u);
      const uint32_t taddr = tmem_base + F::kD2 + (quarter << 16);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float big[16], sm[16], sm2[16];
        tmem_ld16(taddr + c * 16, big);
        tmem_ld16(taddr + 64 + c * 16, sm);
        tmem_ld16(taddr + 128 + c * 16, sm2);
        tmem_wait_ld();
        if (arr < batch) {
#pragma unroll
          for (int i = 0; i < 16; ++i) dst[(c * 16 + i) * 64] = big[i] + (sm[i] + sm2[i]);
        }
      }
      tc_fence_before();
      named_sync(3, 128);
      if (r == 0) mbar_arrive(bars.d2_free);
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
