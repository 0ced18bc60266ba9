// Tensor-core precision forms for batches of 8x8 arrays (tcgen05 + TMEM + TMA).
//
// An 8x8 transform is linear in the 64 inputs: vec(Y) = K vec(X) with the Kronecker matrix
// K[(i,j),(k,l)] = Q[i][k] Q[j][l] (Q = orthonormal DCT-II, 8x8; K^T for the inverse).  For a
// tile of 128 arrays stored contiguously (128 rows of 64 floats) this is one GEMM
//     Y_tile (128 x 64) = X_tile (128 x 64) . K^T (64 x 64)
// i.e. tcgen05.mma with M = 128, N = 64, K = 64, A = X tile (K-major), B = K (K-major),
// D = FP32 accumulator in 64 TMEM columns.  Split precision keeps FP32 accuracy:
//   BF16x3: X = Xh + Xm + Xl and K = Kh + Km + Kl (bf16 each); six products
//           Xl Kh + Xm Km + Xh Kl + Xm Kh + Xh Km + Xh Kh accumulate in FP32 (smallest first).
//   TF32x3: X = Xh + Xl, K = Kh + Kl (tf32); three products Xl Kh + Xh Kl + Xh Kh.
// K and its splits are computed in float64 on the host and uploaded once, already in the
// shared-memory image the MMA reads (128-byte swizzled, K-major).
//
// Per tile: one elected thread starts a TMA load of the FP32 tile (two 128x32 boxes, 128-byte
// swizzle, exactly the UMMA K-major SW128 layout), the 128 threads split it into the operand
// tiles, one thread issues the MMAs and commits them to an mbarrier, the 4 warps read the
// accumulator back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows), write it
// swizzled to shared memory and one thread TMA-stores the tile.  Two CTAs per SM overlap each
// other's load / MMA / store phases.
//
// Every mbarrier wait is bounded: on expiry the CTA records an error code in *err, stops
// issuing work, waits (bounded) for its own bulk stores, frees its TMEM and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bridct {
namespace tc {

constexpr int kRows = 128;          // arrays per tile (MMA M)
constexpr int kCols = 64;           // elements per array (MMA N and K)
constexpr int kThreads = 128;
constexpr int kTmemCols = 64;
constexpr uint32_t kSpinLimit = 1u << 26;   // bounded mbarrier polls (~seconds)

enum Form { BF16X3 = 1, TF32X3 = 2 };

// Shared-memory byte sizes of the operand images.
template <int FORM> struct Sizes;
template <> struct Sizes<BF16X3> {
  static constexpr int kStage = kRows * kCols * 4;        // FP32 staging tile (TMA target)
  static constexpr int kATile = kRows * kCols * 2;        // one bf16 A split (16 KB)
  static constexpr int kANum = 3;
  static constexpr int kBTile = kCols * kCols * 2;        // one bf16 B split (8 KB)
  static constexpr int kBNum = 3;
};
template <> struct Sizes<TF32X3> {
  static constexpr int kStage = kRows * kCols * 4;        // FP32 tile; becomes Xh in place
  static constexpr int kATile = kRows * kCols * 4;        // Xl (32 KB)
  static constexpr int kANum = 1;
  static constexpr int kBTile = kCols * kCols * 4;        // one tf32 B split (16 KB)
  static constexpr int kBNum = 2;
};

template <int FORM>
struct Layout {
  using S = Sizes<FORM>;
  static constexpr int kStageOff = 0;
  static constexpr int kAOff = kStageOff + S::kStage;
  static constexpr int kBOff = kAOff + S::kANum * S::kATile;
  static constexpr int kBarOff = kBOff + S::kBNum * S::kBTile;   // 2 mbarriers + tmem slot
  static constexpr int kBytes = kBarOff + 64;
  static constexpr int kDynamic = kBytes + 1024;                  // room for 1024-B alignment
  static constexpr int kBImage = S::kBNum * S::kBTile;
};

// Byte offset of 16-byte chunk `chunk` of row `row` in a K-major SW128 atom column
// (rows of 128 bytes, 8-row groups of 1024 bytes, chunk index XOR row%8).
__host__ __device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);          // start address
  d |= (uint64_t)1 << 16;                            // leading byte offset (unused for SW128 K-major)
  d |= (uint64_t)(1024u >> 4) << 32;                 // stride byte offset
  d |= (uint64_t)1 << 46;                            // descriptor version (sm100)
  d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D FP32, A/B format fmt (1 = BF16, 2 = TF32), K-major, M=128, N=64.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(kCols >> 3) << 17) |
         ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded parity wait; returns false when the poll budget is exhausted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                     uint32_t accumulate, int form) {
  if (form == BF16X3) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  }
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
      " [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// Splits the FP32 staging tile into the A operand tiles.  Thread t owns tile row t.
template <int FORM>
__device__ __forceinline__ void split_tile(uint8_t* base) {
  using L = Layout<FORM>;
  const uint32_t r = threadIdx.x;
  uint8_t* stage = base + L::kStageOff;
  uint8_t* a = base + L::kAOff;
  if constexpr (FORM == TF32X3) {
    // elementwise: Xh = rna_tf32(X) in place, Xl = X - Xh in the second tile (same layout)
#pragma unroll
    for (int box = 0; box < 2; ++box)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t off = box * 16384u + sw128(r, j);
        float4 v = *reinterpret_cast<const float4*>(stage + off);
        const uint32_t h0 = tf32_rna(v.x), h1 = tf32_rna(v.y), h2 = tf32_rna(v.z), h3 = tf32_rna(v.w);
        float4 lo = make_float4(v.x - __uint_as_float(h0), v.y - __uint_as_float(h1),
                                v.z - __uint_as_float(h2), v.w - __uint_as_float(h3));
        *reinterpret_cast<uint4*>(stage + off) = make_uint4(h0, h1, h2, h3);
        *reinterpret_cast<float4*>(a + off) = lo;
      }
  } else {
    // bf16 chunk j' holds elements 8j'..8j'+7 = fp32 chunks 2j', 2j'+1 of box j'/4
#pragma unroll
    for (int jp = 0; jp < 8; ++jp) {
      const int box = jp >> 2;
      const int c0 = (2 * jp) & 7;
      const float4 u = *reinterpret_cast<const float4*>(stage + box * 16384u + sw128(r, c0));
      const float4 w = *reinterpret_cast<const float4*>(stage + box * 16384u + sw128(r, c0 + 1));
      const float x[8] = {u.x, u.y, u.z, u.w, w.x, w.y, w.z, w.w};
      uint32_t hi[4], mid[4], lo[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        __nv_bfloat16 h[2], m[2], l[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const float v = x[2 * e + q];
          h[q] = __float2bfloat16_rn(v);
          const float r1 = v - __bfloat162float(h[q]);
          m[q] = __float2bfloat16_rn(r1);
          l[q] = __float2bfloat16_rn(r1 - __bfloat162float(m[q]));
        }
        hi[e] = pack_bf16(h[0], h[1]);
        mid[e] = pack_bf16(m[0], m[1]);
        lo[e] = pack_bf16(l[0], l[1]);
      }
      const uint32_t off = sw128(r, jp);
      *reinterpret_cast<uint4*>(a + 0 * 16384u + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4*>(a + 1 * 16384u + off) = make_uint4(mid[0], mid[1], mid[2], mid[3]);
      *reinterpret_cast<uint4*>(a + 2 * 16384u + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
  }
}

// Issues the split-product MMAs of one tile (one thread).
template <int FORM>
__device__ __forceinline__ void issue_mmas(uint8_t* base, uint32_t tmem_d) {
  using L = Layout<FORM>;
  const uint32_t sbase = smem_u32(base);
  if constexpr (FORM == BF16X3) {
    // (A split, B split) products, smallest magnitude first: A = {Xh, Xm, Xl}, B = {Kh, Km, Kl}
    constexpr int pa[6] = {2, 1, 0, 1, 0, 0};
    constexpr int pb[6] = {0, 1, 2, 0, 1, 0};
    constexpr uint32_t idesc = instr_desc(1);
#pragma unroll
    for (int p = 0; p < 6; ++p)
#pragma unroll
      for (int k = 0; k < 4; ++k) {   // K = 16 bf16 = 32 bytes per MMA
        const uint64_t ad = sw128_desc(sbase + L::kAOff + pa[p] * 16384u + k * 32u);
        const uint64_t bd = sw128_desc(sbase + L::kBOff + pb[p] * 8192u + k * 32u);
        umma(tmem_d, ad, bd, idesc, (p | k) ? 1u : 0u, BF16X3);
      }
  } else {
    // A = {Xh (in the staging tile), Xl}, B = {Kh, Kl}; products Xl Kh, Xh Kl, Xh Kh
    constexpr uint32_t aoff[3] = {(uint32_t)L::kAOff, (uint32_t)L::kStageOff, (uint32_t)L::kStageOff};
    constexpr int pb[3] = {0, 1, 0};
    constexpr uint32_t idesc = instr_desc(2);
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int k = 0; k < 8; ++k) {   // K = 8 tf32 = 32 bytes per MMA; 32-element atoms
        const uint32_t koff = (k >> 2) * 16384u + (k & 3) * 32u;
        const uint32_t kboff = (k >> 2) * 8192u + (k & 3) * 32u;
        const uint64_t ad = sw128_desc(sbase + aoff[p] + koff);
        const uint64_t bd = sw128_desc(sbase + L::kBOff + pb[p] * 16384u + kboff);
        umma(tmem_d, ad, bd, idesc, (p | k) ? 1u : 0u, TF32X3);
      }
  }
}

// x, y: tensor maps of the (batch x 64) FP32 matrices (box 32 x 128, SWIZZLE_128B).
// bimage: the B operand shared-memory image (Layout<FORM>::kBImage bytes, 16-byte aligned).
template <int FORM>
__global__ void __launch_bounds__(kThreads) k_tc8(const __grid_constant__ CUtensorMap xmap,
                                                  const __grid_constant__ CUtensorMap ymap,
                                                  const uint4* __restrict__ bimage, int ntiles,
                                                  int* __restrict__ err) {
  using L = Layout<FORM>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t bar_load = smem_u32(base + L::kBarOff);
  const uint32_t bar_mma = bar_load + 8;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + L::kBarOff + 16);
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5;

  if (tid == 0) {
    s_abort = 0;
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // B operand image: plain copy, once per CTA
  {
    uint4* dst = reinterpret_cast<uint4*>(base + L::kBOff);
    for (int i = tid; i < L::kBImage / 16; i += kThreads) dst[i] = __ldg(bimage + i);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_d = *tmem_slot;
  uint32_t phase = 0;
  bool ok = true;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (tid == 0) {
      bulk_wait_read0();                                // previous tile's store has read its staging
      mbar_expect_tx(bar_load, 2u * 16384u);
      tma_load_2d(smem_u32(base + L::kStageOff), &xmap, 0, tile * kRows, bar_load);
      tma_load_2d(smem_u32(base + L::kStageOff) + 16384u, &xmap, 32, tile * kRows, bar_load);
    }
    ok = mbar_wait(bar_load, phase);
    if (__syncthreads_or(!ok)) break;
    split_tile<FORM>(base);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      issue_mmas<FORM>(base, tmem_d);
      umma_commit(bar_mma);
    }
    ok = mbar_wait(bar_mma, phase);
    if (__syncthreads_or(!ok)) break;
    tc_fence_after();
    // epilogue: TMEM lane (32 warp + lane) = tile row; 64 FP32 columns -> swizzled staging
    {
      const uint32_t row = tid;
      const uint32_t lane_addr = tmem_d + ((uint32_t)(warp * 32) << 16);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float v[16];
        tmem_ld16(lane_addr + q * 16, v);
        tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int col = q * 16 + c * 4;
          const uint32_t off = (col >> 5) * 16384u + sw128(row, (col & 31) >> 2);
          *reinterpret_cast<float4*>(base + L::kStageOff + off) =
              make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        }
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tma_store_2d(&ymap, 0, tile * kRows, smem_u32(base + L::kStageOff));
      tma_store_2d(&ymap, 32, tile * kRows, smem_u32(base + L::kStageOff) + 16384u);
      bulk_commit();
    }
    phase ^= 1u;
  }
  if (tid == 0) {
    bulk_wait0();
    if (!ok) atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(kTmemCols));
  }
}

}  // namespace tc
}  // namespace bridct
