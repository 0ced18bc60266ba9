// Tensor-core precision forms for batches of 8x8 arrays (tcgen05 + TMEM + TMA).
//
// An 8x8 transform is linear in the 64 inputs: vec(Y) = K vec(X) with the Kronecker matrix
// K[(i,j),(k,l)] = Q[i][k] Q[j][l] (Q = orthonormal DCT-II, 8x8; K^T for the inverse).  For a
// tile of 128 arrays stored contiguously (128 rows of 64 floats) this is one GEMM
//     Y_tile (128 x 64) = X_tile (128 x 64) . K^T (64 x 64)
// i.e. tcgen05.mma with M = 128, N = 64, K = 64, A = X tile (K-major), B = K (K-major),
// D = FP32 accumulators in TMEM.  Split precision keeps FP32 accuracy:
//   BF16x3: X = Xh + Xm + Xl (exact truncation split) and K = Kh + Km + Kl (bf16 each); six products
//           Xh Kh + (Xh Km + Xm Kh + Xl Kh) + (Xh Kl + Xm Km), in three MMAs per K step.
//   TF32x3: X = Xh + Xl, K = Kh + Kl (tf32); three products Xh Kh + (Xh Kl + Xl Kh), two MMAs.
// K and its splits are computed in float64 on the host and uploaded once, already in the
// shared-memory image the MMA reads (128-byte swizzled, K-major).
//
// The kernel is a persistent, warp-specialized pipeline (one CTA per SM): a TMA producer
// fills a 4- or 5-deep ring of FP32 tiles (two 128x32 boxes each, 128-byte swizzle = exactly the
// UMMA K-major SW128 layout), four split warps turn ring tiles into operand tiles, one thread
// issues the MMAs into one of two TMEM accumulator sets, and four epilogue warps read the
// accumulator with tcgen05.ld (warp w owns TMEM lanes 32(w%4)..+31 = tile rows), write the
// result swizzled back into the ring tile and TMA-store it.  Loads, splits, MMAs and stores of
// consecutive tiles overlap.
//
// Every mbarrier wait is bounded: on expiry the role stops, the CTA records a nonzero code in
// *err, and all roles leave their loops (the others' waits expire too); TMEM is freed after
// the issuer has seen its last MMAs complete.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bridct {
namespace tc {

constexpr int kRows = 128;          // arrays per tile (MMA M)
constexpr int kCols = 64;           // elements per array (MMA N and K)
constexpr int kTmemCols = 192;      // per tile: [big | small | smaller] x 64 columns
constexpr int kTmemAlloc = 512;    // two tiles, rounded up to a power of two
constexpr uint32_t kSpinLimit = 1u << 26;   // bounded mbarrier polls (~seconds)

enum Form { BF16X3 = 1, TF32X3 = 2 };

// Shared-memory plan of the warp-specialized pipeline (per CTA, one CTA per SM):
//   kStages FP32 tiles (TMA ring; a tile later holds the TF32 Xh split and finally the
//   output tile for the TMA store), kABufs A-operand buffers (BF16: Xh|Xm|Xl, TF32: Xl),
//   the B image, and the mbarriers.
constexpr int kABufs = 2;
constexpr int kAccs = 2;            // TMEM accumulator sets (kTmemCols columns each)
constexpr int kTile = kRows * kCols * 4;   // FP32 tile bytes (32 KB)
constexpr int kMaxStages = 5;

// Splits live in the ring tile itself where they fit: a thread owns one tile row, reads its
// 64 FP32 values into registers and overwrites the same bytes (BF16: Xh over the first
// 128-byte box row, Xm over the second; TF32: Xh in place); only Xl needs an A buffer.
template <int FORM> struct Sizes;
template <> struct Sizes<BF16X3> {
  static constexpr int kStages = 5;
  static constexpr int kABuf = kRows * kCols * 2;         // Xl, bf16 (16 KB)
  static constexpr int kBImage = 3 * kCols * kCols * 2;   // Kh|Km|Kl (24 KB)
};
template <> struct Sizes<TF32X3> {
  static constexpr int kStages = 4;
  static constexpr int kABuf = kRows * kCols * 4;         // Xl, tf32 (32 KB)
  static constexpr int kBImage = 2 * kCols * kCols * 4;   // Kh|Kl (32 KB)
};

template <int FORM>
struct Layout {
  using S = Sizes<FORM>;
  static constexpr int kStages = S::kStages;
  static constexpr int kStageOff = 0;
  static constexpr int kAOff = kStages * kTile;
  static constexpr int kBOff = kAOff + kABufs * S::kABuf;
  static constexpr int kBarOff = kBOff + S::kBImage;
  // barriers: stage_full[5] stage_free[5] a_full[2] a_free[2] acc_full[2] acc_free[2], tmem slot
  static constexpr int kTmemSlot = 8 * (2 * kMaxStages + 2 * kABufs + 2 * kAccs);
  static constexpr int kBytes = kBarOff + kTmemSlot + 16;
  static constexpr int kDynamic = kBytes + 1024;          // room for 1024-byte alignment
  static constexpr int kBImage = S::kBImage;
  static_assert(kDynamic <= 232448, "shared memory budget");
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

// Instruction descriptor: D FP32, A/B format fmt (1 = BF16, 2 = TF32), K-major, M=128, N=n.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt, uint32_t n = kCols) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
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

// Brings a box of the tensor into L2 ahead of its load (no shared memory, no completion).
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y)
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
// Waits until at most one committed bulk group is still reading shared memory.
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
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

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Exact 3-way bf16 split of two FP32 values by truncation: hi = x with its low 16 bits cleared,
// mid = (x - hi) likewise, lo = x - hi - mid.  Both subtractions are exact (same exponent, the
// remaining significand bits), lo keeps at most 8 significant bits, so x = hi + mid + lo holds
// exactly and every part is its FP32 value's upper 16 bits.  Returns the packed bf16 pairs
// (first value in the low half).
__device__ __forceinline__ void split_bf16x3_pair(float x0, float x1, uint32_t& hi, uint32_t& mid, uint32_t& lo) {
  const uint32_t u0 = __float_as_uint(x0), u1 = __float_as_uint(x1);
  const float r0 = x0 - __uint_as_float(u0 & 0xFFFF0000u), r1 = x1 - __uint_as_float(u1 & 0xFFFF0000u);
  const uint32_t v0 = __float_as_uint(r0), v1 = __float_as_uint(r1);
  const float q0 = r0 - __uint_as_float(v0 & 0xFFFF0000u), q1 = r1 - __uint_as_float(v1 & 0xFFFF0000u);
  hi = __byte_perm(u0, u1, 0x7632);
  mid = __byte_perm(v0, v1, 0x7632);
  lo = __byte_perm(__float_as_uint(q0), __float_as_uint(q1), 0x7632);
}

// TF32 split of four values: Xh = x with its low 13 bits cleared (the tf32 the MMA reads),
// Xl = rna_tf32(x - Xh).
__device__ __forceinline__ void split_tf32x2(const float4& v, uint4& h, uint4& l) {
  h = make_uint4(__float_as_uint(v.x) & 0xFFFFE000u, __float_as_uint(v.y) & 0xFFFFE000u,
                 __float_as_uint(v.z) & 0xFFFFE000u, __float_as_uint(v.w) & 0xFFFFE000u);
  l = make_uint4(tf32_rna(v.x - __uint_as_float(h.x)), tf32_rna(v.y - __uint_as_float(h.y)),
                 tf32_rna(v.z - __uint_as_float(h.z)), tf32_rna(v.w - __uint_as_float(h.w)));
}

// Splits FP32 ring tile `stage` into A buffer `abuf` (thread r of 128 owns tile row r).
template <int FORM>
__device__ __forceinline__ void split_tile(uint8_t* stage, uint8_t* abuf, uint32_t r) {
  if constexpr (FORM == TF32X3) {
    // elementwise: Xh in place, Xl into the A buffer (same layout)
#pragma unroll
    for (int box = 0; box < 2; ++box)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t off = box * 16384u + sw128(r, j);
        uint4 h, l;
        split_tf32x2(*reinterpret_cast<const float4*>(stage + off), h, l);
        *reinterpret_cast<uint4*>(stage + off) = h;
        *reinterpret_cast<uint4*>(abuf + off) = l;
      }
  } else {
    // Row r holds 64 FP32 values: box 0 row r = elements 0..31, box 1 row r = 32..63.  bf16
    // chunk jp (elements 8jp..8jp+7) of Xh goes to box 0 row r chunk jp, of Xm to box 1 row r
    // chunk jp, of Xl to the A buffer, all in the K-major SW128 layout.  Box 0 is split first;
    // its Xm chunks would overwrite box 1 values not yet read, so they are held in registers
    // until box 1 has been read and split.
    uint32_t mid0[4][4];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float x[32];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float4 u = *reinterpret_cast<const float4*>(stage + half * 16384u + sw128(r, c));
        x[4 * c] = u.x; x[4 * c + 1] = u.y; x[4 * c + 2] = u.z; x[4 * c + 3] = u.w;
      }
#pragma unroll
      for (int jq = 0; jq < 4; ++jq) {
        const int jp = half * 4 + jq;
        uint32_t hi[4], mid[4], lo[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) split_bf16x3_pair(x[8 * jq + 2 * e], x[8 * jq + 2 * e + 1], hi[e], mid[e], lo[e]);
        const uint32_t off = sw128(r, jp);
        *reinterpret_cast<uint4*>(stage + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(abuf + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        if (half == 1) {
          *reinterpret_cast<uint4*>(stage + 16384u + off) = make_uint4(mid[0], mid[1], mid[2], mid[3]);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) mid0[jq][e] = mid[e];
        }
      }
    }
#pragma unroll
    for (int jq = 0; jq < 4; ++jq)
      *reinterpret_cast<uint4*>(stage + 16384u + sw128(r, jq)) =
          make_uint4(mid0[jq][0], mid0[jq][1], mid0[jq][2], mid0[jq][3]);
  }
}

// Issues the split-product MMAs of one tile (one thread).  sstage / sabuf / sb: shared
// addresses of the ring tile, the A buffer and the B image.
//
// Products that share an A split go into one MMA with the B splits stacked along N (the B
// image holds [Kh; Km; Kl] as 64-row blocks per 32- or 64-element K atom), so each A split is
// read once per K step.  The accumulator set of a tile is [big | small | smaller] (64 columns
// each): the dominant Xh.Kh product accumulates apart from the small products, whose own FP32
// accumulation losses are then negligible, and the epilogue adds the three in FP32.
//   BF16x3: Xh.[Kh|Km|Kl] -> [big|small|smaller], Xm.[Kh|Km] -> [small|smaller], Xl.Kh -> small
//   TF32x3: Xh.[Kh|Kl]    -> [big|small],         Xl.Kh     -> small
template <int FORM>
__device__ __forceinline__ void issue_mmas(uint32_t sstage, uint32_t sabuf, uint32_t sb, uint32_t tmem_d) {
  if constexpr (FORM == BF16X3) {
    constexpr uint32_t i192 = instr_desc(1, 192), i128 = instr_desc(1, 128), i64 = instr_desc(1, 64);
#pragma unroll
    for (int k = 0; k < 4; ++k) {   // K = 16 bf16 = 32 bytes per MMA
      const uint64_t bd = sw128_desc(sb + k * 32u);
      umma(tmem_d, sw128_desc(sstage + k * 32u), bd, i192, k ? 1u : 0u, BF16X3);
      umma(tmem_d + 64, sw128_desc(sstage + 16384u + k * 32u), bd, i128, 1u, BF16X3);
      umma(tmem_d + 64, sw128_desc(sabuf + k * 32u), bd, i64, 1u, BF16X3);
    }
  } else {
    constexpr uint32_t i128 = instr_desc(2, 128), i64 = instr_desc(2, 64);
#pragma unroll
    for (int k = 0; k < 8; ++k) {   // K = 8 tf32 = 32 bytes per MMA; 32-element atoms
      const uint32_t koff = (k >> 2) * 16384u + (k & 3) * 32u;
      const uint64_t bd = sw128_desc(sb + (k >> 2) * 16384u + (k & 3) * 32u);
      umma(tmem_d, sw128_desc(sstage + koff), bd, i128, k ? 1u : 0u, TF32X3);
      umma(tmem_d + 64, sw128_desc(sabuf + koff), bd, i64, 1u, TF32X3);
    }
  }
}

// Warp roles of k_tc8 (16 warps):
//   warp 0 lane 0  TMA producer: ring tile s <- X tile j      (waits stage_free, arms stage_full)
//                  (ring depth: 5 tiles for BF16x3, 4 for TF32x3)
//   warp 1 lane 0  MMA issuer: TMEM acc t <- A buffer a . B    (waits a_full, acc_free;
//                  commits to acc_full and a_free)
//   warp 2         TMEM allocator / deallocator
//   warps 4-7      split group 0: even tiles, ring tile s -> A buffer 0  (waits stage_full, a_free)
//   warps 8-11     split group 1: odd tiles, ring tile s -> A buffer 1
//   warps 12-15    epilogue: acc t -> ring tile s (16 columns at a time) -> TMA store
//                  (waits acc_full; frees acc t, then ring tile s once the store has read it;
//                  BF16x3, with its 5-tile ring, frees ring tile s one tile later so that the
//                  store's read overlaps the next tile's epilogue: +9% on the block batch, while
//                  TF32x3's 4-tile ring measured 8% slower with the later release)
// Tile j of this CTA uses ring tile j % kStages, A buffer j % 2 and accumulator j % 2.  The split
// is the longest role per tile, so two groups (one warp per sub-partition each) alternate.
constexpr int kTc8Threads = 512;

struct Bars {
  uint32_t stage_full, stage_free, a_full, a_free, acc_full, acc_free;
  __device__ Bars(uint32_t b)
      : stage_full(b), stage_free(b + 8 * kMaxStages), a_full(b + 16 * kMaxStages),
        a_free(b + 16 * kMaxStages + 8 * kABufs), acc_full(b + 16 * kMaxStages + 16 * kABufs),
        acc_free(b + 16 * kMaxStages + 16 * kABufs + 8 * kAccs) {}
};

// x, y: tensor maps of the (batch x 64) FP32 matrices (box 32 x 128, SWIZZLE_128B).
// bimage: the B operand shared-memory image (Layout<FORM>::kBImage bytes, 16-byte aligned).
template <int FORM>
__global__ void __launch_bounds__(kTc8Threads, 1) k_tc8(const __grid_constant__ CUtensorMap xmap,
                                                        const __grid_constant__ CUtensorMap ymap,
                                                        const uint4* __restrict__ bimage, int ntiles,
                                                        int* __restrict__ err) {
  using L = Layout<FORM>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(base);
  const Bars bars(sbase + L::kBarOff);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + L::kBarOff + L::kTmemSlot);
  constexpr int kStages = L::kStages;
  __shared__ volatile int s_abort;
  __shared__ volatile int s_group_ok[3];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntile_local = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < kStages; ++i) {
      mbar_init(bars.stage_full + 8 * i, 1);
      mbar_init(bars.stage_free + 8 * i, 1);
    }
    for (int i = 0; i < kABufs; ++i) {
      mbar_init(bars.a_full + 8 * i, 1);
      mbar_init(bars.a_free + 8 * i, 1);
    }
    for (int i = 0; i < kAccs; ++i) {
      mbar_init(bars.acc_full + 8 * i, 1);
      mbar_init(bars.acc_free + 8 * i, 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemAlloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  {
    uint4* dst = reinterpret_cast<uint4*>(base + L::kBOff);
    for (int i = tid; i < L::kBImage / 16; i += kTc8Threads) dst[i] = __ldg(bimage + i);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  bool ok = true;
  // Launched with programmatic stream serialization: the prologue above (barriers, TMEM, the B
  // image, which no kernel writes) overlaps the previous grid's tail; X and Y are touched only
  // after the wait.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (warp == 0 && lane == 0) {
    for (int j = 0; j < ntile_local && ok && !s_abort; ++j) {
      const int s = j % kStages;
      const uint32_t ph = (uint32_t)(j / kStages) & 1u;
      ok = mbar_wait(bars.stage_free + 8 * s, ph ^ 1u);
      if (!ok) break;
      const int tile = blockIdx.x + j * gridDim.x;
      const uint32_t dst = sbase + L::kStageOff + s * kTile;
      mbar_expect_tx(bars.stage_full + 8 * s, kTile);
      tma_load_2d(dst, &xmap, 0, tile * kRows, bars.stage_full + 8 * s);
      tma_load_2d(dst + 16384u, &xmap, 32, tile * kRows, bars.stage_full + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    for (int j = 0; j < ntile_local && ok && !s_abort; ++j) {
      const int s = j % kStages, a = j % kABufs, t = j % kAccs;
      ok = mbar_wait(bars.a_full + 8 * a, (uint32_t)(j / kABufs) & 1u);
      if (ok) ok = mbar_wait(bars.acc_free + 8 * t, ((uint32_t)(j / kAccs) & 1u) ^ 1u);
      if (!ok) break;
      tc_fence_after();
      issue_mmas<FORM>(sbase + L::kStageOff + s * kTile, sbase + L::kAOff + a * Sizes<FORM>::kABuf,
                       sbase + L::kBOff, tmem_base + t * kTmemCols);
      umma_commit(bars.acc_full + 8 * t);
      umma_commit(bars.a_free + 8 * a);
    }
    if (ok && ntile_local > 0) {   // the last MMAs must finish before TMEM is freed
      const int j = ntile_local - 1;
      ok = mbar_wait(bars.a_free + 8 * (j % kABufs), (uint32_t)(j / kABufs) & 1u);
    }
  } else if (warp >= 4 && warp < 12) {
    // Two split groups alternate tiles; in each, only the leader polls the mbarriers (bounded)
    // and broadcasts the outcome, so the group's named barrier is reached by all 128 threads
    // whatever the outcome.
    const int grp = (warp - 4) >> 2;            // 0: even tiles, 1: odd tiles
    const uint32_t r = tid - 128 - 128 * grp;
    const int bar_id = grp ? 3 : 1, ok_slot = grp ? 2 : 0;
    for (int j = grp; j < ntile_local; j += 2) {
      const int s = j % kStages, a = j % kABufs;
      if (r == 0) {
        bool g = !s_abort && mbar_wait(bars.stage_full + 8 * s, (uint32_t)(j / kStages) & 1u);
        if (g) g = mbar_wait(bars.a_free + 8 * a, ((uint32_t)(j / kABufs) & 1u) ^ 1u);
        s_group_ok[ok_slot] = g ? 1 : 0;
      }
      named_sync(bar_id, 128);
      if (!s_group_ok[ok_slot]) {
        ok = r != 0;      // the leader reports the expiry
        break;
      }
      split_tile<FORM>(base + L::kStageOff + s * kTile, base + L::kAOff + a * Sizes<FORM>::kABuf, r);
      fence_async_smem();
      named_sync(bar_id, 128);
      if (r == 0) mbar_arrive(bars.a_full + 8 * a);
    }
  } else if (warp >= 12) {
    const uint32_t r = tid - 384;               // tile row = TMEM lane
    const uint32_t quarter = (uint32_t)(warp & 3) * 32u;
    for (int j = 0; j < ntile_local; ++j) {
      const int s = j % kStages, t = j % kAccs;
      if (r == 0) s_group_ok[1] = (!s_abort && mbar_wait(bars.acc_full + 8 * t, (uint32_t)(j / kAccs) & 1u)) ? 1 : 0;
      named_sync(2, 128);
      if (!s_group_ok[1]) {
        ok = r != 0;
        break;
      }
      tc_fence_after();
      // the MMAs that read ring tile s are complete (acc_full), so the result goes straight into it
      const uint32_t taddr = tmem_base + t * kTmemCols + (quarter << 16);
      uint8_t* out = base + L::kStageOff + s * kTile;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float big[16], sm[16];
        tmem_ld16(taddr + q * 16, big);
        tmem_ld16(taddr + 64 + q * 16, sm);
        if constexpr (FORM == BF16X3) {
          float sm2[16];
          tmem_ld16(taddr + 128 + q * 16, sm2);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) sm[i] += sm2[i];
        } else {
          tmem_wait_ld();
        }
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
          const int col = q * 16 + c4 * 4;
          const uint32_t off = (col >> 5) * 16384u + sw128(r, (col & 31) >> 2);
          *reinterpret_cast<float4*>(out + off) =
              make_float4(big[4 * c4] + sm[4 * c4], big[4 * c4 + 1] + sm[4 * c4 + 1],
                          big[4 * c4 + 2] + sm[4 * c4 + 2], big[4 * c4 + 3] + sm[4 * c4 + 3]);
        }
      }
      tc_fence_before();
      fence_async_smem();
      named_sync(2, 128);
      if (r == 0) {
        mbar_arrive(bars.acc_free + 8 * t);
        const int tile = blockIdx.x + j * gridDim.x;
        tma_store_2d(&ymap, 0, tile * kRows, sbase + L::kStageOff + s * kTile);
        tma_store_2d(&ymap, 32, tile * kRows, sbase + L::kStageOff + s * kTile + 16384u);
        bulk_commit();
        if constexpr (FORM == BF16X3) {
          if (j > 0) {               // the previous tile's store has read its ring tile
            bulk_wait_read1();
            mbar_arrive(bars.stage_free + 8 * ((j - 1) % kStages));
          }
        } else {
          bulk_wait_read0();
          mbar_arrive(bars.stage_free + 8 * s);
        }
      }
    }
    if (r == 0) {
      if (FORM == BF16X3 && ok && ntile_local > 0) {
        bulk_wait_read0();
        mbar_arrive(bars.stage_free + 8 * ((ntile_local - 1) % kStages));
      }
      bulk_wait0();
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemAlloc));
  }
}

}  // namespace tc
}  // namespace bridct
