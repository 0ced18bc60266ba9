// Tensor-core precision forms for arrays of any supported shape but 8x8 (tcgen05 + TMEM + TMA).
//
// A 2D transform Y = C_H X C_W^T is computed as two row passes.  A row pass takes a matrix of
// contiguous rows of length L (rows grouped into arrays of R rows), multiplies every row by
// C_L^T (forward) or C_L (inverse) on the tensor cores, and writes every array's result
// transposed:
//     pass 1: rows of X (R = H, L = W)      -> T_b = (X_b C_W^T)^T   (W x H per array)
//     pass 2: rows of T (R = W, L = H)      -> Y_b = (T_b C_H^T)^T = C_H X_b C_W^T
// so the second pass is again a plain row pass.  The host runs the passes over chunks of up to
// 1 GB of arrays (T is plan-owned scratch).
//
// One pass is a GEMM with M = rows (tiles of 128), N = L, K = L.  Each CTA owns one N-block of
// 64 output columns: its slice of C_L (64 x L, split into bf16 or tf32 parts, in the K-major
// 128-byte-swizzled image the UMMA B operand reads) is loaded into shared memory once (L <= 256)
// or arrives chunk by chunk with the ring (L = 512, 1024), and the CTA streams M-tiles through a
// TMA ring in K-chunks (64 FP32 per row for BF16x3, 32 for TF32x3).  Rows of 8, 16 or 32 points
// run as 64-float super-rows against a block-diagonal B (SUB).
// Split precision as in the 8x8 forms: BF16x3 = six products of 3-way splits, TF32x3 = three
// products of 2-way splits, all accumulated in FP32 in TMEM.
//
// Warp roles (512 threads):
//   warp 0 lane 0  TMA producer: ring stage s <- K-chunk of an M-tile (+ the B chunk when
//                  streamed; waits stage_free)
//   warp 1 lane 0  MMA issuer: TMEM acc set t += splits(stage s, A buffer a) . B slice; commits
//                  stage_free/a_free per chunk and acc_full after an M-tile's last chunk
//   warp 2         TMEM allocator
//   warps 4-7      split group 0 (even K-chunks), warps 8-11 split group 1 (odd K-chunks):
//                  stage s (FP32) -> hi/mid in place + lo into A buffer j % 2
//   warps 12-15    epilogue: sum of acc set t, 16 columns at a time -> transposed stores,
//                  then frees set t
// Every wait is bounded; on expiry the CTA sets *err and all roles leave their loops.
#pragma once
#include "tc_blocks8.cuh"

namespace bridct {
namespace tc {

template <int FORM> struct PassForm;
template <> struct PassForm<BF16X3> {
  static constexpr int kKC = 64;                         // FP32 row elements per K-chunk
  static constexpr int kSplits = 3;
  static constexpr int kStageBytes = kRows * kKC * 4;    // 32 KB (two 32-wide boxes)
  static constexpr int kABufBytes = kRows * kKC * 2;     // Xl (bf16)
};
template <> struct PassForm<TF32X3> {
  static constexpr int kKC = 32;
  static constexpr int kSplits = 2;
  static constexpr int kStageBytes = kRows * kKC * 4;    // 16 KB (one box)
  static constexpr int kABufBytes = kRows * kKC * 4;     // Xl (tf32)
};

constexpr int kBAtom = 64 * 128;         // one K-major SW128 atom column of 64 B rows
constexpr int kPassNBlock = 64;          // output columns per CTA (MMA N)
constexpr int kPassSmemMax = 232448;     // opt-in shared memory per block
constexpr int kPassMaxStages = 6;
constexpr int kPassThreads = 512;

constexpr int pass_min(int a, int b) { return a < b ? a : b; }

// Shared-memory plan of one row pass.  The CTA's 64-column slice of C_L stays resident when it
// fits beside a two-stage ring (L <= 256); for L = 512 and 1024 it does not (192-384 KB), and every
// ring stage then carries the slice's K-chunk next to the A chunk (STREAM_B), brought in by a bulk
// copy from the pre-split image in global memory (L2-resident: 0.4-1.5 MB per form and direction).
template <int FORM, int L>
struct PassLayout {
  using F = PassForm<FORM>;
  static constexpr int kChunks = L / F::kKC;
  static constexpr int kBlocks = L / kPassNBlock;
  static constexpr int kBBytes = F::kSplits * kChunks * kBAtom;   // this CTA's slice of C_L
  static constexpr int kBChunk = F::kSplits * kBAtom;             // one K-chunk of the slice
  static constexpr int kABufs = 2;
  static constexpr int kBarBytes = 1024;
  static constexpr bool kStreamB =
      kBBytes + kABufs * F::kABufBytes + kBarBytes + 1024 + 2 * F::kStageBytes > kPassSmemMax;
  static constexpr int kResident = kStreamB ? 0 : kBBytes;
  static constexpr int kStageStride = F::kStageBytes + (kStreamB ? kBChunk : 0);
  static constexpr int kStageTx = kStageStride;                  // bytes a stage's loads deliver
  static constexpr int kFixed = kResident + kABufs * F::kABufBytes + kBarBytes + 1024;
  static constexpr int kStages = pass_min(kPassMaxStages, (kPassSmemMax - kFixed) / kStageStride);
  static_assert(kStages >= 2, "pass ring needs two stages");
  static constexpr int kAOff = kStages * kStageStride;
  static constexpr int kBOff = kAOff + kABufs * F::kABufBytes;
  static constexpr int kBarOff = kBOff + kResident;
  static constexpr int kDynamic = kBarOff + kBarBytes + 1024;      // + 1024-byte alignment slack
  static_assert(kDynamic <= kPassSmemMax, "shared memory budget");
};

// Bulk copy of `bytes` (a multiple of 16) from global memory into shared memory, completing on bar.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

struct PassBars {
  uint32_t stage_full, stage_free, a_full, a_free, acc_full, acc_free, tmem_slot;
  __device__ explicit PassBars(uint32_t b)
      : stage_full(b), stage_free(b + 8 * kPassMaxStages), a_full(b + 16 * kPassMaxStages),
        a_free(b + 16 * kPassMaxStages + 16), acc_full(b + 16 * kPassMaxStages + 32),
        acc_free(b + 16 * kPassMaxStages + 48), tmem_slot(b + 16 * kPassMaxStages + 64) {}
};

// TF32 split of a one-box stage (128 rows x 32 FP32): Xh in place, Xl into the A buffer.
__device__ __forceinline__ void split_box_tf32(uint8_t* stage, uint8_t* abuf, uint32_t r) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t off = sw128(r, j);
    uint4 h, l;
    split_tf32x2(*reinterpret_cast<const float4*>(stage + off), h, l);
    *reinterpret_cast<uint4*>(stage + off) = h;
    *reinterpret_cast<uint4*>(abuf + off) = l;
  }
}

// Accumulator set of one M-tile (64 TMEM columns per block).  The FP32 accumulation of an MMA
// into a large accumulator loses the addends' low bits toward zero, so the dominant Xh.Ch
// product accumulates apart from the small products (whose own losses are then negligible),
// and over long K it is spread over kBig group accumulators by K-chunk, each receiving few
// MMAs.  Products sharing an A split go into one MMA with the B splits stacked along N:
//   BF16x3 blocks [big0 | small | smaller | big1]:
//     Xh.[Ch|Cm|Cl] -> [big0|small|smaller] (group 0) or Xh.Ch -> big1, Xh.[Cm|Cl] -> [small|smaller]
//     Xm.[Ch|Cm] -> [small|smaller],  Xl.Ch -> small
//   TF32x3 blocks [big0 | small | big1 | big2]:
//     Xh.[Ch|Cl] -> [big0|small] (group 0) or Xh.Ch -> big_g, Xh.Cl -> small;  Xl.Ch -> small
// The epilogue adds the blocks in FP32.
// SETS accumulator sets share the 512 TMEM columns: two (the epilogue of one M-tile overlaps the
// MMAs of the next) for rows up to 256 points, one for 512- and 1024-point rows, whose long K
// needs more group accumulators than two sets leave room for (TF32x3 round trips of 1024-point
// axes exceeded 3e-6 with three groups; one set holds seven for TF32x3, six for BF16x3).
template <int FORM, int CHUNKS, int SETS = 2>
struct PassAccs {
  static constexpr int kSmallBlocks = FORM == BF16X3 ? 2 : 1;
  static constexpr int kMaxBig = SETS == 2 ? (FORM == BF16X3 ? 2 : 3) : 512 / kPassNBlock - kSmallBlocks;
  static constexpr int kBig = CHUNKS < kMaxBig ? CHUNKS : kMaxBig;
  static constexpr int kPerTile = (1 + kSmallBlocks + (kBig - 1)) * kPassNBlock;   // columns
  static constexpr int kExtraBig = (1 + kSmallBlocks) * kPassNBlock;               // big1 column
  static constexpr int kAlloc = SETS * kPerTile <= 256 ? 256 : 512;
  static_assert(SETS * kPerTile <= 512, "TMEM columns");
  __host__ __device__ static constexpr int group(int kc) { return kc * kBig / CHUNKS; }
};

template <int L> struct PassSets { static constexpr int value = L >= 512 ? 1 : 2; };

// Split products of K-chunk kc (one thread).  bchunk: shared address of the chunk's B splits,
// laid out [split][8 KB atom column of 64 rows].  tmem: column 0 of this M-tile's set.
template <int FORM, int CHUNKS, int SETS>
__device__ __forceinline__ void issue_pass_mmas(uint32_t sstage, uint32_t sabuf, uint32_t bchunk, int kc,
                                                uint32_t tmem) {
  using A = PassAccs<FORM, CHUNKS, SETS>;
  const int g = A::group(kc);
  const bool big_first = kc == 0 || A::group(kc - 1) != g;
  const uint32_t big_g = tmem + A::kExtraBig + (uint32_t)(g - 1) * kPassNBlock;
  if constexpr (FORM == BF16X3) {
    constexpr uint32_t i192 = instr_desc(1, 192), i128 = instr_desc(1, 128), i64 = instr_desc(1, 64);
#pragma unroll
    for (int k = 0; k < 4; ++k) {   // 16 bf16 (32 bytes) per MMA
      const uint64_t bd = sw128_desc(bchunk + k * 32u);
      const uint64_t ah = sw128_desc(sstage + k * 32u);
      if (g == 0) {
        umma(tmem, ah, bd, i192, (kc | k) ? 1u : 0u, BF16X3);
      } else {
        umma(big_g, ah, bd, i64, (big_first && k == 0) ? 0u : 1u, BF16X3);
        umma(tmem + 64, ah, sw128_desc(bchunk + kBAtom + k * 32u), i128, 1u, BF16X3);
      }
      umma(tmem + 64, sw128_desc(sstage + 16384u + k * 32u), bd, i128, 1u, BF16X3);   // Xm
      umma(tmem + 64, sw128_desc(sabuf + k * 32u), bd, i64, 1u, BF16X3);              // Xl
    }
  } else {
    constexpr uint32_t i128 = instr_desc(2, 128), i64 = instr_desc(2, 64);
#pragma unroll
    for (int k = 0; k < 4; ++k) {   // 8 tf32 (32 bytes) per MMA
      const uint64_t bd = sw128_desc(bchunk + k * 32u);
      const uint64_t ah = sw128_desc(sstage + k * 32u);
      if (g == 0) {
        umma(tmem, ah, bd, i128, (kc | k) ? 1u : 0u, TF32X3);
      } else {
        umma(big_g, ah, bd, i64, (big_first && k == 0) ? 0u : 1u, TF32X3);
        umma(tmem + 64, ah, sw128_desc(bchunk + kBAtom + k * 32u), i64, 1u, TF32X3);
      }
      umma(tmem + 64, sw128_desc(sabuf + k * 32u), bd, i64, 1u, TF32X3);   // Xl
    }
  }
}

// xmap: the (nrows x L) FP32 row matrix (box 32 x 128, SWIZZLE_128B).  out: destination of
// the transposed arrays (R rows per array, rshift = log2 R).  bimage: kBlocks slices of
// PassLayout::kBBytes.  Grid: a multiple of kBlocks CTAs; CTA c computes N-block c % kBlocks.
// SUB > 1 (rows of LS = 64 / SUB = 8, 16 or 32 points): L = 64 and every matrix row holds SUB
// consecutive rows of length LS (a super-row); B is block-diagonal (SUB copies of C_LS), so
// column n = j * LS + c of super-row g is output column c of row g * SUB + j, and nrows counts
// super-rows.
template <int FORM, int L, int SUB = 1>
__global__ void __launch_bounds__(kPassThreads, 1)
    k_tcpass(const __grid_constant__ CUtensorMap xmap, float* __restrict__ out,
             const uint4* __restrict__ bimage, long long nrows, int rshift, int* __restrict__ err) {
  static_assert(SUB == 1 || L == 64, "super-rows are 64 floats");
  constexpr int LS = L / SUB;   // points per original row
  using PL = PassLayout<FORM, L>;
  using F = PassForm<FORM>;
  constexpr int kStages = PL::kStages;
  constexpr int kChunks = PL::kChunks;
  constexpr int kSets = PassSets<L>::value;
  using ACC = PassAccs<FORM, kChunks, kSets>;
  constexpr uint32_t kTileCols = ACC::kPerTile;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(base);
  const PassBars bars(sbase + PL::kBarOff);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + PL::kBarOff + 16 * kPassMaxStages + 64);
  __shared__ volatile int s_abort;
  __shared__ volatile int s_group_ok[3];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int nblk = blockIdx.x % PL::kBlocks;
  const long long slot = blockIdx.x / PL::kBlocks;
  const long long nslots = gridDim.x / PL::kBlocks;
  const long long mtiles = (nrows + kRows - 1) / kRows;
  const long long ntile_local = slot < mtiles ? (mtiles - 1 - slot) / nslots + 1 : 0;
  const long long nchunk_local = ntile_local * kChunks;

  if (tid == 0) {
    s_abort = 0;
    for (int i = 0; i < kStages; ++i) {
      mbar_init(bars.stage_full + 8 * i, 1);
      mbar_init(bars.stage_free + 8 * i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(bars.a_full + 8 * i, 1);
      mbar_init(bars.a_free + 8 * i, 1);
      mbar_init(bars.acc_full + 8 * i, 1);
      mbar_init(bars.acc_free + 8 * i, 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ACC::kAlloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if constexpr (!PL::kStreamB) {
    const uint4* src = bimage + (size_t)nblk * (PL::kBBytes / 16);
    uint4* dst = reinterpret_cast<uint4*>(base + PL::kBOff);
    for (int i = tid; i < PL::kBBytes / 16; i += kPassThreads) dst[i] = __ldg(src + i);
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
    for (long long j = 0; j < nchunk_local && ok && !s_abort; ++j) {
      const int s = (int)(j % kStages);
      ok = mbar_wait(bars.stage_free + 8 * s, ((uint32_t)(j / kStages) & 1u) ^ 1u);
      if (!ok) break;
      const long long m = slot + (j / kChunks) * nslots;
      const int kc = (int)(j % kChunks);
      const uint32_t dst = sbase + s * PL::kStageStride;
      mbar_expect_tx(bars.stage_full + 8 * s, PL::kStageTx);
      tma_load_2d(dst, &xmap, kc * F::kKC, (int)(m * kRows), bars.stage_full + 8 * s);
      if constexpr (F::kKC == 64)
        tma_load_2d(dst + 16384u, &xmap, kc * F::kKC + 32, (int)(m * kRows), bars.stage_full + 8 * s);
      if constexpr (PL::kStreamB)
        bulk_load(dst + F::kStageBytes,
                  reinterpret_cast<const uint8_t*>(bimage) + (size_t)nblk * PL::kBBytes + (size_t)kc * PL::kBChunk,
                  PL::kBChunk, bars.stage_full + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    for (long long j = 0; j < nchunk_local && ok && !s_abort; ++j) {
      const int s = (int)(j % kStages), a = (int)(j & 1);
      const long long jt = j / kChunks;
      const int kc = (int)(j % kChunks), t = (int)(jt % kSets);
      ok = mbar_wait(bars.a_full + 8 * a, (uint32_t)(j >> 1) & 1u);
      if (ok && kc == 0) ok = mbar_wait(bars.acc_free + 8 * t, ((uint32_t)(jt / kSets) & 1u) ^ 1u);
      if (!ok) break;
      tc_fence_after();
      const uint32_t sstage = sbase + s * PL::kStageStride;
      const uint32_t bchunk = PL::kStreamB ? sstage + F::kStageBytes
                                           : sbase + PL::kBOff + (uint32_t)(kc * F::kSplits) * kBAtom;
      issue_pass_mmas<FORM, kChunks, kSets>(sstage, sbase + PL::kAOff + a * F::kABufBytes, bchunk, kc,
                                     tmem_base + t * kTileCols);
      umma_commit(bars.stage_free + 8 * s);
      umma_commit(bars.a_free + 8 * a);
      if (kc == kChunks - 1) umma_commit(bars.acc_full + 8 * t);
    }
    if (ok && nchunk_local > 0) {   // the last MMAs must finish before TMEM is freed
      const long long j = nchunk_local - 1;
      ok = mbar_wait(bars.a_free + 8 * (int)(j & 1), (uint32_t)(j >> 1) & 1u);
    }
  } else if (warp >= 4 && warp < 12) {
    const int grp = (warp - 4) >> 2;              // 0: even K-chunks, 1: odd K-chunks
    const uint32_t r = tid - 128 - 128 * grp;
    const int bar_id = grp ? 3 : 1, ok_slot = grp ? 2 : 0;
    for (long long j = grp; j < nchunk_local; j += 2) {
      const int s = (int)(j % kStages), a = (int)(j & 1);
      if (r == 0) {
        bool g = !s_abort && mbar_wait(bars.stage_full + 8 * s, (uint32_t)(j / kStages) & 1u);
        if (g) g = mbar_wait(bars.a_free + 8 * a, ((uint32_t)(j >> 1) & 1u) ^ 1u);
        s_group_ok[ok_slot] = g ? 1 : 0;
      }
      named_sync(bar_id, 128);
      if (!s_group_ok[ok_slot]) {
        ok = r != 0;
        break;
      }
      uint8_t* stage = base + s * PL::kStageStride;
      uint8_t* abuf = base + PL::kAOff + a * F::kABufBytes;
      if constexpr (FORM == BF16X3) split_tile<BF16X3>(stage, abuf, r);
      else split_box_tf32(stage, abuf, r);
      fence_async_smem();
      named_sync(bar_id, 128);
      if (r == 0) mbar_arrive(bars.a_full + 8 * a);
    }
  } else if (warp >= 12) {
    const uint32_t r = tid - 384;                 // tile row = TMEM lane
    const uint32_t quarter = (uint32_t)(warp & 3) * 32u;
    const long long rmask = (1ll << rshift) - 1;
    for (long long jt = 0; jt < ntile_local; ++jt) {
      const int t = (int)(jt % kSets);
      if (r == 0)
        s_group_ok[1] = (!s_abort && mbar_wait(bars.acc_full + 8 * t, (uint32_t)(jt / kSets) & 1u)) ? 1 : 0;
      named_sync(2, 128);
      if (!s_group_ok[1]) {
        ok = r != 0;
        break;
      }
      tc_fence_after();
      // row g = (array b, row h of that array); its column n goes to out[b][n][h].  With
      // super-rows, column n = j * LS + c of super-row g goes to out[b][c][h0 + j], h0 = g * SUB
      // within its array (SUB divides R, so a super-row lies in one array).
      const long long g = (slot + jt * nslots) * kRows + r;
      const bool live = g < nrows;
      const long long g0 = g * SUB;
      const long long b = g0 >> rshift, h = g0 & rmask;
      float* dst = out + ((b * LS + (long long)nblk * kPassNBlock) << rshift) + h;
      const uint32_t taddr = tmem_base + t * kTileCols + (quarter << 16);
#pragma unroll
      for (int q = 0; q < kPassNBlock / 16; ++q) {
        float big[16], sm[16], w[16];
        tmem_ld16(taddr + q * 16, big);
        tmem_ld16(taddr + kPassNBlock + q * 16, sm);
        tmem_wait_ld();
#pragma unroll
        for (int a = 0; a < ACC::kSmallBlocks - 1; ++a) {
          tmem_ld16(taddr + (2 + a) * kPassNBlock + q * 16, w);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) sm[i] += w[i];
        }
#pragma unroll
        for (int a = 1; a < ACC::kBig; ++a) {
          tmem_ld16(taddr + ACC::kExtraBig + (a - 1) * kPassNBlock + q * 16, w);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) big[i] += w[i];
        }
        if (live) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            constexpr int kLS = LS;
            const int n = q * 16 + i, j = n / kLS, c = n % kLS;
            dst[((long long)c << rshift) + j] = big[i] + sm[i];
          }
        }
      }
      tc_fence_before();
      named_sync(2, 128);
      if (r == 0) mbar_arrive(bars.acc_free + 8 * t);
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(ACC::kAlloc));
  }
}

}  // namespace tc
}  // namespace bridct
