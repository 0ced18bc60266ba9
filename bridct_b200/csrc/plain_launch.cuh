// Host-side launch logic of the plain form for one compile-time shape (H, W) and mode.
#pragma once
#include <cuda_runtime.h>
#include "sj_kernels.cuh"
#include "sj_blocks8.cuh"

namespace bridct {

// Tile-class batches of at most this many floats (16 MiB) take the small-batch tiles where
// small_batch_tiles says so.
constexpr long long kSmallBatchFloats = 4LL << 20;

// Shapes and modes whose 16 MiB batches measured faster with tiles of half the 8192-float target
// (several CTAs per SM instead of one uneven wave of large tiles; 24 shapes A/B'd on one box):
// 8x16 +17%, 16x16 +16%, 32x16 +9..12%, 16x64 +8..14%, 32x32 +8..10%, 16x32 +6..10%, 8x32 +4..10%,
// 16x8 +5%, 64x8 +4..7%, and the inverse and round trip of 32x64 (+10..13%) and the round trip of
// 8x64 (+9%).  Tiles of 64-point register lines (64x16, 64x32, 64x64: one thread per line, so a
// 4096-float tile leaves most threads idle) and of 128-point lines measured 5..25% slower.  64x64
// round trips instead take two arrays per 128-thread CTA (a thread for each register line): +11%;
// forward equal, inverse 5% slower that way.
__host__ __device__ constexpr bool small_batch_tiles(int h, int w, int mode) {
  return (h == 8 && (w == 16 || w == 32)) || (h == 16 && w <= 64) || (h == 32 && (w == 16 || w == 32)) ||
         (h == 64 && w == 8) || (h == 32 && w == 64 && mode != LM_FWD) || (h == 8 && w == 64 && mode == LM_RT) ||
         (h == 64 && w == 64 && mode == LM_RT);
}

struct LaunchCtx {
  int sm_count;
};

// lx, ly: general layouts of x and y (both NULL: a contiguous batch).
using PlainLauncher = cudaError_t (*)(const float*, float*, long long, cudaStream_t,
                                      LineTables, const LaunchCtx&, const BatchLayout*, const BatchLayout*);

int kernel_setup(const void* kernel, int smem, int threads);   // bridct_api.cu

// Blocks per SM for a kernel at a given dynamic shared-memory size (set up once per device).
template <typename Kernel>
static int kernel_blocks_per_sm(Kernel k, int smem, int threads = kThreads) {
  return kernel_setup(reinterpret_cast<const void*>(k), smem, threads);
}

// Launches a plain-form kernel with programmatic stream serialization (see griddep_wait): its
// CTAs may be scheduled, and run up to their first global access, while the previous kernel in
// the stream finishes, which hides most of the launch gap between back-to-back launches (the two
// passes of a two-pass shape, or consecutive calls).
// With pdl = false it is an ordinary launch (the kernels' griddepcontrol instructions are then
// no-ops).  Measured on 128 MiB batches of every shape (two A/B runs on one box): +1..5% on every
// single-kernel shape, but 6..10% slower on most two-pass shapes with full-grid passes (the passes
// of the few-array geometry keep it: one 1024 x 1024 array 529 -> 577 GB/s).
template <typename... Params, typename... Args>
static cudaError_t launch_pdl(void (*k)(Params...), unsigned grid, unsigned threads, int smem, cudaStream_t st,
                              bool pdl, Args... args) {
  if (!pdl) {
    k<<<grid, threads, smem, st>>>(args...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

template <typename Kernel>
static cudaError_t launch_tiles(Kernel k, int smem, int bps, TileArgs a, const LaunchCtx& ctx,
                                cudaStream_t st, int threads = kThreads, bool pdl = true) {
  if (bps <= 0) return cudaErrorInvalidConfiguration;
  if (a.ntiles <= 0) return cudaSuccess;
  long long grid = (long long)ctx.sm_count * bps;
  if (grid > a.ntiles) grid = a.ntiles;
  return launch_pdl(k, (unsigned)grid, (unsigned)threads, smem, st, pdl, a);
}

// Route of an (H, W, MODE) batch: whole 32768-float arrays as single tiles in the modes where that
// measured faster than two passes; other shapes above 16384 floats take the two passes.
__host__ __device__ constexpr bool whole_array_route(int H, int W, int MODE) {
  return H * W == 32768 && (MODE == LM_INV || H == 1024 || H == 64 || (H == 32 && MODE == LM_FWD));
}
__host__ __device__ constexpr bool two_pass_route(int H, int W, int MODE) {
  return H * W > 16384 && !whole_array_route(H, W, MODE);
}

// GEN: the batch has general layouts (strided arrays or an offset table, BatchLayout); the same
// geometry choices run the GEN instantiations of the kernels, except that 8x8 arrays take the
// generic tile kernel instead of the dedicated one-thread-per-array kernels.
template <int H, int W, int MODE, bool GEN>
cudaError_t launch_plain_impl(const float* x, float* y, long long batch, cudaStream_t st,
                              LineTables tab, const LaunchCtx& ctx, const BatchLayout& lx,
                              const BatchLayout& ly) {
  using Gm = Geometry<H, W>;
  if (batch <= 0) return cudaSuccess;
  if constexpr (H == 8 && W == 8 && !GEN) {
    // Measured on B200 (GB/s, device-resident, back-to-back launches): the double-buffered kernel
    // wins forward/inverse batches up to a few hundred thousand arrays (262,144: 5131 vs 4937)
    // and round trips from about 200,000 (524,288: 5655 vs 5130); the single-buffer kernel
    // wins larger forward batches (1,048,576: 5930 vs 5355) and small round trips.
    const bool db = MODE == LM_RT ? batch >= 196608 : batch <= 393216;
    if (db) {
      auto k = k_blocks8_db<MODE>;
      constexpr int smem = 2 * kB8dbChunks * 16;
      const int bps = kernel_blocks_per_sm(k, smem, kB8dbThreads);
      if (bps <= 0) return cudaErrorInvalidConfiguration;
      const long long ntiles = (batch + kB8dbThreads - 1) / kB8dbThreads;
      long long grid = (long long)ctx.sm_count * bps;
      if (grid > ntiles) grid = ntiles;
      return launch_pdl(k, (unsigned)grid, kB8dbThreads, smem, st, true, x, y, batch);
    }
    auto k = k_blocks8<MODE>;
    constexpr int smem = kB8Chunks * 16;
    const int bps = kernel_blocks_per_sm(k, smem, kB8Threads);
    if (bps <= 0) return cudaErrorInvalidConfiguration;
    const long long ntiles = (batch + kB8Threads - 1) / kB8Threads;
    long long grid = (long long)ctx.sm_count * bps;
    if (grid > ntiles) grid = ntiles;
    return launch_pdl(k, (unsigned)grid, kB8Threads, smem, st, true, x, y, batch);
  } else if constexpr (Gm::kTile) {
    // 16384-float tiles instead of 8192 where they measured faster on 128 MiB batches: 64-wide
    // arrays up to 64 high (+6..14%, except the 64 x 64 inverse, -2%) and forward/inverse of
    // 8..32 x 128 (+17..22%); narrower tiles, 64 x 128 and those round trips measured 5..21%
    // slower with them (64 x 8 and 64 x 16, whose 8192-float tiles give half the threads a column
    // line, 5-8% slower too).
    constexpr bool kBig = (W == 64 && H <= 64 && !(H == 64 && MODE == LM_INV)) ||
                          (W == 128 && H <= 32 && MODE != LM_RT);
    // Forward / inverse tiles of 128-point register columns and 8..32 columns hold one CTA per SM
    // (227+ registers), so their tiles are sized against one CTA's shared memory (kTRWide): twice
    // the arrays, so that 128 instead of 64 threads have a column line (+18..26%); round trips
    // (128-thread CTAs, two per SM) measured 18-20% slower that way, and so did 32768-float tiles
    // of 8..32 x 128 (all rows busy, but no register prefetch at that size): -20%.
    constexpr bool kWide = H == 128 && W <= 32 && MODE != LM_RT;
    constexpr int TR = kWide ? Gm::kTRWide : kBig ? Gm::kTRBig : Gm::kTR;
    // 128 x 128 tiles (both passes 128-point register lines, 255 registers) and round trips of
    // tiles with a 128-point axis run 128-thread CTAs: two CTAs share an SM (128 x 128 +31..64%
    // over one 256-thread CTA with register prefetch, in which half the warps have no line; the
    // round trips +3..30% together with their register lines).  Forward / inverse tiles that mix
    // 128-point register lines with many short lines measured 5..13% slower that way.
    constexpr int T = (H == 128 && W == 128) || (MODE == LM_RT && (H == 128 || W == 128)) ? 128 : kThreads;
    // Shared memory as the kernel uses it (no exchange buffer for register lines), except the
    // 128 x 128 round trip, which measured 2-3% faster at two CTAs per SM than at three.
    constexpr int smem = H == 128 && W == 128 && MODE == LM_RT ? Gm::kSmemFull : Gm::template tile_smem<MODE, T>(TR / H);
    if constexpr (Gm::kTRSmall < TR && small_batch_tiles(H, W, MODE)) {
      if (batch * H * W <= kSmallBatchFloats) {
        constexpr bool k64 = H == 64 && W == 64;   // two arrays, 128 threads (see small_batch_tiles)
        constexpr int TS = k64 ? 128 : T;
        constexpr int TRS = k64 ? Gm::kTR : Gm::kTRSmall;
        constexpr int SMS = Gm::template tile_smem<MODE, TS>(TRS / H);
        auto ks = k_full<H, W, TRS, true, true, MODE, TS, GEN>;
        TileArgs a{x, y, (batch * H + TRS - 1) / TRS, batch * H, tab, lx, ly};
        return launch_tiles(ks, SMS, kernel_blocks_per_sm(ks, SMS, TS), a, ctx, st, TS);
      }
    }
    auto k = k_full<H, W, TR, true, true, MODE, T, GEN>;
    const int bps = kernel_blocks_per_sm(k, smem, T);
    TileArgs a{x, y, (batch * H + TR - 1) / TR, batch * H, tab, lx, ly};
    return launch_tiles(k, smem, bps, a, ctx, st, T);
  } else if constexpr (whole_array_route(H, W, MODE)) {
    // Whole 32768-float arrays as tiles (one CTA per SM, both passes in shared memory) instead of
    // the two passes, where that measured faster: every inverse (+5..21%), forward of 1024 x 32,
    // 32 x 1024 and 64 x 512 (+2..14%), round trips of 1024 x 32 and 64 x 512 (+2..6%); round
    // trips of 128 x 256 and 256 x 128 measured 30% slower.
    auto k = k_full<H, W, H, true, true, MODE, kThreads, GEN>;
    const int bps = kernel_blocks_per_sm(k, Gm::kSmemWhole);
    TileArgs a{x, y, batch, batch * H, tab, lx, ly};
    return launch_tiles(k, Gm::kSmemWhole, bps, a, ctx, st);
  } else {
    // Round trips of 128-point register lines run 128-thread CTAs without register prefetch:
    // every warp has a line and two CTAs share an SM, which measured +8..13% over one 256-thread
    // CTA with prefetch; forward and inverse measured 5..9% slower that way and keep 256 threads.
    constexpr int TC_T = H == 128 && MODE == LM_RT ? 128 : kThreads;
    constexpr int TR_T = W == 128 && MODE == LM_RT ? 128 : kThreads;
    constexpr int kSmemC = Gm::template strip_smem_used<MODE, TC_T>(Gm::kTC);
    constexpr int kSmemCs = Gm::template strip_smem_used<MODE, TC_T>(Gm::kTCs);
    constexpr int kSmemR = Gm::template rows_smem_used<MODE, TR_T>(Gm::kRB);
    constexpr int kSmemRs = Gm::template rows_smem_used<MODE, TR_T>(Gm::kRBs);
    auto kc = k_colstrip<H, W, Gm::kTC, MODE, TC_T, GEN>;
    auto kr = k_full<H, W, Gm::kRB, false, true, MODE, TR_T, GEN>;
    const int bpc = kernel_blocks_per_sm(kc, kSmemC, TC_T);
    const int bpr = kernel_blocks_per_sm(kr, kSmemR, TR_T);
    // One column-strip launch and one row-block launch over the whole batch.  Cutting the batch
    // into L2-sized chunks (so that the intermediate stays in L2 between the two passes) measured
    // slower on every two-pass shape: the four-step kernels are bound by shared-memory latency,
    // not by HBM, while every chunk adds two launch tails (128 MiB batches +16..48% unchunked,
    // 2048 x 256^2 1669 -> 2129 GB/s).
    const long long nb = batch;
    cudaError_t e;
    const bool few = nb * (W / Gm::kTC) < 2LL * ctx.sm_count;   // passes below a full grid: PDL
    const bool small = few || (GEN && lx.small_units);
    if (small) {   // few arrays (or asked for): smaller strips and row blocks
      auto kcs = k_colstrip<H, W, Gm::kTCs, MODE, TC_T, GEN>;
      TileArgs ac{x, y, nb * (W / Gm::kTCs), nb * H, tab, lx, ly};
      e = launch_tiles(kcs, kSmemCs, kernel_blocks_per_sm(kcs, kSmemCs, TC_T), ac, ctx, st, TC_T,
                       few);
    } else {
      TileArgs ac{x, y, nb * (W / Gm::kTC), nb * H, tab, lx, ly};
      e = launch_tiles(kc, kSmemC, bpc, ac, ctx, st, TC_T, false);
    }
    if (e != cudaSuccess) return e;
    if constexpr (Gm::kNarrowRows) {
      auto krn = k_full<H, W, Gm::kRBn, false, true, MODE, 128, GEN>;
      TileArgs ar{y, y, nb * H / Gm::kRBn, nb * H, tab, ly, ly};
      e = launch_tiles(krn, Gm::kSmemRowsN, kernel_blocks_per_sm(krn, Gm::kSmemRowsN, 128), ar, ctx, st, 128, few);
    } else if (nb * H / Gm::kRB < 2LL * ctx.sm_count || (GEN && lx.small_units)) {
      auto krs = k_full<H, W, Gm::kRBs, false, true, MODE, TR_T, GEN>;
      TileArgs ar{y, y, nb * H / Gm::kRBs, nb * H, tab, ly, ly};
      e = launch_tiles(krs, kSmemRs, kernel_blocks_per_sm(krs, kSmemRs, TR_T), ar, ctx, st, TR_T,
                       few);
    } else {
      TileArgs ar{y, y, nb * H / Gm::kRB, nb * H, tab, ly, ly};
      e = launch_tiles(kr, kSmemR, bpr, ar, ctx, st, TR_T, false);
    }
    if (e != cudaSuccess) return e;
    return cudaSuccess;
  }
}

template <int H, int W, int MODE>
cudaError_t launch_plain(const float* x, float* y, long long batch, cudaStream_t st, LineTables tab,
                         const LaunchCtx& ctx, const BatchLayout* lx, const BatchLayout* ly) {
  if (lx && ly) return launch_plain_impl<H, W, MODE, true>(x, y, batch, st, tab, ctx, *lx, *ly);
  return launch_plain_impl<H, W, MODE, false>(x, y, batch, st, tab, ctx, BatchLayout{}, BatchLayout{});
}

// Merged passes of a ragged batch (UNITS kernels): one launch over the column strips of arrays of
// column length H and any width (launch_col_units), or over the row blocks of arrays of row length
// W and any height (launch_row_units), with the geometry the two-pass route uses for them (the
// strip width depends only on H and the row-block height only on W for two-pass shapes; the
// templates take 1024 for the other axis).  `units` lists the strips (or blocks), n of them.
using UnitLauncher = cudaError_t (*)(const float*, float*, const PassUnit*, long long, cudaStream_t,
                                     LineTables, const LaunchCtx&);

template <int H, int MODE>
cudaError_t launch_col_units(const float* x, float* y, const PassUnit* units, long long n, cudaStream_t st,
                             LineTables tab, const LaunchCtx& ctx) {
  using Gm = Geometry<H, 1024>;
  constexpr int TC_T = H == 128 && MODE == LM_RT ? 128 : kThreads;
  auto k = k_colstrip<H, 1024, Gm::kTC, MODE, TC_T, false, true>;
  TileArgs a{x, y, n, n * H, tab, BatchLayout{}, BatchLayout{}, units};
  return launch_tiles(k, Gm::kSmemStrip, kernel_blocks_per_sm(k, Gm::kSmemStrip, TC_T), a, ctx, st, TC_T, false);
}

template <int W, int MODE>
cudaError_t launch_row_units(const float* x, float* y, const PassUnit* units, long long n, cudaStream_t st,
                             LineTables tab, const LaunchCtx& ctx) {
  using Gm = Geometry<1024, W>;
  if constexpr (Gm::kNarrowRows) {
    auto k = k_full<1024, W, Gm::kRBn, false, true, MODE, 128, false, true>;
    TileArgs a{x, y, n, n * Gm::kRBn, tab, BatchLayout{}, BatchLayout{}, units};
    return launch_tiles(k, Gm::kSmemRowsN, kernel_blocks_per_sm(k, Gm::kSmemRowsN, 128), a, ctx, st, 128, false);
  } else {
    constexpr int TR_T = W == 128 && MODE == LM_RT ? 128 : kThreads;
    auto k = k_full<1024, W, Gm::kRB, false, true, MODE, TR_T, false, true>;
    TileArgs a{x, y, n, n * Gm::kRB, tab, BatchLayout{}, BatchLayout{}, units};
    return launch_tiles(k, Gm::kSmemRows, kernel_blocks_per_sm(k, Gm::kSmemRows, TR_T), a, ctx, st, TR_T, false);
  }
}

// Strip width of two-pass arrays of column length h, and row-block height of row length w.
int merged_strip_cols(int h);
int merged_block_rows(int w);

// Per-H instantiation units (plain_inst.cu compiled once per H) export this table row.
void plain_table_row(int h, PlainLauncher (*row)[3]);

}  // namespace bridct
