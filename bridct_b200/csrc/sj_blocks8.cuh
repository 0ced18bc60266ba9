// 8x8 arrays (the block-transform batch): one thread owns one whole 8x8 array in registers
// and runs 8 row lines and 8 column lines of the generated SJ 8-point program; the CTA
// stages its tile of 256 arrays through shared memory so that global loads and stores are
// fully coalesced 16-byte accesses.
//
// Shared-memory layout: array b occupies 256 bytes = sixteen 16-byte chunks; chunk j of array
// b is stored at chunk position (j ^ (b & 15)).  A thread reading chunk j of its own array and
// seven neighbours reading chunk j of theirs (one 8-thread phase of a 128-bit access) then hit
// eight distinct 16-byte bank groups, so every shared-memory access is conflict free; the
// coalesced tile copy (consecutive threads, consecutive chunks of one array) is conflict free
// for the same reason.
#pragma once
#include "sj_lines.cuh"

namespace bridct {

constexpr int kB8Threads = 256;            // arrays per tile = threads per CTA
constexpr int kB8Chunks = kB8Threads * 16; // 16-byte chunks per tile

__device__ __forceinline__ int b8_slot(int chunk) {
  const int b = chunk >> 4, j = chunk & 15;
  return (b << 4) | (j ^ (b & 15));
}

template <int MODE>
__device__ __forceinline__ void b8_transform(float (&v)[64]) {
  // columns, then rows (the reference's vertical-then-bands order, src/generated/rect.c:5-15)
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    float t[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) t[r] = v[r * 8 + c];
    reg_line_apply<8, MODE>(t);
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r * 8 + c] = t[r];
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    float t[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) t[c] = v[r * 8 + c];
    reg_line_apply<8, MODE>(t);
#pragma unroll
    for (int c = 0; c < 8; ++c) v[r * 8 + c] = t[c];
  }
}

// x, y: `batch` contiguous 8x8 arrays (16-byte aligned).
template <int MODE>
__global__ void __launch_bounds__(kB8Threads) k_blocks8(const float* __restrict__ x,
                                                        float* __restrict__ y, long long batch) {
  extern __shared__ float4 s8[];
  // Full rounds: tile r*grid + blockIdx of 256 arrays (all CTAs stream one contiguous region
  // together).  The arrays left after the full rounds are split evenly over all CTAs (fewer
  // than 256 each), so the launch has no tail round in which a fraction of the SMs works alone.
  const long long round_arrays = (long long)gridDim.x * kB8Threads;
  const long long full = batch / round_arrays;
  const long long rest = batch - full * round_arrays;
  const long long per = rest / gridDim.x, extra = rest % gridDim.x;
  const int t = threadIdx.x;
  griddep_wait();
  for (long long round = 0; round <= full; ++round) {
    if (round == full) griddep_trigger();
    long long first;
    int arrays;
    if (round < full) {
      first = round * round_arrays + (long long)blockIdx.x * kB8Threads;
      arrays = kB8Threads;
    } else {
      first = full * round_arrays + blockIdx.x * per + (blockIdx.x < extra ? blockIdx.x : extra);
      arrays = (int)(per + (blockIdx.x < extra ? 1 : 0));
      if (arrays == 0) break;
    }
    const int chunks = arrays * 16;
    const float4* src = reinterpret_cast<const float4*>(x) + first * 16;
    float4 buf[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int q = t + k * kB8Threads;
      buf[k] = q < chunks ? __ldg(src + q) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) s8[b8_slot(t + k * kB8Threads)] = buf[k];
    __syncthreads();
    float v[64];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const float4 c = s8[b8_slot(t * 16 + j)];
      v[4 * j] = c.x; v[4 * j + 1] = c.y; v[4 * j + 2] = c.z; v[4 * j + 3] = c.w;
    }
    b8_transform<MODE>(v);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      s8[b8_slot(t * 16 + j)] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    __syncthreads();
    float4* dst = reinterpret_cast<float4*>(y) + first * 16;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int q = t + k * kB8Threads;
      if (q < chunks) dst[q] = s8[b8_slot(q)];
    }
    __syncthreads();
  }
}

// Double-buffered variant: 128-array tiles (32 KB) in two shared-memory buffers filled with
// cp.async, so each CTA has its next tile in flight while it transforms the current one (three
// CTAs per SM).  Same work split: full rounds tile-strided, the last partial round spread over
// all CTAs.
constexpr int kB8dbThreads = 128;                  // arrays per tile = threads per CTA
constexpr int kB8dbChunks = kB8dbThreads * 16;     // 16-byte chunks per tile

__device__ __forceinline__ void b8_cp_async16(float4* dst, const float4* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(kB8dbThreads) k_blocks8_db(const float* __restrict__ x, float* __restrict__ y,
                                                             long long batch) {
  extern __shared__ float4 s8[];
  const long long round_arrays = (long long)gridDim.x * kB8dbThreads;
  const long long full = batch / round_arrays;
  const long long rest = batch - full * round_arrays;
  const long long per = rest / gridDim.x, extra = rest % gridDim.x;
  const long long nrounds = full + ((per + (blockIdx.x < extra ? 1 : 0)) > 0 ? 1 : 0);
  const int t = threadIdx.x;
  auto range = [&](long long round, long long& first, int& arrays) {
    if (round < full) {
      first = round * round_arrays + (long long)blockIdx.x * kB8dbThreads;
      arrays = kB8dbThreads;
    } else {
      first = full * round_arrays + blockIdx.x * per + (blockIdx.x < extra ? blockIdx.x : extra);
      arrays = (int)(per + (blockIdx.x < extra ? 1 : 0));
    }
  };
  auto issue = [&](long long round) {
    long long first;
    int arrays;
    range(round, first, arrays);
    float4* buf = s8 + (round & 1) * kB8dbChunks;
    const float4* src = reinterpret_cast<const float4*>(x) + first * 16;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int q = t + k * kB8dbThreads;
      if (q < arrays * 16) b8_cp_async16(buf + b8_slot(q), src + q);
    }
  };
  griddep_wait();
  if (nrounds > 0) issue(0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  if (nrounds <= 1) griddep_trigger();
  for (long long round = 0; round < nrounds; ++round) {
    if (round + 1 == nrounds - 1) griddep_trigger();   // the last round's loads are being issued
    if (round + 1 < nrounds) issue(round + 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");   // this round's copies have landed
    __syncthreads();
    long long first;
    int arrays;
    range(round, first, arrays);
    float4* buf = s8 + (round & 1) * kB8dbChunks;
    if (t < arrays) {
      float v[64];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float4 c = buf[b8_slot(t * 16 + j)];
        v[4 * j] = c.x; v[4 * j + 1] = c.y; v[4 * j + 2] = c.z; v[4 * j + 3] = c.w;
      }
      b8_transform<MODE>(v);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        buf[b8_slot(t * 16 + j)] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
    __syncthreads();
    float4* dst = reinterpret_cast<float4*>(y) + first * 16;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int q = t + k * kB8dbThreads;
      if (q < arrays * 16) dst[q] = buf[b8_slot(q)];
    }
    __syncthreads();   // the buffer is refilled by the next round's issue
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

}  // namespace bridct
