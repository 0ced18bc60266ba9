// Host-buffer paths of the C-ABI: the chunked H2D / kernel / D2H pipeline behind
// bridct_plan_apply_batch, and the per-thread plan cache behind bridct_apply.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>

#include "../../include/bridct.h"
#include "../../include/bridct_b200.h"
#include "bridct_internal.h"

namespace bridct {

static constexpr size_t kChunkBytes = 16u << 20;   // per slot and direction

static int ensure_batch_staging(bridct_plan* p, bool need_pinned) {
  const size_t per = p->elements * sizeof(float);
  if (!p->d_batch) {
    size_t c = kChunkBytes / per;
    p->chunk = c ? c : 1;
    cudaError_t e = cudaMalloc((void**)&p->d_batch, 4 * p->chunk * per);
    if (e != cudaSuccess) return cuda_fail(e, "batch staging");
    for (int i = 0; i < 2; ++i) {
      e = cudaStreamCreateWithFlags(&p->aux[i], cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "batch streams");
    }
  }
  if (need_pinned && !p->pin_batch) {
    cudaError_t e = cudaHostAlloc((void**)&p->pin_batch, 4 * p->chunk * per, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "pinned batch staging");
  }
  return BRIDCT_OK;
}

// Chunks of the batch alternate between two slots, each with its own stream, so that the
// copy engines (H2D, D2H) and the SMs work on different chunks at the same time.
int host_batch_pipeline(bridct_plan* p, int mode, const float* in, float* out, size_t batch,
                        const float* dx, float* dy, bool pin_in, bool pin_out) {
  const bool stage_in = !dx && !pin_in, stage_out = !dy && !pin_out;
  int s = ensure_batch_staging(p, stage_in || stage_out);
  if (s) return s;
  const size_t per = p->elements;              // floats per array
  const size_t cf = p->chunk * per;            // floats per chunk
  const size_t cbytes = cf * sizeof(float);
  const bool dx_ok = dx && (uintptr_t)dx % 16 == 0, dy_ok = dy && (uintptr_t)dy % 16 == 0;
  size_t pending_off[2] = {0, 0}, pending_n[2] = {0, 0};
  bool pending[2] = {false, false};
  cudaError_t e = cudaSuccess;
  size_t ci = 0;
  for (size_t a0 = 0; a0 < batch; a0 += p->chunk, ++ci) {
    const int slot = (int)(ci & 1);
    cudaStream_t st = p->aux[slot];
    const size_t na = batch - a0 < p->chunk ? batch - a0 : p->chunk;
    const size_t off = a0 * per, nbytes = na * per * sizeof(float);
    float* sx = p->d_batch + (size_t)slot * 2 * cf;
    float* sy = sx + cf;
    float* px = p->pin_batch ? p->pin_batch + (size_t)slot * 2 * cf : nullptr;
    float* py = px ? px + cf : nullptr;
    if (pending[slot]) {        // slot reuse: finish the chunk that used it before
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
      if (stage_out) memcpy(out + pending_off[slot], py, pending_n[slot]);
      pending[slot] = false;
    }
    const float* kx;
    if (dx_ok) {
      kx = dx + off;
    } else {
      if (dx) {
        e = cudaMemcpyAsync(sx, dx + off, nbytes, cudaMemcpyDeviceToDevice, st);
      } else if (pin_in) {
        e = cudaMemcpyAsync(sx, in + off, nbytes, cudaMemcpyHostToDevice, st);
      } else {
        memcpy(px, in + off, nbytes);
        e = cudaMemcpyAsync(sx, px, nbytes, cudaMemcpyHostToDevice, st);
      }
      if (e != cudaSuccess) return cuda_fail(e, "batch H2D");
      kx = sx;
    }
    float* ky = dy_ok ? dy + off : sy;
    s = launch_plain_form(p, mode, kx, ky, (long long)na, st);
    if (s) return s;
    if (!dy_ok) {
      if (dy) {
        e = cudaMemcpyAsync(dy + off, sy, nbytes, cudaMemcpyDeviceToDevice, st);
      } else if (pin_out) {
        e = cudaMemcpyAsync(out + off, sy, nbytes, cudaMemcpyDeviceToHost, st);
      } else {
        e = cudaMemcpyAsync(py, sy, nbytes, cudaMemcpyDeviceToHost, st);
        pending_off[slot] = off;
        pending_n[slot] = nbytes;
      }
      if (e != cudaSuccess) return cuda_fail(e, "batch D2H");
    }
    pending[slot] = true;
    (void)cbytes;
  }
  for (int slot = 0; slot < 2; ++slot) {
    if (!pending[slot]) continue;
    e = cudaStreamSynchronize(p->aux[slot]);
    if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
    if (stage_out) {
      float* py = p->pin_batch + (size_t)slot * 2 * cf + cf;
      memcpy(out + pending_off[slot], py, pending_n[slot]);
    }
  }
  return BRIDCT_OK;
}

// bridct_apply (caller-workspace square API) has no plan argument; the device staging it
// needs comes from one cached plan per (thread, device, size).  The plans live until the
// process exits.
bridct_plan* thread_square_plan(int n) {
  static thread_local std::map<std::pair<int, int>, bridct_plan*> cache;
  int dev = 0;
  if (current_device(&dev) != BRIDCT_OK) return nullptr;
  auto key = std::make_pair(dev, n);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  bridct_plan* p = bridct_plan_create(n, n);
  if (p) cache[key] = p;
  return p;
}

void release_plan_extras(bridct_plan* p) {
  if (p->tc_mem) cudaFree(p->tc_mem);
  p->tc_mem = nullptr;
}

}  // namespace bridct
