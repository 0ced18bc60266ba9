// Host-buffer paths of the C-ABI: the chunked H2D / kernel / D2H pipeline behind
// bridct_plan_apply_batch, and the per-thread plan cache behind bridct_apply.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/bridct.h"
#include "../../include/bridct_b200.h"
#include "bridct_internal.h"

namespace bridct {

// Host copies between pageable caller memory and the pinned staging, split over a small pool of
// host threads: one thread's memcpy into pinned memory runs near 10 GB/s, far below the PCIe rate
// the staging feeds.  The pool starts on first use (and again in a forked child, whose copy of
// the parent's pool has no threads); every call waits for its own pieces only.
class CopyPool {
 public:
  static CopyPool& get() {
    static std::mutex mu;
    static CopyPool* pool = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pool || pool->pid_ != getpid()) pool = new CopyPool();   // a forked child's copy is left alone
    return *pool;
  }

  // A copy that runs entirely on the pool threads, started later (submit, e.g. from a CUDA host
  // callback once the source has arrived) and waited for with wait().
  struct Deferred {
    std::mutex mu;
    std::condition_variable cv;
    size_t left = 0;
    char* d = nullptr;
    const char* s = nullptr;
    size_t n = 0, step = 0, parts = 0;
  };

  void prepare(Deferred& c, void* dst, const void* src, size_t n) {
    c.d = static_cast<char*>(dst);
    c.s = static_cast<const char*>(src);
    c.n = n;
    c.parts = std::min<size_t>(threads_.size(), std::max<size_t>(1, n / kPiece));
    c.step = (n / c.parts + 63) & ~size_t(63);
    std::lock_guard<std::mutex> lock(c.mu);
    c.left = c.parts;
  }

  // Queues the pieces of a prepared copy (no CUDA calls: safe inside a CUDA host callback).
  void submit(Deferred& c) {
    size_t skipped = 0;
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (size_t i = 0; i < c.parts; ++i) {
        const size_t off = i * c.step;
        if (off >= c.n) {
          ++skipped;
          continue;
        }
        jobs_.push_back(Job{c.d + off, c.s + off, std::min(c.step, c.n - off), nullptr, &c});
      }
    }
    cv_.notify_all();
    if (skipped) {
      std::lock_guard<std::mutex> lock(c.mu);
      c.left -= skipped;
      if (c.left == 0) c.cv.notify_all();
    }
  }

  static void wait(Deferred& c) {
    std::unique_lock<std::mutex> lock(c.mu);
    c.cv.wait(lock, [&] { return c.left == 0; });
  }

  void copy(void* dst, const void* src, size_t n) {
    const size_t parts = std::min<size_t>(threads_.size() + 1, std::max<size_t>(1, n / kPiece));
    if (parts <= 1) {
      memcpy(dst, src, n);
      return;
    }
    Call call;
    call.left = parts - 1;
    const size_t step = (n / parts + 63) & ~size_t(63);
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (size_t i = 1; i < parts; ++i) {
        const size_t off = i * step;
        if (off >= n) {
          --call.left;
          continue;
        }
        jobs_.push_back(Job{static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                            std::min(step, n - off), &call, nullptr});
      }
    }
    cv_.notify_all();
    memcpy(dst, src, std::min(step, n));
    std::unique_lock<std::mutex> lock(call.mu);
    call.cv.wait(lock, [&] { return call.left == 0; });
  }

 private:
  // Pieces of at least 256 KB: an 8 MB slot is split over every thread (one thread's memcpy into
  // pinned memory measured 16.6 GB/s on a B200 host, twelve threads together 67 GB/s).
  static constexpr size_t kPiece = 256u << 10;
  struct Call {
    std::mutex mu;
    std::condition_variable cv;
    size_t left = 0;
  };
  struct Job {
    char* d;
    const char* s;
    size_t n;
    Call* call;          // a synchronous copy's state, or
    Deferred* deferred;  // a deferred copy's
  };

  CopyPool() : pid_(getpid()) {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned n = std::max(1u, std::min(hw ? hw : 4u, 12u)) - 1;
    for (unsigned i = 0; i < n; ++i) threads_.emplace_back([this] { work(); });
    for (auto& t : threads_) t.detach();
  }

  void work() {
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return !jobs_.empty(); });
        j = jobs_.front();
        jobs_.pop_front();
      }
      memcpy(j.d, j.s, j.n);
      if (j.call) {
        std::lock_guard<std::mutex> lock(j.call->mu);
        if (--j.call->left == 0) j.call->cv.notify_all();
      } else {
        std::lock_guard<std::mutex> lock(j.deferred->mu);
        if (--j.deferred->left == 0) j.deferred->cv.notify_all();
      }
    }
  }

  pid_t pid_;
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Job> jobs_;
};

void host_copy(void* dst, const void* src, size_t n) { CopyPool::get().copy(dst, src, n); }

// CUDA host callback: the copy-out's device-to-host copy has finished, start its pool copy.
static void CUDART_CB start_copy_out(void* p) { CopyPool::get().submit(*static_cast<CopyPool::Deferred*>(p)); }

static constexpr size_t kChunkBytes = 8u << 20;      // staging per slot and direction
static constexpr size_t kMinChunkBytes = 4u << 20;   // smallest chunk a call cuts
static constexpr int kSlots = bridct_plan::kPipeSlots;

static int ensure_batch_staging(bridct_plan* p, bool need_pinned) {
  const size_t per = p->elements * sizeof(float);
  if (!p->d_batch) {
    size_t c = kChunkBytes / per;
    p->chunk = c ? c : 1;
    // per slot: input, output and (materialized round trips) the float32 spectrum
    cudaError_t e = cudaMalloc((void**)&p->d_batch, 3 * kSlots * p->chunk * per);
    if (e != cudaSuccess) return cuda_fail(e, "batch staging");
    for (int i = 0; i < 3; ++i) {
      e = cudaStreamCreateWithFlags(&p->aux[i], cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "batch streams");
      for (int k = 0; k < kSlots; ++k) {
        e = cudaEventCreateWithFlags(&p->pipe_ev[i][k], cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "batch events");
      }
    }
  }
  if (need_pinned && !p->pin_batch) {
    cudaError_t e = cudaHostAlloc((void**)&p->pin_batch, 2 * kSlots * p->chunk * per, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "pinned batch staging");
  }
  if (need_pinned && !p->copyout) p->copyout = new CopyPool::Deferred[2 * kSlots];   // copies out, copies in
  return BRIDCT_OK;
}

// Chunks of the batch rotate through kSlots staging slots.  Copies in run on one stream, the
// transforms on a second and copies out on a third, so both copy engines and the SMs work on
// different chunks at once; a slot's reuse is ordered on the GPU by its events (the next copy
// in waits for the transform that read the slot, the next transform for the copy out that read
// it).  The host waits only where it copies through its own pinned staging (pageable callers)
// and at the end.
int host_batch_pipeline(bridct_plan* p, int mode, const float* in, float* out, size_t batch,
                        const float* dx, float* dy, bool pin_in, bool pin_out) {
  const bool stage_in = !dx && !pin_in, stage_out = !dy && !pin_out;
  int s = ensure_batch_staging(p, stage_in || stage_out);
  if (s) return s;
  const size_t per = p->elements;              // floats per array
  const size_t cf = p->chunk * per;            // floats per staging slot
  // About four chunks per call, each between kMinChunkBytes and the slot size (PCIe copies below a
  // few MB lose efficiency, and every chunk adds its copies, events and launch to the chain).
  // Measured on one box against eight chunks with a 1/4, 1/2 size ramp at both ends (three
  // alternating runs of over 1000 calls): 16.8 MB calls 3% faster, 4.2 and 67 MB calls equal.
  size_t chunk = (batch + 3) / 4;
  const size_t min_chunk = kMinChunkBytes / (per * sizeof(float));
  if (chunk < min_chunk) chunk = min_chunk;
  if (chunk > p->chunk) chunk = p->chunk;
  if (chunk < 1) chunk = 1;
  const bool dx_ok = dx && (uintptr_t)dx % 16 == 0, dy_ok = dy && (uintptr_t)dy % 16 == 0;
  cudaStream_t hs = p->aux[0], ks = p->aux[1], ds = p->aux[2];
  cudaEvent_t* ev_in = p->pipe_ev[0];
  cudaEvent_t* ev_k = p->pipe_ev[1];
  cudaEvent_t* ev_out = p->pipe_ev[2];
  // A pageable output's copy out of a slot's pinned staging starts on the pool threads as soon as
  // the slot's device-to-host copy has finished (a host callback on the copy-out stream), so copies
  // out overlap the host's copies in; a slot is reused only after its copy out has completed.  The
  // copies' state belongs to the plan, so a callback never outlives it; every exit from this
  // function waits for the copies it started.
  // A pageable input's copy into a slot's pinned staging runs on the pool threads one chunk ahead:
  // chunk k+1's copy is queued before the host waits for chunk k's, so the pool never idles
  // between chunks.
  CopyPool::Deferred* outcopy = static_cast<CopyPool::Deferred*>(p->copyout);
  CopyPool::Deferred* incopy = outcopy ? outcopy + kSlots : nullptr;
  bool used[kSlots] = {}, pending[kSlots] = {}, loading[kSlots] = {};
  struct Drain {
    cudaStream_t ds;
    CopyPool::Deferred* outcopy;
    CopyPool::Deferred* incopy;
    bool* pending;
    bool* loading;
    ~Drain() {
      for (int i = 0; i < kSlots; ++i)
        if (loading[i]) CopyPool::wait(incopy[i]);
      bool any = false;
      for (int i = 0; i < kSlots; ++i) any = any || pending[i];
      if (!any || cudaStreamSynchronize(ds) != cudaSuccess) return;
      for (int i = 0; i < kSlots; ++i)
        if (pending[i]) CopyPool::wait(outcopy[i]);
    }
  } drain{p->aux[2], outcopy, incopy, pending, loading};
  cudaError_t e = cudaSuccess;
  size_t ci = 0;
  std::vector<size_t> sizes;
  for (size_t a = 0; a < batch; a += chunk) sizes.push_back(batch - a < chunk ? batch - a : chunk);
  // queues chunk k's copy into its slot's pinned staging (after the slot's previous copy in has
  // read it out)
  auto queue_copy_in = [&](size_t k) -> cudaError_t {
    const int sl = (int)(k % kSlots);
    if (k >= (size_t)kSlots) {
      const cudaError_t ee = cudaEventSynchronize(ev_in[sl]);
      if (ee != cudaSuccess) return ee;
    }
    const size_t first = k * chunk;
    CopyPool::get().prepare(incopy[sl], p->pin_batch + (size_t)sl * 2 * cf, in + first * per,
                            sizes[k] * per * sizeof(float));
    CopyPool::get().submit(incopy[sl]);
    loading[sl] = true;
    return cudaSuccess;
  };
  if (stage_in && !sizes.empty()) {
    e = queue_copy_in(0);
    if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
  }
  size_t a0 = 0;
  for (size_t na : sizes) {
    const int slot = (int)(ci % kSlots);
    const size_t off = a0 * per, nbytes = na * per * sizeof(float);
    float* sx = p->d_batch + (size_t)slot * 3 * cf;
    float* sy = sx + cf;
    float* sz = sy + cf;
    float* px = p->pin_batch ? p->pin_batch + (size_t)slot * 2 * cf : nullptr;
    float* py = px ? px + cf : nullptr;
    if (pending[slot]) {        // the slot's previous output has left its pinned staging
      CopyPool::wait(outcopy[slot]);
      pending[slot] = false;
    }
    const float* kx;
    if (dx_ok) {
      kx = dx + off;
    } else {
      if (used[slot]) {
        e = cudaStreamWaitEvent(hs, ev_k[slot], 0);   // the slot's last transform has read sx
        if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
      }
      if (dx) {
        e = cudaMemcpyAsync(sx, dx + off, nbytes, cudaMemcpyDeviceToDevice, hs);
      } else if (pin_in) {
        e = cudaMemcpyAsync(sx, in + off, nbytes, cudaMemcpyHostToDevice, hs);
      } else {
        if (ci + 1 < sizes.size()) {   // the next chunk's copy in goes to the pool now
          e = queue_copy_in(ci + 1);
          if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
        }
        CopyPool::wait(incopy[slot]);
        loading[slot] = false;
        e = cudaMemcpyAsync(sx, px, nbytes, cudaMemcpyHostToDevice, hs);
      }
      if (e == cudaSuccess) e = cudaEventRecord(ev_in[slot], hs);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ks, ev_in[slot], 0);
      if (e != cudaSuccess) return cuda_fail(e, "batch H2D");
      kx = sx;
    }
    float* ky = dy_ok ? dy + off : sy;
    if (!dy_ok && used[slot]) {
      e = cudaStreamWaitEvent(ks, ev_out[slot], 0);     // the slot's last copy out has read sy
      if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
    }
    if (mode == kModeSpectrumRT) {   // forward into the slot's spectrum, inverse out of it
      s = launch_plain_form(p, BRIDCT_FORWARD, kx, sz, (long long)na, ks);
      if (!s) s = launch_plain_form(p, BRIDCT_INVERSE, sz, ky, (long long)na, ks);
    } else {
      s = launch_plain_form(p, mode, kx, ky, (long long)na, ks);
    }
    if (s) return s;
    e = cudaEventRecord(ev_k[slot], ks);
    if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
    if (!dy_ok) {
      e = cudaStreamWaitEvent(ds, ev_k[slot], 0);
      if (e == cudaSuccess) {
        if (dy) {
          e = cudaMemcpyAsync(dy + off, sy, nbytes, cudaMemcpyDeviceToDevice, ds);
        } else if (pin_out) {
          e = cudaMemcpyAsync(out + off, sy, nbytes, cudaMemcpyDeviceToHost, ds);
        } else {
          e = cudaMemcpyAsync(py, sy, nbytes, cudaMemcpyDeviceToHost, ds);
          if (e == cudaSuccess) {
            CopyPool::get().prepare(outcopy[slot], out + off, py, nbytes);
            e = cudaLaunchHostFunc(ds, start_copy_out, &outcopy[slot]);
            pending[slot] = e == cudaSuccess;
          }
        }
      }
      if (e == cudaSuccess) e = cudaEventRecord(ev_out[slot], ds);
      if (e != cudaSuccess) return cuda_fail(e, "batch D2H");
    }
    used[slot] = true;
    a0 += na;
    ++ci;
  }
  // Every copy in is ordered before the transform that reads it and every transform before its
  // copy out, so the last copy out (or, for a device output, the last transform) ends the call.
  e = cudaStreamSynchronize(dy_ok ? ks : ds);
  if (e != cudaSuccess) return cuda_fail(e, "batch pipeline");
  for (int slot = 0; slot < kSlots; ++slot)   // the callbacks have run: wait for their copies
    if (pending[slot]) {
      CopyPool::wait(outcopy[slot]);
      pending[slot] = false;
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
  delete[] static_cast<CopyPool::Deferred*>(p->copyout);
  p->copyout = nullptr;
  if (p->tc_mem) cudaFree(p->tc_mem);
  p->tc_mem = nullptr;
  for (auto& row : p->pipe_ev)
    for (cudaEvent_t& ev : row)
      if (ev) {
        cudaEventDestroy(ev);
        ev = nullptr;
      }
}

}  // namespace bridct
