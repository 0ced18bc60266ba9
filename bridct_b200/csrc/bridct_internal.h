// Internal types shared by the host-side translation units of libbridct_b200.so.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "plain_launch.cuh"

namespace bridct {

// One per CUDA device, created on first use and immutable afterwards.
struct DeviceCtx {
  int device = 0;
  int sm_count = 0;
  int major = 0, minor = 0;
  long long l2_bytes = 0;
  LaunchCtx launch{};
  PlainLauncher plain[8][8][3] = {};
  UnitLauncher col_units[8][3] = {};    // merged column passes, by lg(column length) and mode
  UnitLauncher row_units[8][3] = {};    // merged row passes, by lg(row length) and mode
  FourStepTables fourstep[4] = {};      // N = 128, 256, 512, 1024
  std::vector<void*> table_mem;
  FourStepTables tables(int n) const;
};

void set_error(const std::string& s);
int cuda_fail(cudaError_t e, const char* what);
double sj_scale(int n, int k);
// Four-step tables of line length N (twiddles, post-rotation coefficients), float64-derived.
void build_fourstep_tables(int N, std::vector<float2>& tw, std::vector<float4>& post);
void fill_fourstep_tables(int N, float2* tw, float4* post);
DeviceCtx* device_ctx(int device);
// Opts `kernel` into `smem` bytes of dynamic shared memory on the current device and returns
// its resident blocks per SM at `threads` threads (0 on failure); cached per device, since the
// attribute belongs to the device's copy of the kernel.
int kernel_setup(const void* kernel, int smem, int threads);
int current_device(int* dev);
const void* device_address(const void* p, bool* pinned);

// Makes `device` current for the guard's scope and gives the caller's current device back at
// scope exit, so an entry point never leaves another device current than the one it found.
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int device) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) {
      cudaGetLastError();
      cur = -1;
    }
    if (cur != device) {
      status = cudaSetDevice(device);
      prev = cur;
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace bridct

struct bridct_plan {
  int h = 0, w = 0;
  size_t elements = 0;
  int square = 0;
  int device = 0;
  bridct::DeviceCtx* dev = nullptr;
  cudaStream_t stream = nullptr;
  float* d_x = nullptr;        // one-array device staging
  float* d_y = nullptr;
  float* pin = nullptr;        // one-array pinned staging (in, out)
  // batch pipeline (allocated on the first host-pointer batch call): copy-in, kernel and
  // copy-out streams, and per slot the events that order a slot's reuse on the GPU
  static constexpr int kPipeSlots = 4;
  cudaStream_t aux[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t pipe_ev[3][kPipeSlots] = {};   // [copied in, transformed, copied out][slot]
  float* d_batch = nullptr;    // slots x (in, out) x chunk
  float* pin_batch = nullptr;  // slots x (in, out) x chunk, pageable callers only
  void* copyout = nullptr;     // per slot, the state of a pageable output's copy out (host_pipeline.cu)
  size_t chunk = 0;            // arrays per pipeline chunk
  // precision-form scratch (allocated on first use of a tensor-core form that is not given a
  // caller workspace); tc_mu serializes its (re)allocation
  void* tc_mem = nullptr;
  size_t tc_bytes = 0;
  std::mutex tc_mu;
};

namespace bridct {
// Pipeline-only mode: forward then inverse with the float32 spectrum materialized on the device
// (bitwise the composition of a FORWARD and an INVERSE call).
constexpr int kModeSpectrumRT = 3;
int launch_plain_form(const bridct_plan* p, int mode, const float* x, float* y, long long batch,
                      cudaStream_t st);
// Plain form over `batch` h x w arrays on device d in general layouts (lx, ly NULL: contiguous).
int launch_plain_layout(DeviceCtx* d, int h, int w, int mode, const float* x, float* y, long long batch,
                        const BatchLayout* lx, const BatchLayout* ly, cudaStream_t st);
int host_batch_pipeline(bridct_plan* p, int mode, const float* in, float* out, size_t batch,
                        const float* dx, float* dy, bool pin_in, bool pin_out);
bridct_plan* thread_square_plan(int n);
// memcpy split over the library's host copy threads (pageable <-> pinned staging).
void host_copy(void* dst, const void* src, size_t n);
void release_plan_extras(bridct_plan* p);
}  // namespace bridct

namespace bridct {
// Tensor-core precision forms (tc_forms.cu).
// workspace: caller-owned scratch of ws_bytes (NULL: the plan's own scratch).
int apply_tc_form(bridct_plan* p, int mode, int form, const float* x, float* y, size_t batch,
                  void* stream, void* workspace, size_t ws_bytes);
// Scratch bytes a tensor-core form needs for `batch` arrays of the plan's shape (0: none).
size_t tc_workspace_bytes(const bridct_plan* p, int form, size_t batch);
}  // namespace bridct
