// C-ABI of libbridct_b200.so: the reference plan API (include/bridct.h) on B200.
//
// Reference behaviour kept (src/plan.c:33-163, src/bridct.c:13-75, docs/API.md):
//   * bridct_supported / plan_create reject anything but powers of two in [8, 1024];
//   * plan_apply validates NULL/mode, then overlap, and writes nothing on error;
//   * bridct_apply validates invalid -> workspace too small -> 16-byte workspace
//     alignment -> pairwise overlap, in that order;
//   * a plan is not reentrant (one plan per concurrent caller), it owns its scratch and
//     apply performs no allocation;
//   * route strings "paper8-square" / "blocked-extension".
// GPU specifics: every device gets one immutable context (SM count, four-step tables,
// launcher table) created on first use; each plan owns a CUDA stream plus device and
// pinned staging for host-pointer calls.
#include <cuda_runtime.h>
#include <tuple>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bridct.h"
#include "../../include/bridct_b200.h"
#include "plain_launch.cuh"
#include "bridct_internal.h"

namespace bridct {

static thread_local std::string g_last_error;

void set_error(const std::string& s) { g_last_error = s; }

int cuda_fail(cudaError_t e, const char* what) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  set_error(buf);
  return BRIDCT_DEVICE_ERROR;
}

static int lg2(int n) {
  int k = 0;
  while ((8 << k) < n) ++k;
  return k;
}

double sj_scale(int n, int k) {
  if (n <= 4) return 1.0;
  k %= n / 4;
  const double angle = 2 * M_PI * k / n;
  return sj_scale(n / 4, k) * (k <= n / 8 ? std::cos(angle) : std::sin(angle));
}

// Four-step tables for N = 32 G (see sj_lines.cuh): twiddles w_N^{bc} s(32,c) and the
// post-rotation coefficients with the stage-2 SJ scale of each column and the orthonormal
// factor folded in.  Stage 2 of column c produces V(d) / scale(c, d) with
//   scale = s(G, d)          columns 1..15 when G < 32 (SJ scaled complex FFT),
//           s(16, d >> 1)    columns 1..15 when G = 32 (split into two radix-2 halves),
//           1                columns 0 and 16 (cooperative shuffle DFT across the lanes).
// Fills caller-provided arrays of G*17 float2 (tw[b*17+c]) and G*17 float4 (post at
// post_index(G, d, c)).
void fill_fourstep_tables(int N, float2* tw, float4* post) {
  const int G = N / 32;
  for (int b = 0; b < G; ++b)
    for (int c = 0; c < 17; ++c) {
      const double ang = -2 * M_PI * (double)b * c / N;
      const double s = sj_scale(32, c);
      tw[(size_t)b * 17 + c] = float2{(float)(std::cos(ang) * s), (float)(std::sin(ang) * s)};
    }
  auto sig = [N](int k) { return std::sqrt((k == 0 ? 1.0 : 2.0) / N); };
  for (int c = 0; c < 17; ++c)
    for (int d = 0; d < G; ++d) {
      const int k = c + 32 * d;
      const double th = M_PI * k / (2.0 * N);
      const double sg = (c == 0 || c == 16) ? 1.0 : G == 32 ? sj_scale(16, d >> 1) : sj_scale(G, d);
      float4 p;
      p.x = (float)(sig(k) * sg * std::cos(th));
      p.y = (float)(sig(k) * sg * std::sin(th));
      p.z = k ? (float)(sig(N - k) * sg * std::sin(th)) : 0.f;
      p.w = k ? (float)(-sig(N - k) * sg * std::cos(th)) : 0.f;
      post[post_index(G, d, c)] = p;
    }
}

void build_fourstep_tables(int N, std::vector<float2>& tw, std::vector<float4>& post) {
  const int G = N / 32;
  tw.assign((size_t)G * 17, float2{0, 0});
  post.assign((size_t)17 * G, float4{0, 0, 0, 0});
  fill_fourstep_tables(N, tw.data(), post.data());
}

#define BRIDCT_DECL_H(H)                                                            \
  void plain_table_h##H(PlainLauncher (*row)[3], UnitLauncher* col, UnitLauncher* rowu); \
  int merged_strip_cols_h##H();                                                      \
  int merged_block_rows_w##H();
BRIDCT_DECL_H(8)
BRIDCT_DECL_H(16)
BRIDCT_DECL_H(32)
BRIDCT_DECL_H(64)
BRIDCT_DECL_H(128)
BRIDCT_DECL_H(256)
BRIDCT_DECL_H(512)
BRIDCT_DECL_H(1024)
#undef BRIDCT_DECL_H

int merged_strip_cols(int h) {
  switch (h) {
    case 32: return merged_strip_cols_h32();
    case 64: return merged_strip_cols_h64();
    case 128: return merged_strip_cols_h128();
    case 256: return merged_strip_cols_h256();
    case 512: return merged_strip_cols_h512();
    case 1024: return merged_strip_cols_h1024();
    default: return 0;
  }
}

int merged_block_rows(int w) {
  switch (w) {
    case 32: return merged_block_rows_w32();
    case 64: return merged_block_rows_w64();
    case 128: return merged_block_rows_w128();
    case 256: return merged_block_rows_w256();
    case 512: return merged_block_rows_w512();
    case 1024: return merged_block_rows_w1024();
    default: return 0;
  }
}

static std::mutex g_dev_mutex;
static std::map<int, std::unique_ptr<DeviceCtx>> g_devices;

DeviceCtx* device_ctx(int device) {
  std::lock_guard<std::mutex> lock(g_dev_mutex);
  auto it = g_devices.find(device);
  if (it != g_devices.end()) return it->second.get();
  std::unique_ptr<DeviceCtx> d(new DeviceCtx());
  d->device = device;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    cuda_fail(e, "cudaGetDeviceProperties");
    return nullptr;
  }
  d->sm_count = prop.multiProcessorCount;
  d->major = prop.major;
  d->minor = prop.minor;
  d->l2_bytes = prop.l2CacheSize;
  d->launch.sm_count = prop.multiProcessorCount;
  // Two-pass chunk: a quarter of L2 keeps the column pass's output resident for the row pass.
  PlainLauncher (*tab)[8][3] = d->plain;
  plain_table_h8(tab[0], d->col_units[0], d->row_units[0]);
  plain_table_h16(tab[1], d->col_units[1], d->row_units[1]);
  plain_table_h32(tab[2], d->col_units[2], d->row_units[2]);
  plain_table_h64(tab[3], d->col_units[3], d->row_units[3]);
  plain_table_h128(tab[4], d->col_units[4], d->row_units[4]);
  plain_table_h256(tab[5], d->col_units[5], d->row_units[5]);
  plain_table_h512(tab[6], d->col_units[6], d->row_units[6]);
  plain_table_h1024(tab[7], d->col_units[7], d->row_units[7]);
  for (int i = 0; i < 4; ++i) {
    const int N = 128 << i;
    std::vector<float2> tw;
    std::vector<float4> post;
    build_fourstep_tables(N, tw, post);
    const size_t btw = tw.size() * sizeof(float2), bpo = post.size() * sizeof(float4);
    void* mem = nullptr;
    e = cudaMalloc(&mem, btw + bpo);
    if (e != cudaSuccess) {
      cuda_fail(e, "cudaMalloc(tables)");
      return nullptr;
    }
    d->table_mem.push_back(mem);
    cudaMemcpy(mem, tw.data(), btw, cudaMemcpyHostToDevice);
    e = cudaMemcpy((char*)mem + btw, post.data(), bpo, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cuda_fail(e, "cudaMemcpy(tables)");
      return nullptr;
    }
    d->fourstep[i].tw = (const float2*)mem;
    d->fourstep[i].post = (const float4*)((char*)mem + btw);
  }
  DeviceCtx* raw = d.get();
  g_devices[device] = std::move(d);
  return raw;
}

FourStepTables DeviceCtx::tables(int n) const {
  if (n < 128) return FourStepTables{nullptr, nullptr};
  return fourstep[lg2(n) - 4];
}

int current_device(int* dev) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    set_error(e != cudaSuccess ? std::string("no CUDA device: ") + cudaGetErrorString(e)
                               : std::string("no CUDA device"));
    cudaGetLastError();
    return BRIDCT_DEVICE_ERROR;
  }
  e = cudaGetDevice(dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  return BRIDCT_OK;
}

// Pointer classification: returns the device-usable address or nullptr for host memory.
const void* device_address(const void* p, bool* pinned) {
  cudaPointerAttributes a;
  *pinned = false;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return a.devicePointer;
  if (a.type == cudaMemoryTypeHost) *pinned = true;
  return nullptr;
}

int launch_plain_form(const bridct_plan* p, int mode, const float* x, float* y, long long batch,
                      cudaStream_t st) {
  return launch_plain_layout(p->dev, p->h, p->w, mode, x, y, batch, nullptr, nullptr, st);
}

int launch_plain_layout(DeviceCtx* d, int h, int w, int mode, const float* x, float* y, long long batch,
                        const BatchLayout* lx, const BatchLayout* ly, cudaStream_t st) {
  LineTables tab{d->tables(h), d->tables(w)};
  PlainLauncher fn = d->plain[lg2(h)][lg2(w)][mode];
  cudaError_t e = fn(x, y, batch, st, tab, d->launch, lx, ly);
  if (e != cudaSuccess) return cuda_fail(e, "plain kernel launch");
  return BRIDCT_OK;
}

static bool ranges_overlap(uintptr_t a, size_t na, uintptr_t b, size_t nb) {
  return a <= b ? b - a < na : a - b < nb;
}

}  // namespace bridct

using namespace bridct;

namespace bridct {

int kernel_setup(const void* kernel, int smem, int threads) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, int, int>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  const auto key = std::make_tuple(kernel, dev, smem, threads);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int blocks = 0;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem) != cudaSuccess) return 0;
  cache[key] = blocks;
  return blocks;
}

}  // namespace bridct

extern "C" {

BRIDCT_API int bridct_supported(int height, int width) {
  return height >= 8 && height <= 1024 && width >= 8 && width <= 1024 && !(height & (height - 1)) &&
         !(width & (width - 1));
}

BRIDCT_API void bridct_plan_destroy(bridct_plan* plan) {
  if (!plan) return;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  cudaSetDevice(plan->device);
  if (plan->stream) cudaStreamSynchronize(plan->stream);
  for (int i = 0; i < 3; ++i)
    if (plan->aux[i]) {
      cudaStreamSynchronize(plan->aux[i]);
      cudaStreamDestroy(plan->aux[i]);
    }
  cudaFree(plan->d_x);
  cudaFree(plan->d_y);
  cudaFree(plan->d_batch);
  cudaFreeHost(plan->pin);
  cudaFreeHost(plan->pin_batch);
  if (plan->stream) cudaStreamDestroy(plan->stream);
  release_plan_extras(plan);
  if (prev >= 0) cudaSetDevice(prev);
  delete plan;
}

BRIDCT_API bridct_plan* bridct_plan_create(int height, int width) {
  if (!bridct_supported(height, width)) {
    set_error("unsupported shape: both axes must be powers of two from 8 to 1024");
    return nullptr;
  }
  int dev = 0;
  if (current_device(&dev) != BRIDCT_OK) return nullptr;
  DeviceCtx* d = device_ctx(dev);
  if (!d) return nullptr;
  bridct_plan* p = new bridct_plan();
  p->h = height;
  p->w = width;
  p->elements = (size_t)height * width;
  p->device = dev;
  p->dev = d;
  p->square = height == width && height <= 256;
  const size_t bytes = p->elements * sizeof(float);
  cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->d_x, bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->d_y, bytes);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&p->pin, 2 * bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cuda_fail(e, "bridct_plan_create");
    bridct_plan_destroy(p);
    return nullptr;
  }
  return p;
}

BRIDCT_API const char* bridct_plan_route(const bridct_plan* plan) {
  return !plan ? nullptr : plan->square ? "paper8-square" : "blocked-extension";
}

BRIDCT_API const char* bridct_plan_gpu_route(const bridct_plan* plan) {
  if (!plan) return nullptr;
  return plan->elements <= 16384 ? "sj-tile" : "sj-two-pass";
}

BRIDCT_API const char* bridct_last_error(void) { return g_last_error.c_str(); }

BRIDCT_API int bridct_plan_apply(bridct_plan* plan, enum bridct_mode mode, const float* input,
                                 float* output) {
  if (!plan || !input || !output || (unsigned)mode > BRIDCT_ROUNDTRIP) return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = plan->elements * sizeof(float);
  if (ranges_overlap((uintptr_t)input, bytes, (uintptr_t)output, bytes)) return BRIDCT_OVERLAPPING_BUFFERS;
  DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(plan device)");
  bool pin_in = false, pin_out = false;
  const float* dx = (const float*)device_address(input, &pin_in);
  float* dy = (float*)device_address(output, &pin_out);
  cudaStream_t st = plan->stream;
  cudaError_t e = cudaSuccess;
  // Device pointers need only float alignment (docs/API.md:17); the kernels use 16-byte
  // vector accesses, so an unaligned device buffer goes through the plan's staging.
  if (dx && (uintptr_t)dx % 16) {
    e = cudaMemcpyAsync(plan->d_x, dx, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "D2D");
    dx = plan->d_x;
  }
  const bool dy_unaligned = dy && (uintptr_t)dy % 16;
  const float* kx = dx;
  if (!kx) {
    if (pin_in) {
      e = cudaMemcpyAsync(plan->d_x, input, bytes, cudaMemcpyHostToDevice, st);
    } else {
      host_copy(plan->pin, input, bytes);
      e = cudaMemcpyAsync(plan->d_x, plan->pin, bytes, cudaMemcpyHostToDevice, st);
    }
    if (e != cudaSuccess) return cuda_fail(e, "H2D");
    kx = plan->d_x;
  }
  float* ky = dy && !dy_unaligned ? dy : plan->d_y;
  int s = launch_plain_form(plan, mode, kx, ky, 1, st);
  if (s) return s;
  if (dy_unaligned) {
    e = cudaMemcpyAsync(dy, plan->d_y, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "D2D");
  } else if (!dy) {
    if (pin_out) {
      e = cudaMemcpyAsync(output, plan->d_y, bytes, cudaMemcpyDeviceToHost, st);
    } else {
      e = cudaMemcpyAsync(plan->pin + plan->elements, plan->d_y, bytes, cudaMemcpyDeviceToHost, st);
    }
    if (e != cudaSuccess) return cuda_fail(e, "D2H");
  }
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "bridct_plan_apply");
  if (!dy && !pin_out) host_copy(output, plan->pin + plan->elements, bytes);
  return BRIDCT_OK;
}

BRIDCT_API int bridct_plan_apply_device(bridct_plan* plan, enum bridct_mode mode, const float* input,
                                        float* output, size_t batch, void* stream) {
  if (!plan || !input || !output || (unsigned)mode > BRIDCT_ROUNDTRIP || batch == 0)
    return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = plan->elements * sizeof(float) * batch;
  if (ranges_overlap((uintptr_t)input, bytes, (uintptr_t)output, bytes)) return BRIDCT_OVERLAPPING_BUFFERS;
  if (((uintptr_t)input | (uintptr_t)output) % 16) return BRIDCT_BAD_ALIGNMENT;
  // The launch runs on the plan's device (its tables live there) whatever device is current.
  DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(plan device)");
  // NULL is the CUDA default stream, as everywhere in CUDA (torch's default stream too).
  return launch_plain_form(plan, mode, input, output, (long long)batch, (cudaStream_t)stream);
}

// Floats from the first element of a strided batch to one past its last.
static size_t strided_extent(size_t h, size_t w, size_t ld, size_t bs, size_t batch) {
  return (batch - 1) * bs + (h - 1) * ld + w;
}

// A strided layout writes every element once: arrays apart (bs covers a whole array), or arrays
// side by side within every row band (bs covers a row, ld covers the batch's row).
static bool strided_disjoint(size_t h, size_t w, size_t ld, size_t bs, size_t batch) {
  if (ld < w) return false;
  if (batch == 1 || bs >= (h - 1) * ld + w) return true;
  return bs >= w && ld >= (batch - 1) * bs + w;
}

BRIDCT_API int bridct_plan_apply_strided_device(bridct_plan* plan, enum bridct_mode mode, const float* input,
                                                size_t input_row_pitch, size_t input_array_stride, float* output,
                                                size_t output_row_pitch, size_t output_array_stride, size_t batch,
                                                void* stream) {
  if (!plan || !input || !output || (unsigned)mode > BRIDCT_ROUNDTRIP || batch == 0) return BRIDCT_INVALID_ARGUMENT;
  const size_t h = plan->h, w = plan->w;
  if (!strided_disjoint(h, w, input_row_pitch, input_array_stride, batch) ||
      !strided_disjoint(h, w, output_row_pitch, output_array_stride, batch)) {
    set_error("bridct_plan_apply_strided_device: row pitch below the width, or arrays that overlap");
    return BRIDCT_INVALID_ARGUMENT;
  }
  if ((input_row_pitch | output_row_pitch | (batch > 1 ? input_array_stride | output_array_stride : 0)) % 4 ||
      ((uintptr_t)input | (uintptr_t)output) % 16) {
    set_error("bridct_plan_apply_strided_device: pitches and strides must be multiples of 4 floats and the "
              "pointers 16-byte aligned");
    return BRIDCT_BAD_ALIGNMENT;
  }
  const size_t xe = strided_extent(h, w, input_row_pitch, input_array_stride, batch);
  const size_t ye = strided_extent(h, w, output_row_pitch, output_array_stride, batch);
  const uintptr_t a = (uintptr_t)input, b = (uintptr_t)output;
  if (a <= b ? b - a < xe * sizeof(float) : a - b < ye * sizeof(float)) return BRIDCT_OVERLAPPING_BUFFERS;
  DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(plan device)");
  const BatchLayout lx{nullptr, (long long)input_array_stride, (long long)input_row_pitch};
  const BatchLayout ly{nullptr, (long long)output_array_stride, (long long)output_row_pitch};
  return launch_plain_layout(plan->dev, plan->h, plan->w, mode, input, output, (long long)batch, &lx, &ly,
                             (cudaStream_t)stream);
}

BRIDCT_API int bridct_plan_synchronize(bridct_plan* plan) {
  if (!plan) return BRIDCT_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize(plan->stream);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "bridct_plan_synchronize");
}

BRIDCT_API int bridct_plan_apply_batch(bridct_plan* plan, enum bridct_mode mode, const float* input,
                                       float* output, size_t batch) {
  if (!plan || !input || !output || (unsigned)mode > BRIDCT_ROUNDTRIP || batch == 0)
    return BRIDCT_INVALID_ARGUMENT;
  const size_t per = plan->elements * sizeof(float);
  const size_t bytes = per * batch;
  if (ranges_overlap((uintptr_t)input, bytes, (uintptr_t)output, bytes)) return BRIDCT_OVERLAPPING_BUFFERS;
  DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(plan device)");
  bool pin_in = false, pin_out = false;
  const float* dx = (const float*)device_address(input, &pin_in);
  float* dy = (float*)device_address(output, &pin_out);
  if (dx && dy && ((uintptr_t)dx | (uintptr_t)dy) % 16 == 0) {
    int s = launch_plain_form(plan, mode, dx, dy, (long long)batch, plan->stream);
    if (s) return s;
    cudaError_t e = cudaStreamSynchronize(plan->stream);
    return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "bridct_plan_apply_batch");
  }
  return host_batch_pipeline(plan, mode, input, output, batch, dx, dy, pin_in, pin_out);
}

BRIDCT_API int bridct_plan_roundtrip_batch(bridct_plan* plan, const float* input, float* output, size_t batch) {
  if (!plan || !input || !output || batch == 0) return BRIDCT_INVALID_ARGUMENT;
  const size_t bytes = plan->elements * sizeof(float) * batch;
  if (ranges_overlap((uintptr_t)input, bytes, (uintptr_t)output, bytes)) return BRIDCT_OVERLAPPING_BUFFERS;
  DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return cuda_fail(guard.status, "cudaSetDevice(plan device)");
  bool pin_in = false, pin_out = false;
  const float* dx = (const float*)device_address(input, &pin_in);
  float* dy = (float*)device_address(output, &pin_out);
  return host_batch_pipeline(plan, kModeSpectrumRT, input, output, batch, dx, dy, pin_in, pin_out);
}

BRIDCT_API size_t bridct_workspace_floats(int n) {
  if (n != 8 && n != 16 && n != 32 && n != 64 && n != 128 && n != 256) return 0;
  const size_t e = (size_t)n * n;
  return n <= 16 ? 2 * e : 8 * e + 2 * 1100 * 4 + 4 * 4 * 256 + 4 * (size_t)n * (4 * n + 4);
}

BRIDCT_API int bridct_apply(int n, enum bridct_mode mode, const float* input, float* output,
                            float* workspace, size_t workspace_count) {
  const size_t needed = bridct_workspace_floats(n);
  if (!needed || !input || !output || !workspace || (unsigned)mode > BRIDCT_ROUNDTRIP)
    return BRIDCT_INVALID_ARGUMENT;
  if (workspace_count < needed) return BRIDCT_WORKSPACE_TOO_SMALL;
  if ((uintptr_t)workspace % 16) return BRIDCT_BAD_ALIGNMENT;
  const size_t bytes = (size_t)n * n * sizeof(float), wb = needed * sizeof(float);
  if (ranges_overlap((uintptr_t)input, bytes, (uintptr_t)output, bytes) ||
      ranges_overlap((uintptr_t)input, bytes, (uintptr_t)workspace, wb) ||
      ranges_overlap((uintptr_t)output, bytes, (uintptr_t)workspace, wb))
    return BRIDCT_OVERLAPPING_BUFFERS;
  // The GPU needs no caller scratch.  Device staging comes from a per-thread plan cache
  // (one plan per square size and device), created on the first call of each size.
  bridct_plan* p = thread_square_plan(n);
  if (!p) return BRIDCT_DEVICE_ERROR;
  return bridct_plan_apply(p, mode, input, output);
}

}  // extern "C"

extern "C" BRIDCT_API int bridct_plan_apply_form_device(bridct_plan* plan, enum bridct_mode mode,
                                                        enum bridct_form form, const float* input,
                                                        float* output, size_t batch, void* stream) {
  if (form == BRIDCT_FORM_SJ) return bridct_plan_apply_device(plan, mode, input, output, batch, stream);
  if (!plan) return BRIDCT_INVALID_ARGUMENT;
  bridct::DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return bridct::cuda_fail(guard.status, "cudaSetDevice(plan device)");
  return bridct::apply_tc_form(plan, (int)mode, (int)form, input, output, batch, stream, nullptr, 0);
}

extern "C" BRIDCT_API size_t bridct_plan_form_workspace_bytes(const bridct_plan* plan, enum bridct_form form,
                                                              size_t batch) {
  if (!plan || batch == 0 || form == BRIDCT_FORM_SJ) return 0;
  return bridct::tc_workspace_bytes(plan, (int)form, batch);
}

extern "C" BRIDCT_API int bridct_plan_apply_form_device_ws(bridct_plan* plan, enum bridct_mode mode,
                                                           enum bridct_form form, const float* input,
                                                           float* output, size_t batch, void* workspace,
                                                           size_t workspace_bytes, void* stream) {
  if (form == BRIDCT_FORM_SJ) return bridct_plan_apply_device(plan, mode, input, output, batch, stream);
  if (!plan) return BRIDCT_INVALID_ARGUMENT;
  const size_t need = bridct::tc_workspace_bytes(plan, (int)form, batch);
  if (need && !workspace) return BRIDCT_INVALID_ARGUMENT;
  if (workspace_bytes < need) return BRIDCT_WORKSPACE_TOO_SMALL;
  if ((uintptr_t)workspace % 16) return BRIDCT_BAD_ALIGNMENT;
  bridct::DeviceGuard guard(plan->device);
  if (guard.status != cudaSuccess) return bridct::cuda_fail(guard.status, "cudaSetDevice(plan device)");
  // a form that needs no scratch gets a non-NULL marker so that the plan's own scratch is not used
  static char unused;
  return bridct::apply_tc_form(plan, (int)mode, (int)form, input, output, batch, stream,
                               need ? workspace : static_cast<void*>(&unused), workspace_bytes);
}
