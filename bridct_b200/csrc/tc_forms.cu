// Host side of the tensor-core precision forms (BRIDCT_FORM_TC_*), 8x8 arrays.
//
// The Kronecker matrix of the orthonormal 8x8 DCT-II (and its transpose for the inverse) is
// built in float64, split into bf16 (hi/mid/lo) or tf32 (hi/lo) parts and laid out as the
// exact shared-memory image the UMMA B operand reads (K-major, 128-byte swizzle); the images
// are uploaded once per device.  Each call encodes two TMA tensor maps (input and output
// viewed as batch x 64 FP32 matrices, box 32 x 128, 128-byte swizzle) and launches k_tc8.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bridct_b200.h"
#include "bridct_internal.h"
#include "tc_blocks8.cuh"

namespace bridct {
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Round to bf16 (nearest even) and back, on the float32 representation.
float bf16_round(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&f, &u, 4);
  return f;
}

uint16_t bf16_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return (uint16_t)(u >> 16);
}

// Round to tf32 (10-bit mantissa), ties away from zero like cvt.rna.tf32.f32.
float tf32_round(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  memcpy(&f, &u, 4);
  return f;
}

// K[n][k]: n = output coefficient (i*8+j), k = input element (p*8+q).
std::vector<double> kron8(bool inverse) {
  double q[8][8];
  for (int k = 0; k < 8; ++k)
    for (int j = 0; j < 8; ++j) q[k][j] = std::sqrt((k ? 2.0 : 1.0) / 8) * std::cos(M_PI * k * (j + 0.5) / 8);
  std::vector<double> K(64 * 64);
  for (int n = 0; n < 64; ++n)
    for (int k = 0; k < 64; ++k) {
      const double f = q[n / 8][k / 8] * q[n % 8][k % 8];     // forward entry K[n][k]
      const double b = q[k / 8][n / 8] * q[k % 8][n % 8];     // transpose entry K[k][n]
      K[n * 64 + k] = inverse ? b : f;
    }
  return K;
}

std::vector<uint8_t> b_image(int form, bool inverse) {
  const std::vector<double> K = kron8(inverse);
  if (form == tc::BF16X3) {
    std::vector<uint8_t> img(tc::Layout<tc::BF16X3>::kBImage, 0);
    for (int n = 0; n < 64; ++n)
      for (int k = 0; k < 64; ++k) {
        const double v = K[n * 64 + k];
        const float h = bf16_round(v);
        const double r1 = v - h;
        const float m = bf16_round(r1);
        const float l = bf16_round(r1 - m);
        const float parts[3] = {h, m, l};
        const uint32_t off = tc::sw128(n, k / 8) + (k % 8) * 2;
        for (int s = 0; s < 3; ++s) {
          const uint16_t bits = bf16_bits(parts[s]);
          memcpy(&img[s * 8192 + off], &bits, 2);
        }
      }
    return img;
  }
  std::vector<uint8_t> img(tc::Layout<tc::TF32X3>::kBImage, 0);
  for (int n = 0; n < 64; ++n)
    for (int k = 0; k < 64; ++k) {
      const double v = K[n * 64 + k];
      const float h = tf32_round(v);
      const float l = tf32_round(v - h);
      const float parts[2] = {h, l};
      const uint32_t off = (k / 32) * 8192 + tc::sw128(n, (k % 32) / 4) + (k % 4) * 4;
      for (int s = 0; s < 2; ++s) memcpy(&img[s * 16384 + off], &parts[s], 4);
    }
  return img;
}

struct TcDevice {
  void* images[3][2] = {};   // [form][inverse]
  int* err = nullptr;
};

std::mutex g_tc_mutex;
std::map<int, TcDevice> g_tc;

TcDevice* tc_device(int dev) {
  std::lock_guard<std::mutex> lock(g_tc_mutex);
  auto it = g_tc.find(dev);
  if (it != g_tc.end()) return &it->second;
  TcDevice d;
  for (int form = 1; form <= 2; ++form)
    for (int inv = 0; inv < 2; ++inv) {
      const std::vector<uint8_t> img = b_image(form, inv != 0);
      if (cudaMalloc(&d.images[form][inv], img.size()) != cudaSuccess) return nullptr;
      if (cudaMemcpy(d.images[form][inv], img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return nullptr;
    }
  if (cudaMalloc(&d.err, sizeof(int)) != cudaSuccess || cudaMemset(d.err, 0, sizeof(int)) != cudaSuccess)
    return nullptr;
  g_tc[dev] = d;
  return &g_tc[dev];
}

bool make_map(CUtensorMap* m, const float* ptr, size_t rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[2] = {64, (cuuint64_t)rows};
  cuuint64_t strides[1] = {64 * sizeof(float)};
  cuuint32_t box[2] = {32, tc::kRows};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int FORM>
int launch_tc8(const bridct_plan* p, int inverse, const float* x, float* y, size_t batch, cudaStream_t st,
               TcDevice* d) {
  using L = tc::Layout<FORM>;
  auto k = tc::k_tc8<FORM>;
  static const int bps = [&]() {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kDynamic) != cudaSuccess) return 0;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, tc::kWsThreads, L::kDynamic) != cudaSuccess) return 0;
    return b;
  }();
  if (bps <= 0) return cuda_fail(cudaErrorInvalidConfiguration, "k_tc8 occupancy");
  CUtensorMap xm, ym;
  if (!make_map(&xm, x, batch) || !make_map(&ym, y, batch)) {
    set_error("cuTensorMapEncodeTiled failed");
    return BRIDCT_DEVICE_ERROR;
  }
  const int ntiles = (int)((batch + tc::kRows - 1) / tc::kRows);
  int grid = p->dev->sm_count * bps;
  if (grid > ntiles) grid = ntiles;
  k<<<grid, tc::kWsThreads, L::kDynamic, st>>>(xm, ym, reinterpret_cast<const uint4*>(d->images[FORM][inverse]),
                                               ntiles, d->err);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_tc8 launch");
}

}  // namespace

int apply_tc_form(bridct_plan* p, int mode, int form, const float* x, float* y, size_t batch, void* stream) {
  if (!p || !x || !y || mode < 0 || mode > 2 || batch == 0) return BRIDCT_INVALID_ARGUMENT;
  if (form != BRIDCT_FORM_TC_BF16X3 && form != BRIDCT_FORM_TC_TF32X3) {
    set_error("unsupported execution form");
    return BRIDCT_INVALID_ARGUMENT;
  }
  if (p->h != 8 || p->w != 8) {
    set_error("the tensor-core forms cover batches of 8x8 arrays");
    return BRIDCT_INVALID_ARGUMENT;
  }
  const size_t bytes = batch * 64 * sizeof(float);
  const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
  if ((a <= b ? b - a : a - b) < bytes) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((a | b) % 16) return BRIDCT_BAD_ALIGNMENT;
  if (batch > (size_t)0x7FFFFFFF * tc::kRows) return BRIDCT_INVALID_ARGUMENT;
  TcDevice* d = tc_device(p->device);
  if (!d) return cuda_fail(cudaGetLastError(), "tensor-core setup");
  cudaStream_t st = (cudaStream_t)stream;
  int s;
  if (mode == 2) {   // normalized round trip: forward into y, then inverse in place
    s = form == BRIDCT_FORM_TC_BF16X3 ? launch_tc8<tc::BF16X3>(p, 0, x, y, batch, st, d)
                                     : launch_tc8<tc::TF32X3>(p, 0, x, y, batch, st, d);
    if (s) return s;
    return form == BRIDCT_FORM_TC_BF16X3 ? launch_tc8<tc::BF16X3>(p, 1, y, y, batch, st, d)
                                        : launch_tc8<tc::TF32X3>(p, 1, y, y, batch, st, d);
  }
  return form == BRIDCT_FORM_TC_BF16X3 ? launch_tc8<tc::BF16X3>(p, mode, x, y, batch, st, d)
                                      : launch_tc8<tc::TF32X3>(p, mode, x, y, batch, st, d);
}

// Reads and clears the device's bounded-wait error flag (nonzero: a wait expired).
int tc_take_error(int device) {
  TcDevice* d = tc_device(device);
  if (!d) return 0;
  int v = 0;
  cudaMemcpy(&v, d->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (v) cudaMemset(d->err, 0, sizeof(int));
  return v;
}

}  // namespace bridct

extern "C" BRIDCT_API int bridct_device_timeout_flag(int device) { return bridct::tc_take_error(device); }
