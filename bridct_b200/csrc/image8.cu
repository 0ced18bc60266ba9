// Block transform of an image in place-layout: every 8x8 block of a height x width float32
// image (any row pitch) is transformed where it lies, with optional JPEG-style quantization
// fused in (forward: round(Y / Q); inverse: X = Q . input before the DCT-III).
//
// One thread owns one block: it reads the block's eight 32-byte row segments straight from the
// image (consecutive threads own consecutive blocks of a block row, so each of a warp's loads
// covers 1 KB of one image row), runs the same register program as the contiguous 8x8 kernel
// (columns then rows, the reference's vertical-then-bands order, src/generated/rect.c:5-15),
// and writes the block back in image layout.  No shared memory, no workspace: reading a block
// completely before writing it makes in-place operation (output == input) safe.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/bridct.h"
#include "../../include/bridct_b200.h"
#include "bridct_internal.h"
#include "sj_blocks8.cuh"

namespace bridct {
namespace {

struct QuantTable {
  float q[64];
};

constexpr int kImgThreads = 128;

template <int MODE, bool QUANT>
__global__ void __launch_bounds__(kImgThreads) k_image8(const float* __restrict__ x, long long xpitch,
                                                        float* __restrict__ y, long long ypitch, int bcols,
                                                        QuantTable qt) {
  const int bx = blockIdx.x * kImgThreads + threadIdx.x;
  if (bx >= bcols) return;
  const float* src = x + (long long)blockIdx.y * 8 * xpitch + (long long)bx * 8;
  float v[64];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(src + r * xpitch));
    const float4 b = __ldcs(reinterpret_cast<const float4*>(src + r * xpitch) + 1);
    v[8 * r] = a.x; v[8 * r + 1] = a.y; v[8 * r + 2] = a.z; v[8 * r + 3] = a.w;
    v[8 * r + 4] = b.x; v[8 * r + 5] = b.y; v[8 * r + 6] = b.z; v[8 * r + 7] = b.w;
  }
  if constexpr (!QUANT) {
    b8_transform<MODE>(v);
  } else if constexpr (MODE == LM_FWD) {
    b8_transform<LM_FWD>(v);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = rintf(__fdiv_rn(v[k], qt.q[k]));
  } else if constexpr (MODE == LM_INV) {
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] *= qt.q[k];
    b8_transform<LM_INV>(v);
  } else {   // quantize / dequantize round trip
    b8_transform<LM_FWD>(v);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = rintf(__fdiv_rn(v[k], qt.q[k])) * qt.q[k];
    b8_transform<LM_INV>(v);
  }
  float* dst = y + (long long)blockIdx.y * 8 * ypitch + (long long)bx * 8;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    float4* d = reinterpret_cast<float4*>(dst + r * ypitch);
    __stcs(d, make_float4(v[8 * r], v[8 * r + 1], v[8 * r + 2], v[8 * r + 3]));
    __stcs(d + 1, make_float4(v[8 * r + 4], v[8 * r + 5], v[8 * r + 6], v[8 * r + 7]));
  }
}

template <bool QUANT>
cudaError_t launch_image8(int mode, const float* x, long long xp, float* y, long long yp, int h, int w,
                          const QuantTable& qt, cudaStream_t st) {
  const int bcols = w / 8;
  const dim3 grid((bcols + kImgThreads - 1) / kImgThreads, h / 8);
  if (mode == 0) k_image8<LM_FWD, QUANT><<<grid, kImgThreads, 0, st>>>(x, xp, y, yp, bcols, qt);
  else if (mode == 1) k_image8<LM_INV, QUANT><<<grid, kImgThreads, 0, st>>>(x, xp, y, yp, bcols, qt);
  else k_image8<LM_RT, QUANT><<<grid, kImgThreads, 0, st>>>(x, xp, y, yp, bcols, qt);
  return cudaGetLastError();
}

}  // namespace
}  // namespace bridct

extern "C" BRIDCT_API int bridct_image_blocks8_device(int mode, const float* input, size_t input_pitch,
                                                     float* output, size_t output_pitch, int height, int width,
                                                     const float* quant, void* stream) {
  using namespace bridct;
  if (!input || !output || mode < 0 || mode > 2 || height <= 0 || width <= 0 || height % 8 || width % 8 ||
      height / 8 > 65535 || input_pitch < (size_t)width || output_pitch < (size_t)width) {
    set_error("bridct_image_blocks8_device: invalid mode, pointer or geometry (axes must be positive "
              "multiples of 8, pitches at least the width)");
    return BRIDCT_INVALID_ARGUMENT;
  }
  if ((uintptr_t)input % 16 || (uintptr_t)output % 16 || input_pitch % 4 || output_pitch % 4) {
    set_error("bridct_image_blocks8_device: pointers must be 16-byte aligned and pitches multiples of 4");
    return BRIDCT_BAD_ALIGNMENT;
  }
  // The two footprints may be identical (in place) but must not otherwise overlap.
  const uintptr_t a0 = (uintptr_t)input, a1 = a0 + ((size_t)(height - 1) * input_pitch + width) * 4;
  const uintptr_t b0 = (uintptr_t)output, b1 = b0 + ((size_t)(height - 1) * output_pitch + width) * 4;
  const bool same = a0 == b0 && input_pitch == output_pitch;
  if (!same && a0 < b1 && b0 < a1) return BRIDCT_OVERLAPPING_BUFFERS;
  QuantTable qt{};
  if (quant) {
    for (int k = 0; k < 64; ++k) {
      if (!(quant[k] > 0.0f) || !std::isfinite(quant[k])) {
        set_error("bridct_image_blocks8_device: quantization steps must be finite and positive");
        return BRIDCT_INVALID_ARGUMENT;
      }
      qt.q[k] = quant[k];
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t e = quant ? launch_image8<true>(mode, input, (long long)input_pitch, output,
                                                     (long long)output_pitch, height, width, qt, st)
                              : launch_image8<false>(mode, input, (long long)input_pitch, output,
                                                      (long long)output_pitch, height, width, qt, st);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_image8 launch");
}
