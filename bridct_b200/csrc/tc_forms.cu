// Host side of the tensor-core precision forms (BRIDCT_FORM_TC_*).
//
// 8x8 arrays: the Kronecker matrix of the orthonormal 8x8 DCT-II (and its transpose for the inverse) is
// built in float64, split into bf16 (hi/mid/lo) or tf32 (hi/lo) parts and laid out as the
// exact shared-memory image the UMMA B operand reads (K-major, 128-byte swizzle); the images
// are uploaded once per device.  Each call encodes two TMA tensor maps (input and output
// viewed as batch x 64 FP32 matrices, box 32 x 128, 128-byte swizzle) and launches k_tc8.
//
// Every other shape: two row passes of k_tcpass per batch of arrays (pass 1 over rows of length W
// into scratch, pass 2 over rows of length H into the output), over chunks of up to 1 GB of
// arrays; BF16x3 on 64x64 arrays runs both passes in one launch (k_tc64) with the intermediate on
// chip.  The B images hold C_L (or C_L^T for the inverse) split into bf16 or tf32 parts, one
// 64-row slice per N-block, in the K-major 128-byte-swizzled layout; rows of 8, 16 or 32 points
// run as 64-float super-rows against a block-diagonal B, and the 512- and 1024-point passes stream
// their B slices through the ring instead of keeping them resident.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bridct_b200.h"
#include "bridct_internal.h"
#include "tc_blocks8.cuh"
#include "tc_pass.cuh"
#include "tc_fused64.cuh"
#include "tc_fp8.cuh"

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
      // per 32-element K atom: Kh rows then Kl rows (the N = 128 MMA reads both)
      const uint32_t off = (k / 32) * 16384 + tc::sw128(n, (k % 32) / 4) + (k % 4) * 4;
      for (int s = 0; s < 2; ++s) memcpy(&img[off + s * 8192], &parts[s], 4);
    }
  return img;
}

struct TcDevice {
  void* images[3][2] = {};   // [form][inverse]
  void* pass_images[3][8][2] = {};   // [form][log2(points per row) - 3][inverse], built on first use
  void* fp8_images[8][2] = {};       // [log2(L) - 3][inverse]: E4M3 codes of C or C^T (block-diagonal below 128)
  float* fp8_scales[8][2] = {};      // their 32x32 tile scales
  int* err = nullptr;
};

// Orthonormal DCT-II matrix C_L[n][k] = sqrt((n ? 2 : 1) / L) cos(pi n (k + 1/2) / L).
std::vector<double> dct_matrix(int L) {
  std::vector<double> c((size_t)L * L);
  for (int n = 0; n < L; ++n)
    for (int k = 0; k < L; ++k)
      c[(size_t)n * L + k] = std::sqrt((n ? 2.0 : 1.0) / L) * std::cos(M_PI * n * (k + 0.5) / L);
  return c;
}

// B image of the row pass for rows of length L: slice nb (64 output columns) at nb * kBBytes,
// laid out [K-chunk][split][8 KB atom column]; B[n][k] = C_L[n][k] (forward) or C_L[k][n].  With
// SUB > 1 the 64-float super-rows hold SUB rows of LS = 64 / SUB points, and B is block-diagonal:
// SUB copies of C_LS (zeros elsewhere).
template <int FORM, int L, int SUB = 1>
std::vector<uint8_t> pass_image(bool inverse) {
  using PL = tc::PassLayout<FORM, L>;
  constexpr int kc_len = tc::PassForm<FORM>::kKC;
  constexpr int LS = L / SUB;
  const std::vector<double> c = dct_matrix(LS);
  std::vector<uint8_t> img((size_t)PL::kBlocks * PL::kBBytes, 0);
  for (int n = 0; n < L; ++n)
    for (int k = 0; k < L; ++k) {
      if (n / LS != k / LS) continue;   // off the diagonal blocks: zero
      const int nn = n % LS, kk0 = k % LS;
      const double v = inverse ? c[(size_t)kk0 * LS + nn] : c[(size_t)nn * LS + kk0];
      const int nb = n / 64, nl = n % 64, kc = k / kc_len, kk = k % kc_len;
      uint8_t* slice = &img[(size_t)nb * PL::kBBytes];
      if (FORM == tc::BF16X3) {
        const float h = bf16_round(v);
        const double r1 = v - h;
        const float m = bf16_round(r1);
        const float l = bf16_round(r1 - m);
        const float parts[3] = {h, m, l};
        const uint32_t off = tc::sw128(nl, kk / 8) + (kk % 8) * 2;
        for (int sp = 0; sp < 3; ++sp) {
          const uint16_t bits = bf16_bits(parts[sp]);
          memcpy(slice + (size_t)(kc * 3 + sp) * tc::kBAtom + off, &bits, 2);
        }
      } else {
        const float h = tf32_round(v);
        const float l = tf32_round(v - h);
        const float parts[2] = {h, l};
        const uint32_t off = tc::sw128(nl, kk / 4) + (kk % 4) * 4;
        for (int sp = 0; sp < 2; ++sp)
          memcpy(slice + (size_t)(kc * 2 + sp) * tc::kBAtom + off, &parts[sp], 4);
      }
    }
  return img;
}

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

// Value of E4M3 code c (1 sign, 4 exponent bits with bias 7, 3 mantissa bits; 0x7F is NaN).
double e4m3_value(int c) {
  const int e = (c >> 3) & 15, m = c & 7;
  const double mag = e == 0 ? m * std::ldexp(1.0, -9) : (1.0 + m / 8.0) * std::ldexp(1.0, e - 7);
  return (c & 0x80) ? -mag : mag;
}

// Nearest E4M3 code to v (ties to the even code), saturating at +-448.
uint8_t e4m3_encode(double v) {
  const double a = std::fabs(v);
  int best = 0;
  double bd = a;
  for (int c = 1; c <= 0x7E; ++c) {
    const double d = std::fabs(e4m3_value(c) - a);
    if (d < bd || (d == bd && (c & 1) == 0)) {
      best = c;
      bd = d;
    }
  }
  return (uint8_t)(best | (v < 0 && best ? 0x80 : 0));
}

// E4M3 image of the FP8 pass's B for rows of L points: C_L (forward) or C_L^T, block-diagonal
// with LS / L copies for super-rows of LS = max(L, 128) codes.  Slice nb (64 rows) at nb * 64 * LS
// bytes, laid out [K atom of 128][64 rows x 128 bytes, SW128]; scales [LS/32 row bands][LS/32
// K-tiles] (1 for the all-zero tiles off the diagonal).
void fp8_image(int L, bool inverse, std::vector<uint8_t>& img, std::vector<float>& sc) {
  const std::vector<double> c = dct_matrix(L);
  const int LS = L < 128 ? 128 : L;
  auto at = [&](int n, int k) {
    if (n / L != k / L) return 0.0;
    n %= L;
    k %= L;
    return inverse ? c[(size_t)k * L + n] : c[(size_t)n * L + k];
  };
  const int nt = LS / 32;
  sc.assign((size_t)nt * nt, 1.0f);
  img.assign((size_t)LS * LS, 0);
  for (int bn = 0; bn < nt; ++bn)
    for (int bk = 0; bk < nt; ++bk) {
      double amax = 0.0;
      for (int i = 0; i < 32; ++i)
        for (int j = 0; j < 32; ++j) amax = std::max(amax, std::fabs(at(bn * 32 + i, bk * 32 + j)));
      const float s = amax > 0 ? (float)(amax / tc::kE4M3Max) : 1.0f;
      sc[(size_t)bn * nt + bk] = s;
      for (int i = 0; i < 32; ++i)
        for (int j = 0; j < 32; ++j) {
          const int n = bn * 32 + i, k = bk * 32 + j;
          const size_t slice = (size_t)(n / 64) * 64 * LS;
          const size_t off = slice + (size_t)(k / 128) * 8192 + tc::sw128(n % 64, (k % 128) / 16) + (k % 16);
          img[off] = e4m3_encode(at(n, k) / s);
        }
    }
}

// Row matrix (rows x L FP32) viewed by TMA in boxes of 32 x 128, 128-byte swizzle.
bool make_rows_map(CUtensorMap* m, const float* ptr, size_t rows, int L) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)L, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)L * sizeof(float)};
  cuuint32_t box[2] = {32, tc::kRows};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr int lg_points(int n) { return n <= 8 ? 0 : 1 + lg_points(n / 2); }

template <int FORM, int L, int SUB = 1>
const uint4* pass_image_device(TcDevice* d, bool inverse) {
  constexpr int li = lg_points(L / SUB);
  std::lock_guard<std::mutex> lock(g_tc_mutex);
  void*& slot = d->pass_images[FORM][li][inverse ? 1 : 0];
  if (!slot) {
    const std::vector<uint8_t> img = pass_image<FORM, L, SUB>(inverse);
    void* ptr = nullptr;
    if (cudaMalloc(&ptr, img.size()) != cudaSuccess) return nullptr;
    if (cudaMemcpy(ptr, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(ptr);
      return nullptr;
    }
    slot = ptr;
  }
  return reinterpret_cast<const uint4*>(slot);
}

// One row pass: rows x (L / SUB) matrix at x -> transposed arrays (R = 1 << rshift rows each) at
// out.  SUB > 1: the rows are read as rows / SUB super-rows of L = 64 floats.
template <int FORM, int L, int SUB = 1>
int launch_pass(const bridct_plan* p, bool inverse, const float* x, float* out, size_t rows, int rshift,
                cudaStream_t st, TcDevice* d) {
  using PL = tc::PassLayout<FORM, L>;
  auto k = tc::k_tcpass<FORM, L, SUB>;
  if (kernel_setup(reinterpret_cast<const void*>(k), PL::kDynamic, tc::kPassThreads) <= 0)
    return cuda_fail(cudaErrorInvalidConfiguration, "k_tcpass shared memory");
  const uint4* img = pass_image_device<FORM, L, SUB>(d, inverse);
  if (!img) return cuda_fail(cudaGetLastError(), "tensor-core coefficient upload");
  const size_t srows = rows / SUB;   // SUB divides every array's row count (>= 8)
  CUtensorMap xm;
  if (!make_rows_map(&xm, x, srows, L)) {
    set_error("cuTensorMapEncodeTiled failed");
    return BRIDCT_DEVICE_ERROR;
  }
  const long long mtiles = (long long)((srows + tc::kRows - 1) / tc::kRows);
  long long slots = p->dev->sm_count / PL::kBlocks;
  if (slots > mtiles) slots = mtiles;
  if (slots < 1) slots = 1;
  cudaError_t e = launch_pdl(k, (unsigned)(slots * PL::kBlocks), tc::kPassThreads, PL::kDynamic, st, true, xm, out,
                             img, (long long)srows, rshift, d->err);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_tcpass launch");
}

// BF16x3 on 64x64 arrays: both passes in one launch of k_tc64.
int launch_fused64(const bridct_plan* p, bool inverse, const float* x, float* y, size_t batch, cudaStream_t st,
                   TcDevice* d) {
  using F = tc::Fused64;
  if (kernel_setup(reinterpret_cast<const void*>(tc::k_tc64), F::kDynamic, F::kThreads) <= 0)
    return cuda_fail(cudaErrorInvalidConfiguration, "k_tc64 shared memory");
  const uint4* img = pass_image_device<tc::BF16X3, 64>(d, inverse);
  if (!img) return cuda_fail(cudaGetLastError(), "tensor-core coefficient upload");
  CUtensorMap xm;
  if (!make_rows_map(&xm, x, batch * 64, 64)) {
    set_error("cuTensorMapEncodeTiled failed");
    return BRIDCT_DEVICE_ERROR;
  }
  const long long tiles = (long long)((batch + 1) / 2);
  const long long grid = tiles < p->dev->sm_count ? tiles : p->dev->sm_count;
  cudaError_t e = launch_pdl(tc::k_tc64, (unsigned)grid, F::kThreads, F::kDynamic, st, true, xm, y, img,
                             (long long)batch, d->err);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_tc64 launch");
}

// ---- FP8 form ---------------------------------------------------------------------------

int log2i(int v);

// E4M3 super-rows (rows x LS codes) viewed by TMA in boxes of 128 rows x 128 bytes.
bool make_fp8_map(CUtensorMap* m, const uint8_t* ptr, size_t rows, int L) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)L, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)L};
  cuuint32_t box[2] = {128, tc::kRows};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(ptr), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool fp8_tables(TcDevice* d, int L, bool inverse, const uint4** img, const float** sc) {
  std::lock_guard<std::mutex> lock(g_tc_mutex);
  const int li = log2i(L) - 3, iv = inverse ? 1 : 0;
  if (!d->fp8_images[li][iv]) {
    std::vector<uint8_t> im;
    std::vector<float> scl;
    fp8_image(L, inverse, im, scl);
    void* pi = nullptr;
    void* ps = nullptr;
    if (cudaMalloc(&pi, im.size()) != cudaSuccess || cudaMalloc(&ps, scl.size() * 4) != cudaSuccess) return false;
    if (cudaMemcpy(pi, im.data(), im.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(ps, scl.data(), scl.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
      return false;
    d->fp8_images[li][iv] = pi;
    d->fp8_scales[li][iv] = static_cast<float*>(ps);
  }
  *img = reinterpret_cast<const uint4*>(d->fp8_images[li][iv]);
  *sc = d->fp8_scales[li][iv];
  return true;
}

// One FP8 row pass over `rows` rows of L = LS / SUB codes (super-rows of SUB rows).
template <int LS, int SUB, int UKT>
int launch_fp8pass(const bridct_plan* p, bool inverse, const uint8_t* q, const float* sx, float* out, size_t rows,
                   int rshift, cudaStream_t st, TcDevice* d) {
  using F = tc::Fp8Layout<LS, SUB, UKT>;
  constexpr int L = LS / SUB;
  auto k = tc::k_fp8pass<LS, SUB, UKT>;
  if (kernel_setup(reinterpret_cast<const void*>(k), F::kDynamic, F::kThreads) <= 0)
    return cuda_fail(cudaErrorInvalidConfiguration, "k_fp8pass shared memory");
  const uint4* img = nullptr;
  const float* sc = nullptr;
  if (!fp8_tables(d, L, inverse, &img, &sc)) return cuda_fail(cudaGetLastError(), "FP8 coefficient upload");
  CUtensorMap m;
  const size_t srows = (rows + SUB - 1) / SUB;
  if (!make_fp8_map(&m, q, srows, LS)) {
    set_error("cuTensorMapEncodeTiled failed");
    return BRIDCT_DEVICE_ERROR;
  }
  constexpr int kBlocks = LS / 64;
  const long long mtiles = (long long)((srows + tc::kRows - 1) / tc::kRows);
  long long slots = p->dev->sm_count / kBlocks;
  if (slots > mtiles) slots = mtiles;
  if (slots < 1) slots = 1;
  cudaError_t e = launch_pdl(k, (unsigned)(slots * kBlocks), F::kThreads, F::kDynamic, st, true, m, sx, out, img, sc,
                             (long long)rows, rshift, d->err);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_fp8pass launch");
}

// Quantizes the rows (nrows x L, arrays of 1 << rshift rows) into E4M3 codes q and scales sx of
// min(R, 32) x min(L, 32) tiles, and zeroes the codes after the rows up to the end of the last
// 128-code super-row.
int launch_quant8(const float* rows, uint8_t* q, float* sx, size_t nrows, int L, int rshift, cudaStream_t st) {
  const int tr_shift = rshift < 5 ? rshift : 5, tl = L < 32 ? L : 32;
  const long long ntiles = (long long)(nrows >> tr_shift) * (L / tl);
  const int sub = L < 128 ? 128 / L : 1;
  const int pad = (int)(((nrows + sub - 1) / sub * sub - nrows) * L);
  const long long per_block = 8LL * tc::quant8_tiles_per_warp(tr_shift, L);
  tc::k_quant8<<<(unsigned)((ntiles + per_block - 1) / per_block), 256, 0, st>>>(rows, q, sx, ntiles, L, tr_shift,
                                                                                  pad);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_quant8 launch");
}

struct Fp8Scratch {
  float *t, *r, *r2, *z, *sx;
  uint8_t* q;
};

// Unrefined FP8 transform of nb arrays: quantize, pass over rows of W, quantize, pass over rows of H.
int fp8_transform(const bridct_plan* p, bool inverse, const float* src, float* dst, size_t nb, const Fp8Scratch& s,
                  cudaStream_t st, TcDevice* d) {
  const int h = p->h, w = p->w;
  auto pass = [&](int L, const uint8_t* q, const float* sx, float* out, size_t rows, int rshift) {
    switch (L) {
      case 8: return launch_fp8pass<128, 16, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
      case 16: return launch_fp8pass<128, 8, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
      case 32: return launch_fp8pass<128, 4, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
      case 64: return launch_fp8pass<128, 2, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
      case 128: return launch_fp8pass<128, 1, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
      case 256: return launch_fp8pass<256, 1, 8>(p, inverse, q, sx, out, rows, rshift, st, d);
      case 512: return launch_fp8pass<512, 1, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
      default: return launch_fp8pass<1024, 1, 4>(p, inverse, q, sx, out, rows, rshift, st, d);
    }
  };
  int e = launch_quant8(src, s.q, s.sx, nb * h, w, log2i(h), st);
  if (!e) e = pass(w, s.q, s.sx, s.t, nb * h, log2i(h));
  if (!e) e = launch_quant8(s.t, s.q, s.sx, nb * w, h, log2i(w), st);
  if (!e) e = pass(h, s.q, s.sx, dst, nb * w, log2i(w));
  return e;
}

// One refinement step: dst = T8(src) + T8(src - T32^-1(T8(src))), with the plain FP32 form for
// the inverse and the residual in FP32.  src and dst must differ.
int fp8_refined(const bridct_plan* p, bool inverse, const float* src, float* dst, size_t nb, const Fp8Scratch& s,
                cudaStream_t st, TcDevice* d) {
  const long long n4 = (long long)(nb * p->elements / 4);
  const unsigned grid = (unsigned)std::min<long long>((n4 + 255) / 256, 4 * 148);
  int e = fp8_transform(p, inverse, src, dst, nb, s, st, d);
  if (!e) e = launch_plain_form(p, inverse ? 0 : 1, dst, s.r, (long long)nb, st);
  if (e) return e;
  tc::k_residual<<<grid, 256, 0, st>>>(reinterpret_cast<const float4*>(src), reinterpret_cast<float4*>(s.r), n4);
  e = fp8_transform(p, inverse, s.r, s.r2, nb, s, st, d);
  if (e) return e;
  tc::k_accumulate<<<grid, 256, 0, st>>>(reinterpret_cast<float4*>(dst), reinterpret_cast<const float4*>(s.r2), n4);
  cudaError_t ce = cudaGetLastError();
  return ce == cudaSuccess ? BRIDCT_OK : cuda_fail(ce, "FP8 refinement");
}

// Arrays per chunk of the FP8 form.  Chunks of 256 MB: the twelve launches of a refined
// transform dominate smaller chunks (2048 arrays of 256x256, same outputs: 16 MB 304 GB/s,
// 32 MB 344, 64 MB 352-366, 256 MB 382, 1 GB 389); the scratch needs about 17 bytes per element
// of a chunk: four FP32 buffers, the E4M3 codes (plus one super-row of padding) and the tile
// scales (at most one per 64 elements).
size_t fp8_scale_floats(size_t ce) { return (ce / 64 + 256 + 63) & ~size_t(63); }

size_t fp8_chunk(size_t elems, size_t batch, size_t* bytes) {
  size_t chunk = (size_t(256) << 20) / (elems * sizeof(float));
  if (chunk < 1) chunk = 1;
  if (chunk > batch) chunk = batch;
  const size_t ce = chunk * elems;
  *bytes = 16 * ce + 4 * fp8_scale_floats(ce) + ce + 1024;
  return chunk;
}

// Scratch of `need` bytes: the caller's workspace when given, else the plan's own (grown under
// the plan's lock, so that two host threads never free and reallocate it at once).
void* scratch_for(bridct_plan* p, void* workspace, size_t need, int* status) {
  *status = BRIDCT_OK;
  if (workspace) return workspace;
  std::lock_guard<std::mutex> lock(p->tc_mu);
  if (p->tc_bytes < need) {
    if (p->tc_mem) cudaFree(p->tc_mem);
    p->tc_mem = nullptr;
    p->tc_bytes = 0;
    cudaError_t e = cudaMalloc(&p->tc_mem, need);
    if (e != cudaSuccess) {
      *status = cuda_fail(e, "tensor-core scratch");
      return nullptr;
    }
    p->tc_bytes = need;
  }
  return p->tc_mem;
}

int apply_fp8(bridct_plan* p, int mode, const float* x, float* y, size_t batch, cudaStream_t st, TcDevice* d,
              void* workspace) {
  const size_t elems = p->elements;
  size_t need = 0;
  const size_t chunk = fp8_chunk(elems, batch, &need);
  const size_t ce = chunk * elems;
  int status = BRIDCT_OK;
  float* base = static_cast<float*>(scratch_for(p, workspace, need, &status));
  if (!base) return status;
  Fp8Scratch s{base, base + ce, base + 2 * ce, base + 3 * ce, base + 4 * ce, nullptr};
  s.q = reinterpret_cast<uint8_t*>(s.sx + fp8_scale_floats(ce));
  for (size_t b0 = 0; b0 < batch; b0 += chunk) {
    const size_t nb = batch - b0 < chunk ? batch - b0 : chunk;
    const float* xc = x + b0 * elems;
    float* yc = y + b0 * elems;
    int e = fp8_refined(p, mode == 1, xc, yc, nb, s, st, d);
    if (!e && mode == 2) {
      e = fp8_refined(p, true, yc, s.z, nb, s, st, d);
      if (!e && cudaMemcpyAsync(yc, s.z, nb * elems * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        e = cuda_fail(cudaGetLastError(), "FP8 round trip copy");
    }
    if (e) return e;
  }
  return BRIDCT_OK;
}

template <int FORM>
int pass_by_length(const bridct_plan* p, int L, bool inverse, const float* x, float* out, size_t rows, int rshift,
                   cudaStream_t st, TcDevice* d) {
  switch (L) {
    case 8: return launch_pass<FORM, 64, 8>(p, inverse, x, out, rows, rshift, st, d);
    case 16: return launch_pass<FORM, 64, 4>(p, inverse, x, out, rows, rshift, st, d);
    case 32: return launch_pass<FORM, 64, 2>(p, inverse, x, out, rows, rshift, st, d);
    case 64: return launch_pass<FORM, 64>(p, inverse, x, out, rows, rshift, st, d);
    case 128: return launch_pass<FORM, 128>(p, inverse, x, out, rows, rshift, st, d);
    case 256: return launch_pass<FORM, 256>(p, inverse, x, out, rows, rshift, st, d);
    case 512: return launch_pass<FORM, 512>(p, inverse, x, out, rows, rshift, st, d);
    case 1024: return launch_pass<FORM, 1024>(p, inverse, x, out, rows, rshift, st, d);
    default: return BRIDCT_INVALID_ARGUMENT;
  }
}

int log2i(int v) {
  int r = 0;
  while ((1 << r) < v) ++r;
  return r;
}

// Arrays per pass pair: up to 1 GB, so that batches up to that size run each pass as one launch.
// Chunks of 48 MB kept the intermediate in L2 but measured slower (2048 x 256^2: BF16x3 826 ->
// 962, TF32x3 565 -> 680 GB/s): the passes are bound by the shared-memory port, not by HBM, and
// every chunk adds launch tails.  The plan-owned scratch holds one chunk.
constexpr size_t kSepChunkBytes = size_t(1024) << 20;

// Separable form: per batch of arrays, pass 1 (rows of W) x -> scratch, pass 2 (rows of H)
// scratch -> y; the round trip runs the forward pair then the inverse pair on the same batch.
size_t sep_chunk(size_t elems, size_t batch, size_t* bytes) {
  size_t chunk = kSepChunkBytes / (elems * sizeof(float));
  if (chunk < 1) chunk = 1;
  if (chunk > batch) chunk = batch;
  *bytes = chunk * elems * sizeof(float);
  return chunk;
}

template <int FORM>
int apply_sep(bridct_plan* p, int mode, const float* x, float* y, size_t batch, cudaStream_t st, TcDevice* d,
              void* workspace) {
  if (FORM == tc::BF16X3 && p->h == 64 && p->w == 64) {
    int s = launch_fused64(p, mode == 1, x, y, batch, st, d);
    if (s || mode != 2) return s;
    return launch_fused64(p, true, y, y, batch, st, d);   // each CTA rewrites only tiles it has read
  }
  const size_t elems = (size_t)p->h * p->w;
  size_t need = 0;
  const size_t chunk = sep_chunk(elems, batch, &need);
  int status = BRIDCT_OK;
  float* t = static_cast<float*>(scratch_for(p, workspace, need, &status));
  if (!t) return status;
  const int lh = log2i(p->h), lw = log2i(p->w);
  for (size_t b0 = 0; b0 < batch; b0 += chunk) {
    const size_t nb = batch - b0 < chunk ? batch - b0 : chunk;
    const float* xc = x + b0 * elems;
    float* yc = y + b0 * elems;
    for (int dir = 0; dir < 2; ++dir) {
      const bool inverse = mode == 1 || dir == 1;
      if (dir == 1 && mode != 2) break;
      const float* src = dir == 0 ? xc : yc;
      int s = pass_by_length<FORM>(p, p->w, inverse, src, t, nb * p->h, lh, st, d);
      if (s) return s;
      s = pass_by_length<FORM>(p, p->h, inverse, t, yc, nb * p->w, lw, st, d);
      if (s) return s;
    }
  }
  return BRIDCT_OK;
}

template <int FORM>
int launch_tc8(const bridct_plan* p, int inverse, const float* x, float* y, size_t batch, cudaStream_t st,
               TcDevice* d) {
  using L = tc::Layout<FORM>;
  auto k = tc::k_tc8<FORM>;
  const int bps = kernel_setup(reinterpret_cast<const void*>(k), L::kDynamic, tc::kTc8Threads);
  if (bps <= 0) return cuda_fail(cudaErrorInvalidConfiguration, "k_tc8 occupancy");
  CUtensorMap xm, ym;
  if (!make_map(&xm, x, batch) || !make_map(&ym, y, batch)) {
    set_error("cuTensorMapEncodeTiled failed");
    return BRIDCT_DEVICE_ERROR;
  }
  const int ntiles = (int)((batch + tc::kRows - 1) / tc::kRows);
  int grid = p->dev->sm_count * bps;
  if (grid > ntiles) grid = ntiles;
  cudaError_t e = launch_pdl(k, (unsigned)grid, tc::kTc8Threads, L::kDynamic, st, true, xm, ym,
                             reinterpret_cast<const uint4*>(d->images[FORM][inverse]), ntiles, d->err);
  return e == cudaSuccess ? BRIDCT_OK : cuda_fail(e, "k_tc8 launch");
}

}  // namespace

size_t tc_workspace_bytes(const bridct_plan* p, int form, size_t batch) {
  if (!p || batch == 0) return 0;
  size_t bytes = 0;
  if (form == BRIDCT_FORM_TC_FP8) {
    fp8_chunk(p->elements, batch, &bytes);
    return bytes;
  }
  if (form != BRIDCT_FORM_TC_BF16X3 && form != BRIDCT_FORM_TC_TF32X3) return 0;
  if (p->h == 8 && p->w == 8) return 0;
  if (form == BRIDCT_FORM_TC_BF16X3 && p->h == 64 && p->w == 64) return 0;
  sep_chunk(p->elements, batch, &bytes);
  return bytes;
}

int apply_tc_form(bridct_plan* p, int mode, int form, const float* x, float* y, size_t batch, void* stream,
                  void* workspace, size_t) {
  if (!p || !x || !y || mode < 0 || mode > 2 || batch == 0) return BRIDCT_INVALID_ARGUMENT;
  if (form != BRIDCT_FORM_TC_BF16X3 && form != BRIDCT_FORM_TC_TF32X3 && form != BRIDCT_FORM_TC_FP8) {
    set_error("unsupported execution form");
    return BRIDCT_INVALID_ARGUMENT;
  }
  const bool kron = p->h == 8 && p->w == 8;   // every other supported shape runs two row passes
  const size_t elems = (size_t)p->h * p->w;
  const size_t bytes = batch * elems * sizeof(float);
  const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
  if ((a <= b ? b - a : a - b) < bytes) return BRIDCT_OVERLAPPING_BUFFERS;
  if ((a | b) % 16) return BRIDCT_BAD_ALIGNMENT;
  if (batch > (size_t)0x7FFFFFFF * tc::kRows / (elems / 64)) return BRIDCT_INVALID_ARGUMENT;
  TcDevice* d = tc_device(p->device);
  if (!d) return cuda_fail(cudaGetLastError(), "tensor-core setup");
  cudaStream_t st = (cudaStream_t)stream;
  if (form == BRIDCT_FORM_TC_FP8) return apply_fp8(p, mode, x, y, batch, st, d, workspace);
  if (!kron)
    return form == BRIDCT_FORM_TC_BF16X3 ? apply_sep<tc::BF16X3>(p, mode, x, y, batch, st, d, workspace)
                                        : apply_sep<tc::TF32X3>(p, mode, x, y, batch, st, d, workspace);
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
