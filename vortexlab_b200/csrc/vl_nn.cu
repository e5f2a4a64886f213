// Tensor-core and elementwise kernels of the learned warm start (a small convolutional network),
// with a C ABI that takes device pointers (the caller owns every buffer). The convolutions are
// expressed as BF16 GEMMs on tcgen05 (vl_gemm.cuh) around gather kernels (im2col / col2im).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/vortexlab.h"
#include "vl_gemm.cuh"
#include "vl_launch.hpp"

using bf16 = __nv_bfloat16;

namespace {

int fail(int code, const std::string& m) { return vl::set_error(code, m.c_str()); }

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mutex;

int encoder(PFN_cuTensorMapEncodeTiled_v12000* out) {
  std::lock_guard<std::mutex> g(g_encode_mutex);
  if (!g_encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return fail(VL_ECUDA, "cuTensorMapEncodeTiled is not available");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  *out = g_encode;
  return VL_OK;
}

// 2-D tensor map of a row-major BF16 matrix [rows][cols] with leading dimension ld (elements),
// box = 64 columns x box_rows rows, 128-byte swizzle. Out-of-range boxes read zeros.
int make_map(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc;
  int rc = encoder(&enc);
  if (rc) return rc;
  if (((uintptr_t)base & 15) || (ld * 2) % 16) return fail(VL_EINVAL, "GEMM operands need 16-byte aligned rows");
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)vl::gemm::BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(VL_EINVAL, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return VL_OK;
}

// Device workspace for split-K partial tiles, one per device, grown on demand. Split-K GEMMs of
// one device are therefore serialised on the caller's stream discipline: the library's own users
// issue them on a single stream.
std::mutex g_ws_mutex;
void* g_ws[64] = {};
size_t g_ws_bytes[64] = {};

int workspace(int dev, size_t bytes, void** out) {
  std::lock_guard<std::mutex> g(g_ws_mutex);
  if (dev < 0 || dev >= 64) return fail(VL_EINVAL, "device index out of range");
  if (g_ws_bytes[dev] < bytes) {
    if (g_ws[dev]) {
      cudaDeviceSynchronize();
      cudaFree(g_ws[dev]);
      g_ws[dev] = nullptr;
      g_ws_bytes[dev] = 0;
    }
    const size_t want = bytes + bytes / 2;
    cudaError_t e = cudaMalloc(&g_ws[dev], want);
    if (e != cudaSuccess) return fail(VL_ENOMEM, std::string("gemm workspace: ") + cudaGetErrorString(e));
    g_ws_bytes[dev] = want;
  }
  *out = g_ws[dev];
  return VL_OK;
}

// out[m, n] (leading dimension ldc) = (accumulate ? out : 0) + sum over z of ws[z][m][n], z in order.
__global__ void k_split_reduce(const float* __restrict__ ws, int splits, int M, int N, float* __restrict__ out,
                               int ldc, int accumulate) {
  const long long total = (long long)M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += ws[(long long)z * total + i];
    float* o = out + (i / N) * ldc + (i % N);
    *o = accumulate ? *o + s : s;
  }
}

template <int BN>
int launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, int K, int op,
                const vl::gemm::EpiParams& ep, cudaStream_t s) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  constexpr int smem = vl::gemm::smem_bytes<BN>();
  if (dev < 64 && !configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute(vl::gemm::k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return fail(VL_ECUDA, std::string("gemm smem attribute: ") + cudaGetErrorString(e));
    configured[dev] = true;
  }
  const int gx = (M + vl::gemm::BM - 1) / vl::gemm::BM, gy = (N + BN - 1) / BN;
  const int kblocks = (K + vl::gemm::BK - 1) / vl::gemm::BK;
  // Too few output tiles to fill the 148 SMs and a long K (weight gradients): split K so that about
  // two CTAs per SM run, each over at least 8 K-blocks; FP32 results without bias/activation only.
  int splits = 1;
  const int tiles = gx * gy;
  if (tiles < 148 && kblocks >= 16 && !(ep.flags & (vl::gemm::EPI_BIAS | vl::gemm::EPI_RELU | vl::gemm::EPI_BF16))) {
    splits = std::min(kblocks / 8, (296 + tiles - 1) / tiles);
    if (splits < 1) splits = 1;
  }
  const int kb_per = (kblocks + splits - 1) / splits;
  splits = (kblocks + kb_per - 1) / kb_per;
  vl::gemm::EpiParams p = ep;
  float* ws = nullptr;
  if (splits > 1) {
    void* w = nullptr;
    int rc = workspace(dev, (size_t)splits * M * N * sizeof(float), &w);
    if (rc) return rc;
    ws = (float*)w;
    p.out = ws;
    p.ldc = N;
    p.flags = 0;
    p.split_stride = (long long)M * N;
  } else {
    p.split_stride = 0;
  }
  // A short K per CTA (the im2col GEMMs of the narrow layers: 1-8 K-blocks) gains nothing from a
  // deep ring; two stages let 2 (BN 256) to 5 (BN 32) CTAs share an SM instead, so one CTA's
  // epilogue overlaps the next one's loads. TMEM stays within its 512 columns in both cases.
  const int stages = kb_per <= 8 ? 2 : vl::gemm::STAGES;
  dim3 grid(gx, gy, splits);
  vl::gemm::k_gemm_bf16<BN><<<grid, 128, vl::gemm::smem_bytes<BN>(stages), s>>>(ta, tb, kblocks, kb_per, stages, op, p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(VL_ECUDA, std::string("gemm launch: ") + cudaGetErrorString(e));
  if (splits > 1) {
    long long total = (long long)M * N;
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
    k_split_reduce<<<blocks, 256, 0, s>>>(ws, splits, M, N, (float*)ep.out, ep.ldc, ep.flags & vl::gemm::EPI_ACCUM);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(VL_ECUDA, std::string("gemm split reduce: ") + cudaGetErrorString(e));
  }
  return VL_OK;
}

}  // namespace

extern "C" {

int vl_nn_gemm_bf16(const void* a, int lda, const void* b, int ldb, int M, int N, int K, void* out, int ldc,
                    const float* bias, int flags, int bn, int* err, void* stream) {
  if (!a || !b || !out || M <= 0 || N <= 0 || K <= 0) return fail(VL_EINVAL, "gemm: bad arguments");
  if (bn != 32 && bn != 64 && bn != 128 && bn != 256) return fail(VL_EINVAL, "gemm: tile N must be 32, 64, 128 or 256");
  if ((flags & vl::gemm::EPI_BIAS) && !bias) return fail(VL_EINVAL, "gemm: bias requested without a bias");
  const int op = ((flags & VL_GEMM_A_MN) ? vl::gemm::OP_A_MN : 0) | ((flags & VL_GEMM_B_MN) ? vl::gemm::OP_B_MN : 0);
  if ((op & vl::gemm::OP_B_MN) && bn < 64) return fail(VL_EINVAL, "gemm: an MN-major B needs a tile N of 64 or more");
  CUtensorMap ta, tb;
  const bool amn = op & vl::gemm::OP_A_MN, bmn = op & vl::gemm::OP_B_MN;
  int rc = make_map(&ta, a, (uint64_t)(amn ? K : M), (uint64_t)(amn ? M : K), (uint64_t)lda, amn ? 64u : vl::gemm::BM);
  if (rc) return rc;
  rc = make_map(&tb, b, (uint64_t)(bmn ? K : N), (uint64_t)(bmn ? N : K), (uint64_t)ldb, bmn ? 64u : (uint32_t)bn);
  if (rc) return rc;
  vl::gemm::EpiParams ep;
  ep.out = out;
  ep.ldc = ldc;
  ep.bias = bias;
  ep.m_valid = M;
  ep.n_valid = N;
  ep.flags = flags & (vl::gemm::EPI_ACCUM | vl::gemm::EPI_BIAS | vl::gemm::EPI_RELU | vl::gemm::EPI_BF16);
  ep.err = err;
  ep.drop_load = (flags & VL_GEMM_TEST_TIMEOUT) ? 1 : 0;
  ep.spin_limit = ep.drop_load ? (1u << 12) : vl::gemm::kSpinLimit;
  cudaStream_t s = (cudaStream_t)stream;
  switch (bn) {
    case 32: return launch_gemm<32>(ta, tb, M, N, K, op, ep, s);
    case 64: return launch_gemm<64>(ta, tb, M, N, K, op, ep, s);
    case 128: return launch_gemm<128>(ta, tb, M, N, K, op, ep, s);
    default: return launch_gemm<256>(ta, tb, M, N, K, op, ep, s);
  }
}

}  // extern "C"

// ------------------------------------------------------------------ convolution gathers
// Activations are NHWC (row r = (b * H + y) * W + x, channels contiguous). A 3x3 convolution with
// padding 1 and stride s reads, for output pixel (b, oy, ox), the input pixels
// (s*oy + ky - 1, s*ox + kx - 1); its im2col row holds them in (ky, kx, c) order, zero-padded to
// kp columns (a multiple of 64, the GEMM's K block).
namespace {

__global__ void k_im2col(const bf16* __restrict__ x, int B, int H, int W, int C, int stride, int Ho, int Wo, int kp,
                         bf16* __restrict__ cols) {
  // one thread per 8 consecutive columns of a row: a single 16-byte load and store when C % 8 == 0
  const int G = kp >> 3;
  const long long total = (long long)B * Ho * Wo * G;
  const bool vec = (C & 7) == 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(i % G);
    const long long r = i / G;
    const int ox = (int)(r % Wo);
    const long long q = r / Wo;
    const int oy = (int)(q % Ho), b = (int)(q / Ho);
    const int k0 = g * 8;
    uint4 out = make_uint4(0u, 0u, 0u, 0u);
    if (vec) {
      if (k0 < 9 * C) {
        const int tap = k0 / C, c = k0 - tap * C;
        const int iy = stride * oy + tap / 3 - 1, ix = stride * ox + tap % 3 - 1;
        if (iy >= 0 && iy < H && ix >= 0 && ix < W)
          out = *reinterpret_cast<const uint4*>(x + (((long long)b * H + iy) * W + ix) * C + c);
      }
    } else {
      __align__(16) bf16 v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = k0 + j;
        v[j] = __float2bfloat16_rn(0.0f);
        if (k < 9 * C) {
          const int tap = k / C, c = k - tap * C;
          const int iy = stride * oy + tap / 3 - 1, ix = stride * ox + tap % 3 - 1;
          if (iy >= 0 && iy < H && ix >= 0 && ix < W) v[j] = x[(((long long)b * H + iy) * W + ix) * C + c];
        }
      }
      out = *reinterpret_cast<const uint4*>(v);
    }
    *reinterpret_cast<uint4*>(cols + r * kp + k0) = out;
  }
}

// dX[b, iy, ix, c] = sum over the (oy, ox, ky, kx) that read it of dcols[(b, oy, ox), (ky, kx, c)].
// One thread per 4 consecutive channels (float4 loads) when C % 4 == 0, else per channel.
__global__ void k_col2im(const float* __restrict__ dcols, int B, int H, int W, int C, int stride, int Ho, int Wo,
                         int kp, float* __restrict__ dx, int accumulate) {
  const int V = (C & 3) == 0 ? 4 : 1;
  const int G = C / V;
  const long long total = (long long)B * H * W * G;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % G) * V;
    const long long p = i / G;
    const int ix = (int)(p % W);
    const long long q = p / W;
    const int iy = (int)(q % H), b = (int)(q / H);
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = iy + 1 - ky;
      if (ty < 0 || ty % stride) continue;
      const int oy = ty / stride;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = ix + 1 - kx;
        if (tx < 0 || tx % stride) continue;
        const int ox = tx / stride;
        if (ox >= Wo) continue;
        const float* src = dcols + (((long long)b * Ho + oy) * Wo + ox) * kp + (ky * 3 + kx) * C + c;
        if (V == 4) {
          const float4 v = *reinterpret_cast<const float4*>(src);
          s[0] += v.x; s[1] += v.y; s[2] += v.z; s[3] += v.w;
        } else {
          s[0] += *src;
        }
      }
    }
    float* o = dx + p * C + c;
    for (int j = 0; j < V; ++j) o[j] = accumulate ? o[j] + s[j] : s[j];
  }
}

// dz = dy * (y > 0) (ReLU; y is the layer output) or dz = dy (no activation); BF16 copies of dz
// row-major [R, C] and transposed [C, R] for the two backward GEMMs, and colsum[c, t] = the sum of
// dz over the 32 rows of row tile t (fixed order), from which the bias gradient is reduced.
__global__ void k_act_bwd(const float* __restrict__ dy, const bf16* __restrict__ y, int R, int C, int relu,
                          bf16* __restrict__ dz, bf16* __restrict__ dzt, float* __restrict__ colsum, int ntiles) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    float v = 0.0f;
    if (r < R && c < C) {
      v = dy[(long long)r * C + c];
      if (relu && !(__bfloat162float(y[(long long)r * C + c]) > 0.0f)) v = 0.0f;
      const bf16 h = __float2bfloat16_rn(v);
      dz[(long long)r * C + c] = h;
      v = __bfloat162float(h);
    }
    tile[j][threadIdx.x] = v;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    const float v = tile[threadIdx.x][j];
    if (dzt && c < C && r < R) dzt[(long long)c * R + r] = __float2bfloat16_rn(v);
    float sum = v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (colsum && threadIdx.x == 0 && c < C) colsum[(long long)c * ntiles + blockIdx.y] = sum;
  }
}

// db[c] = sum over the row tiles t of colsum[c, t] (one block per channel, fixed tree).
__global__ void k_bias_grad(const float* __restrict__ colsum, int ntiles, float* __restrict__ db) {
  __shared__ float red[256];
  const int c = blockIdx.x;
  float s = 0.0f;
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) s += colsum[(long long)c * ntiles + t];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = red[0];
}

// BF16 transpose [R, C] -> [C, R] (R and C even): 64 x 64 tiles moved as pairs of elements.
__global__ void k_transpose_bf16(const bf16* __restrict__ a, int R, int C, bf16* __restrict__ at) {
  __shared__ bf16 tile[64][66];
  const int c0 = blockIdx.x * 64, r0 = blockIdx.y * 64;
  for (int j = threadIdx.y; j < 64; j += blockDim.y) {
    const int r = r0 + j, c = c0 + 2 * threadIdx.x;
    __nv_bfloat162 v = __floats2bfloat162_rn(0.0f, 0.0f);
    if (r < R && c < C) v = *reinterpret_cast<const __nv_bfloat162*>(a + (long long)r * C + c);
    tile[j][2 * threadIdx.x] = v.x;
    tile[j][2 * threadIdx.x + 1] = v.y;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 64; j += blockDim.y) {
    const int c = c0 + j, r = r0 + 2 * threadIdx.x;
    if (c < C && r < R) {
      __nv_bfloat162 v;
      v.x = tile[2 * threadIdx.x][j];
      v.y = tile[2 * threadIdx.x + 1][j];
      *reinterpret_cast<__nv_bfloat162*>(at + (long long)c * R + r) = v;
    }
  }
}

// Weights of the input-gradient convolution of a stride-1 3x3 layer: wf[c, (ky, kx, co)] =
// w[co, (2 - ky, 2 - kx, c)] (taps mirrored, input and output channels swapped), zero-padded to
// kpf columns. With it dX = conv3x3(dZ, wf), an im2col of dZ and one GEMM, with no col2im.
__global__ void k_flip_weights(const bf16* __restrict__ w, int cout, int cin, int kp, int kpf, bf16* __restrict__ wf) {
  const long long total = (long long)cin * kpf;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % kpf), c = (int)(i / kpf);
    bf16 v = __float2bfloat16_rn(0.0f);
    if (k < 9 * cout) {
      const int tap = k / cout, co = k - tap * cout;
      v = w[(long long)co * kp + (8 - tap) * cin + c];
    }
    wf[i] = v;
  }
}

// Nearest 2x upsampling of NHWC BF16 [B, H, W, C] -> [B, 2H, 2W, C] into channels [coff, coff + C)
// of an output with ctot channels; backward sums the four children into FP32.
__global__ void k_up2(const bf16* __restrict__ x, int B, int H, int W, int C, bf16* __restrict__ y, int ctot, int coff) {
  const long long total = (long long)B * 2 * H * 2 * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long p = i / C;
    const int X = (int)(p % (2 * W)), Y = (int)((p / (2 * W)) % (2 * H)), b = (int)(p / (4LL * W * H));
    y[p * ctot + coff + c] = x[(((long long)b * H + Y / 2) * W + X / 2) * C + c];
  }
}

__global__ void k_up2_bwd(const float* __restrict__ dy, int B, int H, int W, int C, int ctot, int coff,
                          float* __restrict__ dx, int accumulate) {
  const long long total = (long long)B * H * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long p = i / C;
    const int x = (int)(p % W), yy = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    float s = 0.0f;
    for (int dy2 = 0; dy2 < 2; ++dy2)
      for (int dx2 = 0; dx2 < 2; ++dx2)
        s += dy[((((long long)b * 2 * H + 2 * yy + dy2) * 2 * W) + 2 * x + dx2) * ctot + coff + c];
    dx[i] = accumulate ? dx[i] + s : s;
  }
}

// Copies channels [0, C) of x ([R, C]) into channels [coff, coff + C) of y ([R, ctot]) and back.
__global__ void k_copy_channels(const bf16* __restrict__ x, long long R, int C, bf16* __restrict__ y, int ctot, int coff) {
  const long long total = R * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
    y[(i / C) * ctot + coff + (i % C)] = x[i];
}

__global__ void k_slice_channels_f32(const float* __restrict__ y, long long R, int ctot, int coff, int C,
                                     float* __restrict__ x, int accumulate) {
  const long long total = R * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const float v = y[(i / C) * ctot + coff + (i % C)];
    x[i] = accumulate ? x[i] + v : v;
  }
}

// Masked mean-squared error over R pixels x the first `cuse` of C output channels (the target is
// [R, cuse]): loss partial sums per block (FP64) and the gradient dOut = 2 w (out - target) / count
// (zero on the other channels).
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ tgt, const float* __restrict__ w,
                      long long R, int C, int cuse, double inv_count, float* __restrict__ dout,
                      double* __restrict__ partial) {
  __shared__ double red[256];
  double s = 0.0;
  const long long total = R * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long r = i / C;
    const float wi = c < cuse ? w[r] : 0.0f;
    const float d = c < cuse ? out[i] - tgt[r * cuse + c] : 0.0f;
    s += (double)wi * d * d;
    dout[i] = (float)(2.0 * inv_count) * wi * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0] * inv_count;
}

// Adam (FP32 master weights); writes the BF16 copy the GEMMs read, padded layout kept by the
// caller (n values).
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16* __restrict__ wb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, long long n, bf16* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn(a[i]);
}

int grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 148 * 32 ? (g < 1 ? 1 : g) : 148 * 32);
}

int launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(VL_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return VL_OK;
}

}  // namespace

extern "C" {

int vl_nn_im2col(const void* x, int B, int H, int W, int C, int stride, int kp, void* cols, void* stream) {
  if (!x || !cols || (stride != 1 && stride != 2) || kp < 9 * C || kp % 64) return fail(VL_EINVAL, "im2col: bad arguments");
  if (((uintptr_t)x & 15) || ((uintptr_t)cols & 15)) return fail(VL_EINVAL, "im2col: buffers must be 16-byte aligned");
  const int Ho = (H + stride - 1) / stride, Wo = (W + stride - 1) / stride;
  k_im2col<<<grid_for((long long)B * Ho * Wo * (kp / 8)), 256, 0, (cudaStream_t)stream>>>(
      (const bf16*)x, B, H, W, C, stride, Ho, Wo, kp, (bf16*)cols);
  return launch_check("im2col");
}

int vl_nn_col2im(const float* dcols, int B, int H, int W, int C, int stride, int kp, float* dx, int accumulate,
                 void* stream) {
  if (!dcols || !dx || (stride != 1 && stride != 2) || kp < 9 * C || kp % 4) return fail(VL_EINVAL, "col2im: bad arguments");
  if (((uintptr_t)dcols & 15) || ((uintptr_t)dx & 15)) return fail(VL_EINVAL, "col2im: buffers must be 16-byte aligned");
  const int Ho = (H + stride - 1) / stride, Wo = (W + stride - 1) / stride;
  const long long work = (long long)B * H * W * ((C & 3) == 0 ? C / 4 : C);
  k_col2im<<<grid_for(work), 256, 0, (cudaStream_t)stream>>>(dcols, B, H, W, C, stride, Ho, Wo, kp, dx, accumulate);
  return launch_check("col2im");
}

int vl_nn_act_bwd(const float* dy, const void* y, int R, int C, int relu, void* dz, void* dzt, float* colsum,
                  void* stream) {
  if (!dy || !dz || (relu && !y)) return fail(VL_EINVAL, "act_bwd: bad arguments");
  dim3 grid((C + 31) / 32, (R + 31) / 32), block(32, 8);
  k_act_bwd<<<grid, block, 0, (cudaStream_t)stream>>>(dy, (const bf16*)y, R, C, relu, (bf16*)dz, (bf16*)dzt, colsum,
                                                      (R + 31) / 32);
  return launch_check("act_bwd");
}

int vl_nn_bias_grad(const float* colsum, int R, int C, float* db, void* stream) {
  if (!colsum || !db) return fail(VL_EINVAL, "bias_grad: bad arguments");
  k_bias_grad<<<C, 256, 0, (cudaStream_t)stream>>>(colsum, (R + 31) / 32, db);
  return launch_check("bias_grad");
}

int vl_nn_transpose_bf16(const void* a, int R, int C, void* at, void* stream) {
  if (!a || !at || (R & 1) || (C & 1)) return fail(VL_EINVAL, "transpose: bad arguments (R and C must be even)");
  if (((uintptr_t)a & 3) || ((uintptr_t)at & 3)) return fail(VL_EINVAL, "transpose: buffers must be 4-byte aligned");
  dim3 grid((C + 63) / 64, (R + 63) / 64), block(32, 8);
  k_transpose_bf16<<<grid, block, 0, (cudaStream_t)stream>>>((const bf16*)a, R, C, (bf16*)at);
  return launch_check("transpose");
}

int vl_nn_flip_weights(const void* w, int cout, int cin, int kp, int kpf, void* wf, void* stream) {
  if (!w || !wf || kp < 9 * cin || kpf < 9 * cout) return fail(VL_EINVAL, "flip_weights: bad arguments");
  k_flip_weights<<<grid_for((long long)cin * kpf), 256, 0, (cudaStream_t)stream>>>((const bf16*)w, cout, cin, kp, kpf,
                                                                                  (bf16*)wf);
  return launch_check("flip_weights");
}

int vl_nn_up2(const void* x, int B, int H, int W, int C, void* y, int ctot, int coff, void* stream) {
  if (!x || !y || coff + C > ctot) return fail(VL_EINVAL, "up2: bad arguments");
  k_up2<<<grid_for(4LL * B * H * W * C), 256, 0, (cudaStream_t)stream>>>((const bf16*)x, B, H, W, C, (bf16*)y, ctot, coff);
  return launch_check("up2");
}

int vl_nn_up2_bwd(const float* dy, int B, int H, int W, int C, int ctot, int coff, float* dx, int accumulate,
                  void* stream) {
  if (!dy || !dx || coff + C > ctot) return fail(VL_EINVAL, "up2_bwd: bad arguments");
  k_up2_bwd<<<grid_for((long long)B * H * W * C), 256, 0, (cudaStream_t)stream>>>(dy, B, H, W, C, ctot, coff, dx,
                                                                                  accumulate);
  return launch_check("up2_bwd");
}

int vl_nn_copy_channels(const void* x, long long R, int C, void* y, int ctot, int coff, void* stream) {
  if (!x || !y || coff + C > ctot) return fail(VL_EINVAL, "copy_channels: bad arguments");
  k_copy_channels<<<grid_for(R * C), 256, 0, (cudaStream_t)stream>>>((const bf16*)x, R, C, (bf16*)y, ctot, coff);
  return launch_check("copy_channels");
}

int vl_nn_slice_channels(const float* y, long long R, int ctot, int coff, int C, float* x, int accumulate,
                         void* stream) {
  if (!x || !y || coff + C > ctot) return fail(VL_EINVAL, "slice_channels: bad arguments");
  k_slice_channels_f32<<<grid_for(R * C), 256, 0, (cudaStream_t)stream>>>(y, R, ctot, coff, C, x, accumulate);
  return launch_check("slice_channels");
}

int vl_nn_mse(const float* out, const float* tgt, const float* w, long long R, int C, int cuse, double inv_count,
              float* dout, double* partial, int blocks, void* stream) {
  if (!out || !tgt || !w || !dout || !partial || blocks < 1 || cuse < 1 || cuse > C)
    return fail(VL_EINVAL, "mse: bad arguments");
  k_mse<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, tgt, w, R, C, cuse, inv_count, dout, partial);
  return launch_check("mse");
}

int vl_nn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
               int step, void* wb, void* stream) {
  if (!w || !g || !m || !v || step < 1) return fail(VL_EINVAL, "adam: bad arguments");
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, (bf16*)wb);
  return launch_check("adam");
}

int vl_nn_f32_to_bf16(const float* a, long long n, void* b, void* stream) {
  if (!a || !b) return fail(VL_EINVAL, "f32_to_bf16: bad arguments");
  k_f32_to_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(a, n, (bf16*)b);
  return launch_check("f32_to_bf16");
}

}  // extern "C"
