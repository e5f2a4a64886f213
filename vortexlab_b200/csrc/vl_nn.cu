// Tensor-core and elementwise kernels of the learned warm start (a small convolutional network),
// with a C ABI that takes device pointers (the caller owns every buffer). The convolutions are
// expressed as BF16 GEMMs on tcgen05 (vl_gemm.cuh) around gather kernels (im2col / col2im).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

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

template <int BN>
int launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, int K, const vl::gemm::EpiParams& ep,
                cudaStream_t s) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  constexpr int smem = vl::gemm::smem_bytes<BN>();
  if (dev < 64 && !configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute(vl::gemm::k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return fail(VL_ECUDA, std::string("gemm smem attribute: ") + cudaGetErrorString(e));
    configured[dev] = true;
  }
  dim3 grid((M + vl::gemm::BM - 1) / vl::gemm::BM, (N + BN - 1) / BN);
  const int kblocks = (K + vl::gemm::BK - 1) / vl::gemm::BK;
  vl::gemm::k_gemm_bf16<BN><<<grid, 128, smem, s>>>(ta, tb, kblocks, ep);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(VL_ECUDA, std::string("gemm launch: ") + cudaGetErrorString(e));
  return VL_OK;
}

}  // namespace

extern "C" {

int vl_nn_gemm_bf16(const void* a, int lda, const void* b, int ldb, int M, int N, int K, void* out, int ldc,
                    const float* bias, int flags, int bn, int* err, void* stream) {
  if (!a || !b || !out || M <= 0 || N <= 0 || K <= 0) return fail(VL_EINVAL, "gemm: bad arguments");
  if (bn != 32 && bn != 64 && bn != 128 && bn != 256) return fail(VL_EINVAL, "gemm: tile N must be 32, 64, 128 or 256");
  if ((flags & vl::gemm::EPI_BIAS) && !bias) return fail(VL_EINVAL, "gemm: bias requested without a bias");
  CUtensorMap ta, tb;
  int rc = make_map(&ta, a, (uint64_t)M, (uint64_t)K, (uint64_t)lda, vl::gemm::BM);
  if (rc) return rc;
  rc = make_map(&tb, b, (uint64_t)N, (uint64_t)K, (uint64_t)ldb, (uint32_t)bn);
  if (rc) return rc;
  vl::gemm::EpiParams ep;
  ep.out = out;
  ep.ldc = ldc;
  ep.bias = bias;
  ep.m_valid = M;
  ep.n_valid = N;
  ep.flags = flags;
  ep.err = err;
  cudaStream_t s = (cudaStream_t)stream;
  switch (bn) {
    case 32: return launch_gemm<32>(ta, tb, M, N, K, ep, s);
    case 64: return launch_gemm<64>(ta, tb, M, N, K, ep, s);
    case 128: return launch_gemm<128>(ta, tb, M, N, K, ep, s);
    default: return launch_gemm<256>(ta, tb, M, N, K, ep, s);
  }
}

}  // extern "C"
