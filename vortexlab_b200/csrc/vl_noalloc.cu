// Allocation-free FP64 reduction of a caller-owned population array: total mass, total momentum
// and largest speed (src/sim.rs:538-579), for callers that cannot allocate device memory — a host
// framework that owns every device byte through its own pool, a plugin that may only use the
// buffers it is handed, code running where cudaMalloc is not allowed. The per-block partial sums
// live in a file-scope __device__ array of fixed size instead of a cudaMalloc'd buffer.
//
// Compiled with -fmad=false like the other FP64 code.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/vortexlab.h"
#include "vl_device.cuh"
#include "vl_launch.hpp"

namespace {

constexpr int kCellsPerBlock = 16384;  // each block reduces one fixed chunk of cells
constexpr int kMaxBlocks = VL_REDUCE_STATIC_MAX_CELLS / kCellsPerBlock;
static_assert(kMaxBlocks * kCellsPerBlock == VL_REDUCE_STATIC_MAX_CELLS, "chunking");

// The scratch: 7 doubles per block (mass, px, py as Neumaier sum + compensation pairs, and the
// largest speed). Every GPU that loads this library holds it (112 KB) until the process exits.
// All calls share it; each call overwrites every slot it later reads, so nothing has to start at
// zero, but two calls whose kernels overlap on the GPU race on it.
static __device__ __align__(256) double g_reduce_scratch[kMaxBlocks * 7];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Per-block compensated sums over the block's chunk, then the same fixed shared-memory tree as
// the sim's reduction; one 7-double record per block.
__global__ void __launch_bounds__(vl::kBlock) k_reduce_chunks(const double* __restrict__ f, unsigned long long ns,
                                                             const uint8_t* __restrict__ flag, unsigned long long n,
                                                             double gx, double gy, double* __restrict__ part) {
  __shared__ double sh[7][vl::kBlock];
  double ms = 0, mc = 0, xs = 0, xc = 0, ys = 0, yc = 0, vmax = 0.0;
  bool nan = false;
  const unsigned long long begin = (unsigned long long)blockIdx.x * kCellsPerBlock;
  const unsigned long long end = begin + kCellsPerBlock < n ? begin + kCellsPerBlock : n;
  for (unsigned long long idx = begin + threadIdx.x; idx < end; idx += vl::kBlock) {
    if (flag[idx] == 2) continue;
    double p[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) p[i] = f[(unsigned long long)i * ns + idx];
#pragma unroll
    for (int i = 0; i < 9; ++i) vl::neumaier_add(ms, mc, p[i]);
#pragma unroll
    for (int i = 1; i < 9; ++i) {
      vl::neumaier_add(xs, xc, (double)vl::cx_of(i) * p[i]);
      vl::neumaier_add(ys, yc, (double)vl::cy_of(i) * p[i]);
    }
    double r, jx, jy;
    vl::moments(p, r, jx, jy);
    const double u = jx / r - 0.5 * gx, v = jy / r - 0.5 * gy;
    const double sp = sqrt(u * u + v * v);
    if (isnan(sp)) nan = true; else vmax = fmax(vmax, sp);
  }
  const int t = threadIdx.x;
  sh[0][t] = ms; sh[1][t] = mc; sh[2][t] = xs; sh[3][t] = xc; sh[4][t] = ys; sh[5][t] = yc;
  sh[6][t] = nan ? __longlong_as_double(0x7ff8000000000000ll) : vmax;
  __syncthreads();
  for (int s = vl::kBlock / 2; s > 0; s >>= 1) {
    if (t < s) {
      for (int k = 0; k < 3; ++k) {
        double s0 = sh[2 * k][t], c0 = sh[2 * k + 1][t];
        vl::neumaier_add(s0, c0, sh[2 * k][t + s]);
        sh[2 * k][t] = s0;
        sh[2 * k + 1][t] = c0 + sh[2 * k + 1][t + s];
      }
      const double o = sh[6][t + s], m = sh[6][t];
      sh[6][t] = (isnan(o) || isnan(m)) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(m, o);
    }
    __syncthreads();
  }
  if (t == 0)
    for (int k = 0; k < 7; ++k) part[7 * blockIdx.x + k] = sh[k][0];
}

// One thread combines the block records in block order (fixed), as the host does for the sim's
// reduction, and writes {mass, px, py, max speed} to the caller's buffer.
__global__ void k_reduce_final(const double* __restrict__ part, int blocks, double* __restrict__ out4) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double vm = 0.0;
  bool nan = false;
  for (int b = 0; b < blocks; ++b) {
    const double* o = part + 7 * b;
    for (int k = 0; k < 3; ++k) {
      double sum = acc[2 * k], comp = acc[2 * k + 1];
      vl::neumaier_add(sum, comp, o[2 * k]);
      acc[2 * k] = sum;
      acc[2 * k + 1] = comp + o[2 * k + 1];
    }
    if (isnan(o[6])) nan = true; else vm = fmax(vm, o[6]);
  }
  out4[0] = acc[0] + acc[1];
  out4[1] = acc[2] + acc[3];
  out4[2] = acc[4] + acc[5];
  out4[3] = nan ? __longlong_as_double(0x7ff8000000000000ll) : vm;
}

int fail(int code, const std::string& m) { return vl::set_error(code, m.c_str()); }

// Device address of the scratch array on the current device, looked up once per device. The
// array's name in host code is only a host-side handle, never a device address.
int scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(VL_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(VL_EUNSUPPORTED, "device index above 63");
  std::lock_guard<std::mutex> g(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_reduce_scratch);
    if (e != cudaSuccess || !p)
      return fail(VL_ECUDA, std::string("cudaGetSymbolAddress(g_reduce_scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = (double*)p;
  }
  *out = g_scratch_ptr[dev];
  return VL_OK;
}

}  // namespace

extern "C" {

int vl_reduce_f64_static(const double* populations, size_t plane_stride, const uint8_t* flag, size_t n,
                         double gx, double gy, double* out4, void* stream) {
  if (!populations || !flag || !out4) return fail(VL_EINVAL, "vl_reduce_f64_static: null pointer");
  if (n == 0) return fail(VL_EINVAL, "vl_reduce_f64_static: no cells");
  if (n > (size_t)VL_REDUCE_STATIC_MAX_CELLS)
    return fail(VL_EINVAL, "vl_reduce_f64_static: " + std::to_string(n) + " cells exceed the fixed scratch limit of " +
                               std::to_string(VL_REDUCE_STATIC_MAX_CELLS) + " (VL_REDUCE_STATIC_MAX_CELLS)");
  if (plane_stride < n) return fail(VL_EINVAL, "vl_reduce_f64_static: plane_stride must be at least n");
  double* scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc) return rc;
  const int blocks = (int)((n + kCellsPerBlock - 1) / kCellsPerBlock);
  cudaStream_t s = (cudaStream_t)stream;
  k_reduce_chunks<<<blocks, vl::kBlock, 0, s>>>(populations, plane_stride, flag, n, gx, gy, scratch);
  k_reduce_final<<<1, 32, 0, s>>>(scratch, blocks, out4);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(VL_ECUDA, std::string("vl_reduce_f64_static launch: ") + cudaGetErrorString(e));
  return VL_OK;
}

}  // extern "C"
