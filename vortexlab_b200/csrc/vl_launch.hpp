// Host-side table of kernel launchers, one per population storage precision. The FP64 table is
// compiled without FMA contraction (bit-identical to the reference); the FP32 and FP16-shifted
// tables are compiled with it.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace vl {

struct StepParams;
struct BatchParams;

struct Launchers {
  size_t elem;  // bytes per stored population value
  // One step: the link kernel then the bulk kernel, both on `s`. ck: 0 BGK, 1 TRT, 2 forced, plus
  // 0x100 link kernel only, 0x200 bulk kernel only, 0x400 the staged pair (k_links_stage, then the
  // bulk kernel that also updates boundary cells).
  cudaError_t (*step)(const StepParams& p, int ck, const void* a, void* b, cudaStream_t s);
  cudaError_t (*init)(int n, unsigned ns, const uint8_t* flag, const double* rho, const double* ux,
                      const double* uy, double rho0, double ux0, double uy0, void* a, void* b, cudaStream_t s);
  // Init from a coarse grid of normalised fields (k_init_grid).
  cudaError_t (*init_grid)(int nx, int n, unsigned ns, const uint8_t* flag, const float* g, int gh, int gw, int gc,
                           double x0, double dx, double y0, double dy, double u, void* a, void* b, cudaStream_t s);
  cudaError_t (*to_f64)(int n, unsigned ns, const void* a, double* out, cudaStream_t s);
  cudaError_t (*from_f64)(int n, unsigned ns, const double* in, void* a, cudaStream_t s);
  cudaError_t (*macros)(int n, unsigned ns, const uint8_t* flag, double gx, double gy, const void* a,
                        double* rho, double* ux, double* uy, cudaStream_t s);
  cudaError_t (*reduce)(int n, unsigned ns, const uint8_t* flag, double gx, double gy, const void* a,
                        double* out, int blocks, cudaStream_t s);
  cudaError_t (*gather)(int m, unsigned ns, const int32_t* cells, const void* a, double* out, cudaStream_t s);
  // Records the pressure probe of the last step of a batch (one block).
  cudaError_t (*probe)(const StepParams& p, const void* a, cudaStream_t s);
  // One step of a batch of tunnels: which = 1 link kernel, 2 bulk kernel, 3 both; + 4 the staged
  // pair (link rules only, then the bulk kernel that also updates boundary cells).
  cudaError_t (*batch_step)(const BatchParams& p, int ntiles, int nchunks, int which, const void* a, void* b,
                            cudaStream_t s);
  // Gathers the boundary nodes' own populations of `a` into the staged step's compact copy.
  cudaError_t (*gather_own)(const StepParams& p, const void* a, cudaStream_t s);
  // The same for the tunnels of a batch's current link chunks.
  cudaError_t (*batch_gather_own)(const BatchParams& p, int nchunks, const void* a, cudaStream_t s);
};

// Records a failure for vl_last_error / vl_last_status (thread-local) and returns `code`.
int set_error(int code, const char* msg);

const Launchers& launchers_f64();
const Launchers& launchers_f32();
const Launchers& launchers_f16s();
const Launchers& launchers_f16c();
const Launchers& launchers_f16x();

}  // namespace vl
