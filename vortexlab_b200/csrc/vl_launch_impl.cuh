// Launcher bodies shared by the per-precision translation units.
#pragma once

#include <type_traits>

#include "vl_batch.cuh"
#include "vl_device.cuh"
#include "vl_launch.hpp"
#include "vl_pair.cuh"
#include "vl_stream.cuh"

namespace vl {

template <class S>
struct LaunchImpl {
  // which: 3 = both kernels of the step, 1 = the link kernel only, 2 = the bulk kernel only
  // (a step launched in two halves, for per-kernel timing). staged: the link-values kernel and the
  // bulk kernel that also updates the boundary cells, which must run in that order.
  // The bulk kernel over rows [p.bulk_b0, p.bulk_b0 + p.bulk_n) (clipped to the grid), in launches
  // of at most 65535 rows (the grid's y limit).
  // Narrow storage without a body force: the multi-cell kernel (k_bulkv, V cells of a row per
  // thread, one block per V * kBlock cells) with the largest V <= p.pairs that divides the row
  // length; otherwise the one-cell kernel (one block per kBlock cells).
  template <int CK>
  static int group_width(const StepParams& p) {
    if constexpr (std::is_same<S, double>::value || CK == 2) {
      return 1;
    } else {
      if (p.pairs >= 4 && p.nx % 4 == 0 && p.ns % 4 == 0) return 4;
      if (p.pairs >= 2 && p.nx % 2 == 0 && p.ns % 2 == 0) return 2;
      return 1;
    }
  }
  // The bulk-copy-fed kernel: narrow storage, a multi-cell form, a row length that is a multiple of
  // 16 cells and a plane stride of whole 16-byte units (every copy aligned). Persistent CTAs, two
  // per SM.
  static int sm_count() {
    static int n = 0;
    if (!n) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
      if (n <= 0) n = 148;
    }
    return n;
  }
  template <int V, int CK, int STAGED>
  static void launch_stream(const StepParams& p, const S* a, S* b, cudaStream_t s, int rows) {
    using G = stream::Geometry<S, V>;
    static bool ready = false;
    if (!ready) {
      cudaFuncSetAttribute(k_bulk_stream<S, V, CK, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
      ready = true;
    }
    const long long units = (long long)rows * ((p.nx + G::TW - 1) / G::TW);
    const long long cap = 2LL * sm_count();
    const unsigned grid = (unsigned)(units < cap ? units : cap);
    if (grid) k_bulk_stream<S, V, CK, STAGED><<<grid, stream::kThreads, G::SMEM_BYTES, s>>>(p, a, b);
  }
  template <int CK, int STAGED>
  static void launch_bulk(const StepParams& p, const S* a, S* b, cudaStream_t s) {
    const int r1 = p.bulk_b0 + p.bulk_n < p.ny ? p.bulk_b0 + p.bulk_n : p.ny;
    const int v = group_width<CK>(p);
    if constexpr (!std::is_same<S, double>::value && CK != 2) {
      if (v > 1 && p.stream && p.nx % 16 == 0 && ((size_t)p.ns * sizeof(S)) % 16 == 0 && r1 > p.bulk_b0) {
        if (v == 4)
          launch_stream<4, CK, STAGED>(p, a, b, s, r1 - p.bulk_b0);
        else
          launch_stream<2, CK, STAGED>(p, a, b, s, r1 - p.bulk_b0);
        return;
      }
    }
    for (int r = p.bulk_b0; r < r1; r += 65535) {
      StepParams q = p;
      q.bulk_b0 = r;
      const int rows = r1 - r < 65535 ? r1 - r : 65535;
      if constexpr (!std::is_same<S, double>::value && CK != 2) {
        if (v > 1) {
          const unsigned tiles = (unsigned)((p.nx + v * kBlock - 1) / (v * kBlock));
          if (v == 4)
            k_bulkv<S, 4, CK, STAGED><<<dim3(tiles, (unsigned)rows), kBlock, 0, s>>>(q, a, b);
          else
            k_bulkv<S, 2, CK, STAGED><<<dim3(tiles, (unsigned)rows), kBlock, 0, s>>>(q, a, b);
          continue;
        }
      }
      k_bulk<S, CK, STAGED><<<dim3((unsigned)p.tiles_per_row, (unsigned)rows), kBlock, 0, s>>>(q, a, b);
    }
  }
  template <int CK>
  static cudaError_t step_ck(const StepParams& p, const S* a, S* b, cudaStream_t s, int which, bool staged) {
    if (staged) {
      if (which & 1) k_links_stage<S><<<p.nlinkblk - p.link_b0 < p.link_n ? p.nlinkblk - p.link_b0 : p.link_n, kBlock, 0, s>>>(p, a);
      if (which & 2) launch_bulk<CK, 1>(p, a, b, s);
    } else {
      if (which & 1) k_links<S, CK><<<p.nlink, kBlock, 0, s>>>(p, a, b);
      if (which & 2) launch_bulk<CK, 0>(p, a, b, s);
    }
    return cudaGetLastError();
  }
  // ck: collision kind (0 BGK, 1 TRT, 2 forced) in the low byte; bit 8 = link kernel only,
  // bit 9 = bulk kernel only, bit 10 = the staged pair.
  static cudaError_t step(const StepParams& p, int ck, const void* a, void* b, cudaStream_t s) {
    const S* A = (const S*)a;
    S* B = (S*)b;
    const int which = (ck & 0x300) ? ((ck & 0x100) ? 1 : 0) | ((ck & 0x200) ? 2 : 0) : 3;
    const bool staged = (ck & 0x400) != 0;
    switch (ck & 0xff) {
      case 0: return step_ck<0>(p, A, B, s, which, staged);
      case 2: return step_ck<2>(p, A, B, s, which, staged);
      default: return step_ck<1>(p, A, B, s, which, staged);
    }
  }
  static int grid_for(int n) { return n <= 0 ? 1 : (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16; }
  static cudaError_t init(int n, unsigned ns, const uint8_t* flag, const double* rho, const double* ux,
                          const double* uy, double rho0, double ux0, double uy0, void* a, void* b, cudaStream_t s) {
    k_init<S><<<grid_for(n), 256, 0, s>>>(n, ns, flag, rho, ux, uy, rho0, ux0, uy0, (S*)a, (S*)b);
    return cudaGetLastError();
  }
  static cudaError_t init_grid(int nx, int n, unsigned ns, const uint8_t* flag, const float* g, int gh, int gw, int gc,
                               double x0, double dx, double y0, double dy, double u, void* a, void* b, cudaStream_t s) {
    k_init_grid<S><<<grid_for(n), 256, 0, s>>>(nx, n, ns, flag, g, gh, gw, gc, x0, dx, y0, dy, u, (S*)a, (S*)b);
    return cudaGetLastError();
  }
  static cudaError_t to_f64(int n, unsigned ns, const void* a, double* out, cudaStream_t s) {
    k_to_f64<S><<<grid_for(n), 256, 0, s>>>(n, ns, (const S*)a, out);
    return cudaGetLastError();
  }
  static cudaError_t from_f64(int n, unsigned ns, const double* in, void* a, cudaStream_t s) {
    k_from_f64<S><<<grid_for(n), 256, 0, s>>>(n, ns, in, (S*)a);
    return cudaGetLastError();
  }
  static cudaError_t macros(int n, unsigned ns, const uint8_t* flag, double gx, double gy, const void* a,
                            double* rho, double* ux, double* uy, cudaStream_t s) {
    k_macros<S><<<grid_for(n), 256, 0, s>>>(n, ns, flag, gx, gy, (const S*)a, rho, ux, uy);
    return cudaGetLastError();
  }
  static cudaError_t reduce(int n, unsigned ns, const uint8_t* flag, double gx, double gy, const void* a,
                            double* out, int blocks, cudaStream_t s) {
    k_reduce<S><<<blocks, kBlock, 0, s>>>(n, ns, flag, gx, gy, (const S*)a, out);
    return cudaGetLastError();
  }
  static cudaError_t gather(int m, unsigned ns, const int32_t* cells, const void* a, double* out, cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    k_gather<S><<<(m + 127) / 128, 128, 0, s>>>(m, ns, cells, (const S*)a, out);
    return cudaGetLastError();
  }
  static cudaError_t probe(const StepParams& p, const void* a, cudaStream_t s) {
    k_probe<S><<<1, kBlock, 0, s>>>(p, (const S*)a);
    return cudaGetLastError();
  }
  // which: 1 link kernel, 2 bulk kernel, 3 both; + 4 the staged pair.
  static cudaError_t batch_step(const BatchParams& p, int ntiles, int nchunks, int which, const void* a, void* b,
                                cudaStream_t s) {
    bool pairs = false;
    if constexpr (!std::is_same<S, double>::value) pairs = p.pairs != 0;
    if ((which & 1) && nchunks > 0 && p.noutl > 0) k_batch_outlet<S><<<p.noutl, kBlock, 0, s>>>(p, (const S*)a);
    if (which & 4) {
      if ((which & 1) && nchunks > 0) k_batch_links<S, 1><<<nchunks, kBlock, 0, s>>>(p, (const S*)a, (S*)b);
      if ((which & 2) && ntiles > 0) {
        if constexpr (!std::is_same<S, double>::value) {
          if (pairs) k_batch_bulk2<S, 1><<<ntiles, kBlock, 0, s>>>(p, (const S*)a, (S*)b);
        }
        if (!pairs) k_batch_bulk<S, 1><<<ntiles, kBlock, 0, s>>>(p, (const S*)a, (S*)b);
      }
    } else {
      if ((which & 1) && nchunks > 0) k_batch_links<S, 0><<<nchunks, kBlock, 0, s>>>(p, (const S*)a, (S*)b);
      if ((which & 2) && ntiles > 0) {
        if constexpr (!std::is_same<S, double>::value) {
          if (pairs) k_batch_bulk2<S, 0><<<ntiles, kBlock, 0, s>>>(p, (const S*)a, (S*)b);
        }
        if (!pairs) k_batch_bulk<S, 0><<<ntiles, kBlock, 0, s>>>(p, (const S*)a, (S*)b);
      }
    }
    return cudaGetLastError();
  }
  static cudaError_t batch_gather_own(const BatchParams& p, int nchunks, const void* a, cudaStream_t s) {
    if (nchunks <= 0) return cudaSuccess;
    k_batch_gather_own<S><<<nchunks, kBlock, 0, s>>>(p, (const S*)a);
    return cudaGetLastError();
  }
  static cudaError_t gather_own(const StepParams& p, const void* a, cudaStream_t s) {
    if (p.nb <= 0) return cudaSuccess;
    k_gather_own<S><<<grid_for(p.nb), 256, 0, s>>>(p.nb, p.ns, p.nbs, p.bnode_idx, (const S*)a, (S*)p.ownc);
    return cudaGetLastError();
  }
  static const Launchers& table() {
    static const Launchers t = {sizeof(S), &step, &init, &init_grid, &to_f64, &from_f64, &macros, &reduce, &gather, &probe, &batch_step,
                                &gather_own, &batch_gather_own};
    return t;
  }
};

}  // namespace vl
