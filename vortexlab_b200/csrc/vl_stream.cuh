// The bulk-copy-fed bulk kernel of the narrow storage formats (FP32 and 16-bit populations).
//
// The register-fed kernels (vl_pair.cuh) keep at most the loads their registers can hold in flight:
// 72 bytes per thread, which at the occupancy their registers allow leaves the HBM pipe short of
// requests (their warps stall on memory most of the time). Here the loads go straight into shared
// memory instead: one producer thread per CTA streams, with the asynchronous bulk copy engine
// (cp.async.bulk, global to shared, completion counted on an mbarrier), the nine plane segments
// each output row tile needs into a ring of NST stages, while 8 consumer warps update the cells
// of earlier tiles from the staged copies and store them. Bytes in flight are then bounded by the
// ring (NST x 9 x (tile + 2 halo) values per CTA), not by registers.
//
// A work unit is a tile of TW = 256 V cells of one output row y. Its plane i streams from row y
// (planes 0, 1, 3), y - 1 (2, 5, 6) or y + 1 (4, 7, 8), periodic in y; each segment covers the
// tile plus a 16-byte halo on each side (for the x-shifted planes), clipped at the row ends, where
// the consumers read the wrapped value from global memory. Every copy starts and ends on a 16-byte
// boundary: the kernel is used only when a row is a whole number of 16-byte units (nx * sizeof(S)
// a multiple of 16) and the plane stride too. CTAs are persistent: CTA c takes units c, c + G, ...
// of the launch's rows. The consumers run the same per-cell code as the register-fed kernel
// (group_update), reading the staged copies, so results are bit-identical to it.
//
// Every mbarrier wait is bounded (kSpinLimit polls): on a timeout the CTA sets the sim's error word
// (StepParams::ctl->nonfinite with the step as t) and stops; the producer then waits, again bounded,
// for its copies in flight before the CTA exits.
#pragma once

#include <cstdint>

#include "vl_pair.cuh"

namespace vl {
namespace stream {

constexpr int kConsumerWarps = 8;
constexpr int kThreads = 32 * (kConsumerWarps + 1);
constexpr int kStages = 4;
constexpr unsigned kSpinLimit = 1u << 24;

__device__ __forceinline__ uint32_t s_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(bar)), "r"(count));
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s_u32(bar)) : "memory");
}
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = s_u32(bar);
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 32) __nanosleep(20);
  }
  return false;
}
// One bulk copy of `bytes` (a multiple of 16) from global to shared memory (both 16-byte aligned),
// counted on `bar`.
__device__ __forceinline__ void copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   s_u32(dst)),
               "l"(src), "r"(bytes), "r"(s_u32(bar))
               : "memory");
}

template <class S, int V>
struct Geometry {
  static constexpr int TW = 32 * V * kConsumerWarps;          // cells of a tile
  static constexpr int H = 16 / (int)sizeof(S);                // halo cells (16 bytes)
  static constexpr int SEG = TW + 2 * H;                       // cells of a staged plane segment
  static constexpr int STAGE_BYTES = 9 * SEG * (int)sizeof(S);
  static constexpr int SMEM_BYTES = kStages * STAGE_BYTES;
};

// Source row of plane i for output row y: the row the population streams from.
__device__ __forceinline__ int src_row(int i, int y, int ny) {
  const int dy = (i == 2 || i == 5 || i == 6) ? -1 : ((i == 4 || i == 7 || i == 8) ? 1 : 0);
  const int r = y + dy;
  return r < 0 ? ny - 1 : (r >= ny ? 0 : r);
}

}  // namespace stream

template <class S, int V, int CK, int STAGED>
__global__ void __launch_bounds__(stream::kThreads, 2) k_bulk_stream(const __grid_constant__ StepParams p,
                                                                    const S* __restrict__ a, S* __restrict__ b) {
  using G = stream::Geometry<S, V>;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[stream::kStages], empty[stream::kStages];
  __shared__ int failed;
  const int nx = p.nx, ny = p.ny;
  const int tpr = (nx + G::TW - 1) / G::TW;
  const int r0 = p.bulk_b0, r1 = min(p.bulk_b0 + p.bulk_n, ny);
  const long long units = (long long)(r1 - r0) * tpr;
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31u);
  if (threadIdx.x == 0) {
    for (int s = 0; s < stream::kStages; ++s) {
      stream::bar_init(&full[s], 1);
      stream::bar_init(&empty[s], stream::kConsumerWarps);
    }
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == stream::kConsumerWarps) {
    // producer
    if (lane == 0) {
      long long j = 0;
      for (long long u = blockIdx.x; u < units; u += gridDim.x, ++j) {
        const int s = (int)(j % stream::kStages);
        const uint32_t round = (uint32_t)(j / stream::kStages);
        if (!stream::bar_wait(&empty[s], (round & 1u) ^ 1u)) { atomicExch(&failed, 1); break; }
        if (*(volatile int*)&failed) break;
        const int y = r0 + (int)(u / tpr);
        const int x0 = (int)(u % tpr) * G::TW;
        const int start = max(x0 - G::H, 0);
        const int end = min(x0 + G::TW + G::H, nx);
        const uint32_t bytes = (uint32_t)(end - start) * (uint32_t)sizeof(S);
        stream::bar_expect_tx(&full[s], 9u * bytes);
        S* stage = reinterpret_cast<S*>(smem + (size_t)s * G::STAGE_BYTES);
#pragma unroll 1
        for (int i = 0; i < 9; ++i) {
          const S* src = a + (size_t)i * p.ns + (size_t)stream::src_row(i, y, ny) * nx + start;
          stream::copy_g2s(stage + i * G::SEG + (start - x0 + G::H), src, bytes, &full[s]);
        }
      }
      // drain: every issued copy has landed (or the bounded waits ran out) before the CTA exits
      const long long issued = j;
      for (long long q = issued > stream::kStages ? issued - stream::kStages : 0; q < issued; ++q)
        stream::bar_wait(&full[q % stream::kStages], (uint32_t)(q / stream::kStages) & 1u);
    }
  } else {
    // consumers
    PairTask t;
    t.nx = nx;
    t.ny = ny;
    t.ns = p.ns;
    t.flag = p.flag;
    t.ck = CK;
    t.op = (float)p.op;
    t.om = (float)p.om;
    t.kend = p.nb;
    t.bdesc = p.bdesc;
    t.lb = (const float*)p.lb;
    t.ownc = p.ownc;
    t.nbs = p.nbs;
    t.bad = &p.ctl->nonfinite;
    t.bad_t = &p.ctl->nonfinite_t;
    t.t_now = &p.ctl->t;
    t.seg = G::SEG;
    t.halo = G::H;
    long long j = 0;
    for (long long u = blockIdx.x; u < units; u += gridDim.x, ++j) {
      const int s = (int)(j % stream::kStages);
      const uint32_t round = (uint32_t)(j / stream::kStages);
      if (!stream::bar_wait(&full[s], round & 1u)) {
        if (lane == 0) atomicExch(&failed, 1);
        break;
      }
      t.y = r0 + (int)(u / tpr);
      t.x0t = (int)(u % tpr) * G::TW;
      t.xw = t.x0t + warp * 32 * V;
      t.stage = smem + (size_t)s * G::STAGE_BYTES;
      t.wfirst = (STAGED && t.xw < nx)
                     ? __ldg(p.warp_bfirst + (size_t)t.y * (size_t)(p.tiles_per_row * (kBlock / 32)) + (t.xw >> 5))
                     : 0;
      if (t.xw < nx) group_update<S, V, STAGED, true>(t, a, b);
      __syncwarp();
      if (lane == 0) stream::bar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && failed) mark_diverged(&p.ctl->nonfinite, &p.ctl->nonfinite_t, &p.ctl->t);
}

}  // namespace vl
