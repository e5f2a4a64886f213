// The bulk-copy-fed bulk kernel of the narrow storage formats (FP32 and 16-bit populations).
//
// The register-fed kernels (vl_pair.cuh) keep at most the loads their registers can hold in flight:
// 72 bytes per thread, which at the occupancy their registers allow leaves the HBM pipe short of
// requests (their warps stall on memory most of the time). Here the loads go straight into shared
// memory instead: one producer thread per CTA streams, with the asynchronous bulk copy engine
// (cp.async.bulk, global to shared, completion counted on an mbarrier), everything a row tile
// needs into a ring of kStages stages, while 8 consumer warps update the cells of earlier tiles
// from the staged copies and store them. Bytes in flight are then bounded by the ring, not by
// registers, and the consumers read nothing but shared memory on the common path.
//
// A work unit is a tile of TW = 256 V cells of one output row y. Its stage holds, per plane i, the
// segment of the row the plane streams from (y for planes 0, 1, 3; y - 1 for 2, 5, 6; y + 1 for
// 4, 7, 8; periodic in y) covering the tile and a 16-byte halo on each side (for the x-shifted
// planes); at the row's first and last tile the halo beyond the row end is filled from the other
// end of the row (the periodic wrap in x); then the tile's flags. Every copy starts and ends on a
// 16-byte boundary: the kernel is used only when the row length is a multiple of 16 cells (so rows
// of populations and of flags are whole 16-byte units) and the plane stride a whole number of
// 16-byte units. CTAs are persistent: CTA c takes units c, c + G, ... of the launch's rows. The
// per-cell operations are those of the register-fed kernel, so results are bit-identical to it.
//
// Every mbarrier wait is bounded (kSpinLimit polls): on a timeout the CTA marks the sim's run as
// failed (the divergence word StepParams::ctl->nonfinite, with the step) and stops; the producer
// then waits, again bounded, for its copies in flight before the CTA exits.
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
  static constexpr int PLANE_BYTES = SEG * (int)sizeof(S);
  static constexpr int FLAG_OFF = 9 * PLANE_BYTES;             // the tile's flags follow the planes
  static constexpr int STAGE_BYTES = FLAG_OFF + TW;
  static constexpr int SMEM_BYTES = kStages * STAGE_BYTES;
  static_assert(PLANE_BYTES % 16 == 0 && STAGE_BYTES % 16 == 0, "16-byte aligned stages");
};

// Source row of plane i for output row y: the row the population streams from.
__device__ __forceinline__ int src_row(int i, int y, int ny) {
  const int dy = (i == 2 || i == 5 || i == 6) ? -1 : ((i == 4 || i == 7 || i == 8) ? 1 : 0);
  const int r = y + dy;
  return r < 0 ? ny - 1 : (r >= ny ? 0 : r);
}

// The pairs of plane i for the thread's group from the staged segment `seg` (element e holds cell
// x0t - H + e); j0 is the element of the group's first cell; the plane arrives from x - cx.
template <class S, int V>
struct StagedPairs;

template <>
struct StagedPairs<float, 2> {
  static __device__ __forceinline__ void get(const float* seg, int j0, int cx, int, float2* o) {
    if (cx == 0) {
      o[0] = *reinterpret_cast<const float2*>(seg + j0);
    } else {
      const int j = j0 - cx;
      o[0] = make_float2(seg[j], seg[j + 1]);
    }
  }
};

template <>
struct StagedPairs<float, 4> {
  static __device__ __forceinline__ void get(const float* seg, int j0, int cx, int, float2* o) {
    const float4 v = *reinterpret_cast<const float4*>(seg + j0);   // j0 is a multiple of 4
    if (cx == 0) {
      o[0] = make_float2(v.x, v.y);
      o[1] = make_float2(v.z, v.w);
    } else if (cx > 0) {
      const float l = seg[j0 - 1];
      o[0] = make_float2(l, v.x);
      o[1] = make_float2(v.y, v.z);
    } else {
      const float r = seg[j0 + 4];
      o[0] = make_float2(v.y, v.z);
      o[1] = make_float2(v.w, r);
    }
  }
};

template <class S>
struct StagedPairs<S, 2> {
  // 16-bit formats: the two values of cells j, j + 1 (j = j0 - cx) as one packed word
  static __device__ __forceinline__ void get(const S* seg, int j0, int cx, int i, float2* o) {
    const unsigned* w = reinterpret_cast<const unsigned*>(seg);   // word k holds elements 2k, 2k + 1
    const int k = j0 >> 1;                                        // j0 is even
    unsigned p0;
    if (cx == 0)
      p0 = w[k];
    else if (cx > 0)
      p0 = __byte_perm(w[k - 1], w[k], 0x5432);
    else
      p0 = __byte_perm(w[k], w[k + 1], 0x5432);
    o[0] = Codec16<S>::dec(i, p0);
  }
};

template <class S>
struct StagedPairs<S, 4> {
  // 16-bit formats: the four values of cells j .. j + 3 (j = j0 - cx) as two packed words
  static __device__ __forceinline__ void get(const S* seg, int j0, int cx, int i, float2* o) {
    const unsigned* w = reinterpret_cast<const unsigned*>(seg);   // word k holds elements 2k, 2k + 1
    const int k = j0 >> 1;                                        // j0 is a multiple of 4
    unsigned p0, p1;
    if (cx == 0) {
      const uint2 v = *reinterpret_cast<const uint2*>(w + k);
      p0 = v.x;
      p1 = v.y;
    } else if (cx > 0) {                                          // elements j0 - 1 .. j0 + 2
      const uint2 lo = *reinterpret_cast<const uint2*>(w + k - 2);
      const uint2 hi = *reinterpret_cast<const uint2*>(w + k);
      p0 = __byte_perm(lo.y, hi.x, 0x5432);
      p1 = __byte_perm(hi.x, hi.y, 0x5432);
    } else {                                                      // elements j0 + 1 .. j0 + 4
      const uint2 lo = *reinterpret_cast<const uint2*>(w + k);
      const unsigned nx = w[k + 2];
      p0 = __byte_perm(lo.x, lo.y, 0x5432);
      p1 = __byte_perm(lo.y, nx, 0x5432);
    }
    o[0] = Codec16<S>::dec(i, p0);
    o[1] = Codec16<S>::dec(i, p1);
  }
};

template <class S, int V>
__device__ __forceinline__ void staged_plane(const S* seg, int j0, int cx, int i, float2 (*f)[9]) {
  float2 o[V / 2];
  StagedPairs<S, V>::get(seg, j0, cx, i, o);
#pragma unroll
  for (int p = 0; p < V / 2; ++p) f[p][i] = o[p];
}

// The update of the thread's V cells from a staged tile: the same per-cell operations as
// group_update, with every population and flag read from shared memory.
template <class S, int V, int STAGED>
__device__ __forceinline__ void staged_update(const PairTask& t, const uint8_t* stage, int lane, S* __restrict__ b) {
  using G = Geometry<S, V>;
  using IO = GroupIO<S, V>;
  const int nx = t.nx, y = t.y;
  const int x0 = t.xw + V * lane;
  const bool in = x0 < nx;
  const int c0 = in ? x0 - t.x0t : 0;                       // the group's first cell in the tile
  const unsigned flw = in ? (V == 2 ? (unsigned)*reinterpret_cast<const unsigned short*>(stage + G::FLAG_OFF + c0)
                                    : *reinterpret_cast<const unsigned*>(stage + G::FLAG_OFF + c0))
                          : 0x02020202u;
  int fl[V];
#pragma unroll
  for (int c = 0; c < V; ++c) fl[c] = (int)((flw >> (8 * c)) & 0xffu);
  float2 f[V / 2][9];
  const int j0 = c0 + G::H;
#pragma unroll
  for (int i = 0; i < 9; ++i)
    staged_plane<S, V>(reinterpret_cast<const S*>(stage + i * G::PLANE_BYTES), j0, cx_of(i), i, f);
  int k[V];
  if (STAGED) {
    const unsigned lt = (1u << lane) - 1u;
    int base = t.wfirst;
#pragma unroll
    for (int c = 0; c < V; ++c) base += __popc(__ballot_sync(0xffffffffu, in && fl[c] == 1) & lt);
#pragma unroll
    for (int c = 0; c < V; ++c) {
      k[c] = base;
      base += fl[c] == 1 ? 1 : 0;
    }
#pragma unroll
    for (int c = 0; c < V; ++c) {
      if (in && fl[c] == 1 && k[c] < t.kend) {
        const int2 dsc = __ldg(t.bdesc + k[c]);
#pragma unroll
        for (int d = 1; d < 9; ++d) {
          const int j = opp_of(d);
          if ((dsc.y >> j) & 1) cell_of(f, c, d) = __ldg(t.lb + dsc.x + __popc((unsigned)dsc.y & ((1u << j) - 1u)));
        }
      }
    }
  }
  if (!in) return;
  float2 rho[V / 2];
#pragma unroll
  for (int p = 0; p < V / 2; ++p) rho[p] = t.ck == 0 ? collide_bgk_n(f[p], t.op) : collide_trt_n(f[p], t.op, t.om);
  const unsigned idx = (unsigned)(y * nx + x0);
  const unsigned ns = t.ns;
  bool all = true, any = false;
#pragma unroll
  for (int c = 0; c < V; ++c) {
    all = all && fl[c] <= STAGED;
    any = any || fl[c] <= STAGED;
  }
  if (Saturates<S>::value) {
    bool bad = false;
#pragma unroll
    for (int c = 0; c < V; ++c) {
      const float r = (c & 1) ? rho[c >> 1].y : rho[c >> 1].x;
      bad = bad || (fl[c] <= STAGED && !(fabsf(r - 1.0f) < 0.5f));
    }
    if (bad) mark_diverged(t.bad, t.bad_t, t.t_now);
  }
  if (all) {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      float2 g[V / 2];
#pragma unroll
      for (int p = 0; p < V / 2; ++p) g[p] = f[p][i];
      IO::st(b + (unsigned)i * ns + idx, IO::enc(i, g));
    }
  } else if (any) {
#pragma unroll
    for (int c = 0; c < V; ++c) {
      if (fl[c] > STAGED) continue;
#pragma unroll
      for (int i = 0; i < 9; ++i) Store<S>::st(b + (unsigned)i * ns + idx + (unsigned)c, i, cell_of(f, c, i));
    }
  }
  if (STAGED) {
    S* __restrict__ oc = (S*)t.ownc;
#pragma unroll
    for (int c = 0; c < V; ++c) {
      if (fl[c] == 1 && k[c] < t.kend) {
#pragma unroll
        for (int i = 0; i < 9; ++i) Store<S>::st(oc + (unsigned)i * t.nbs + (unsigned)k[c], i, cell_of(f, c, i));
      }
    }
  }
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
        const bool first = x0 == 0, last = x0 + G::TW >= nx;
        const uint32_t bytes = (uint32_t)(end - start) * (uint32_t)sizeof(S);
        const uint32_t fbytes = (uint32_t)(min(x0 + G::TW, nx) - x0);
        const uint32_t wrap = (first ? 16u : 0u) + (last ? 16u : 0u);
        stream::bar_expect_tx(&full[s], 9u * (bytes + wrap) + fbytes);
        uint8_t* stage = smem + (size_t)s * G::STAGE_BYTES;
#pragma unroll 1
        for (int i = 0; i < 9; ++i) {
          const S* row = a + (size_t)i * p.ns + (size_t)stream::src_row(i, y, ny) * nx;
          S* seg = reinterpret_cast<S*>(stage + i * G::PLANE_BYTES);
          stream::copy_g2s(seg + (start - x0 + G::H), row + start, bytes, &full[s]);
          // the periodic wrap: the halo beyond the row's ends holds the other end of the row
          if (first) stream::copy_g2s(seg, row + (nx - G::H), 16u, &full[s]);
          if (last) stream::copy_g2s(seg + (nx - x0 + G::H), row, 16u, &full[s]);
        }
        stream::copy_g2s(stage + G::FLAG_OFF, p.flag + (size_t)y * nx + x0, fbytes, &full[s]);
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
      t.wfirst = (STAGED && t.xw < nx)
                     ? __ldg(p.warp_bfirst + (size_t)t.y * (size_t)(p.tiles_per_row * (kBlock / 32)) + (t.xw >> 5))
                     : 0;
      if (t.xw < nx) stream::staged_update<S, V, STAGED>(t, smem + (size_t)s * G::STAGE_BYTES, lane, b);
      __syncwarp();
      if (lane == 0) stream::bar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && failed) mark_diverged(&p.ctl->nonfinite, &p.ctl->nonfinite_t, &p.ctl->t);
}

}  // namespace vl
