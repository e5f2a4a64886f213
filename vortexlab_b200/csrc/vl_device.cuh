// Device data structures and the step kernels (templated on storage and arithmetic type).
//
// One time step of the reference (src/sim.rs:391-420) is two kernels that run concurrently
// (a fork/join over two streams, captured into the step graph):
//
//   k_links  boundary nodes: gather the 9 incoming populations, replace every population that
//            would come out of a wall or open boundary with the boundary rule of its link
//            (src/sim.rs:456-507), accumulate the momentum-exchange force per force group,
//            collide, write. One thread per boundary node of the CSR node list.
//   k_bulk   interior nodes (flag 0): pull the 9 populations from the upstream neighbours with
//            periodic wrap (src/sim.rs:700-735), collide, write. One thread per cell; one
//            block per tile of kBlock cells of a row (grid x = tile of the row, y = row).
//
// Both read only `a` and write disjoint cells of `b`, so their order does not matter; the
// whole-step epilogue runs in the last link block to finish (a counter in device memory, no
// spin-waits): it reduces the per-block force partials in a fixed order, writes the per-step
// record, evaluates the pressure-drop probe of the previous step and advances t.
//
// The staged step is the other pairing: k_links_stage applies the link rules only (one thread per
// link) and writes the population each link returns into the fluid to a compact array (link
// order); then k_bulk<S, CK, 1> updates every fluid cell of its row tiles, boundary cells included, taking
// those populations in place of the pulled ones, and also writes the new populations of each
// boundary node to a compact copy in CSR order, which the next k_links_stage reads instead of
// `a`. The boundary cells then cost coalesced traffic instead of nine scattered 32-byte sectors
// per store, per pull and per own value; the two kernels must run in that order. Both pairings
// compute every population with the same expressions (the staged step sums the force terms per
// block of links rather than per node, a different fixed order: equal to rounding).
//
// Determinism: every population update is a pure function of `a`; the force is summed per thread
// in link order, then by a fixed warp-shuffle tree, a fixed shared-memory tree and a fixed tree
// over block partials, so runs are bit-identical run to run. The outlet density offset
// (src/sim.rs:444-455) is a sequential sum in pnode order, as in the reference.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

#include "vl_lattice.hpp"
#include "vl_narrow.cuh"

namespace vl {

constexpr int kBlock = 256;       // threads per block for both step kernels
constexpr int kMaxGroups = 4;     // force groups
constexpr int kRec = 10;          // doubles per history record
constexpr int kProbeCorners = 24; // 2 wall points x 3 distances x 4 cells

// Device-resident control block of one sim. Written by the host between batches (stream-ordered
// copies) and by the step epilogue.
struct Ctl {
  double vscale[4];
  double target;
  double drho;                 // outlet density offset used in the last step
  double force[2 * kMaxGroups];
  unsigned long long t;
  unsigned long long rec_start;  // t of history record 0
  unsigned long long rec_cap;    // records available (0 = not recording)
  unsigned long long nonfinite_t;
  unsigned int arrive;         // blocks of the current step that have finished
  int has_target;
  int nonfinite;               // set once a non-finite force is seen
  int sched_on;                // channel mode: controls from the schedule below
  int dry;                     // timing runs: the epilogue commits nothing (no t, force or history)
  int absorbing;
  int dp_on;
  double u_ref;
  unsigned long long sched_len;
  const double* sched;         // [sched_len][2] = (inlet ramp, body kick) per step
  double* hist;                // [rec_cap][kRec]
  // pressure-drop probe: per (side, distance) the valid corner cells and bilinear weights
  int probe_idx[kProbeCorners];  // -1: corner skipped (outside, solid or zero weight)
  double probe_w[kProbeCorners];
};

struct StepParams {
  int nx, ny;
  unsigned ns;                 // population plane stride (elements)
  int tiles_per_row, ntiles;   // bulk tiling: one tile = kBlock consecutive cells of a row
  int nbulk, nlink;            // bulk tiles and link blocks of a step
  int coll, forced;
  double op, om, gx, gy;
  double sqrt_cs2;
  const uint8_t* flag;
  const int32_t* bnode_idx;
  const int32_t* bnode_first;  // nb + 1 entries
  int nb;
  const void* links;           // LinkRecDev[]
  const int32_t* pnode_idx;
  const int8_t* pnode_n;       // (nx, ny) pairs
  int np;
  Ctl* ctl;
  double* partials;            // [nlink][2 * kMaxGroups]
  int ngroups;
  // Staged step only: per boundary node (CSR order) {first link, bit j set for each link
  // direction j}; per 32-cell warp slot of the bulk grid, the boundary nodes before its first cell;
  // the population each link sends back into the fluid (arithmetic type, link order); the
  // boundary nodes' own populations of the current state (stored type, 9 planes of stride nbs, CSR
  // order), written by the staged bulk kernel beside `b` for the next step.
  const int2* bdesc;
  const int32_t* warp_bfirst;
  void* lb;
  void* ownc;
  unsigned nbs;
  // Staged link kernel: one thread per link, nlinkblk blocks of kBlock links; lnode[l] = boundary
  // node (CSR index) of link l. Launch ranges (a step may launch each kernel in two parts): link
  // blocks [link_b0, link_b0 + link_n) and bulk rows [bulk_b0, bulk_b0 + bulk_n), clipped.
  const int32_t* lnode;
  int nlinks, nlinkblk;
  int link_b0, link_n, bulk_b0, bulk_n;
  // narrow storage: the most cells of a row the bulk kernel's threads update (1, 2 or 4; fewer
  // where the row length is not a multiple, one with a body force)
  int pairs;
  // narrow storage: 1 = the bulk kernel reads the populations through bulk copies into shared
  // memory where the rows allow it (vl_stream.cuh), 0 = directly
  int stream;
  // rows ahead whose tile a block of the bulk kernel asks the L2 to fetch (0: none)
  int prefetch_rows;
};

// Asks the L2 to fetch (bulk prefetch: no registers or shared memory held; later loads then hit the
// L2) the whole 16-byte units inside [p, p + bytes).
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
  const uintptr_t b0 = ((uintptr_t)p + 15u) & ~(uintptr_t)15u;
  const uintptr_t b1 = ((uintptr_t)p + bytes) & ~(uintptr_t)15u;
  if (b1 > b0)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b0), "r"((unsigned)(b1 - b0)) : "memory");
}

// The nine plane rows that the tile of `cells` cells at x0 of output row `y` reads, prefetched
// into the L2 by one thread of a bulk-kernel block some rows ahead of its own.
template <class S>
__device__ __forceinline__ void prefetch_tile(const S* a, unsigned ns, int nx, int ny, int y, int x0, int cells) {
  const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
  const int end = min(x0 + cells, nx);
  if (end <= x0) return;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int r = (i == 2 || i == 5 || i == 6) ? ym : ((i == 4 || i == 7 || i == 8) ? yp : y);
    prefetch_l2(a + (size_t)i * ns + (size_t)r * nx + x0, (size_t)(end - x0) * sizeof(S));
  }
}

struct alignas(16) LinkRecDev {
  double q, cu6, uw0, uw1, rho;
  int32_t behind;
  uint8_t dir, flags, vgroup;
  int8_t fgroup;
};
static_assert(sizeof(LinkRecDev) == 48, "link record");

// ------------------------------------------------------------------ storage traits
// S = stored type, R = arithmetic type. FP16 storage keeps f_i - w_i (the shifted form), which
// centres the stored values on zero and keeps the half-precision mantissa for the deviation from
// the rest state.
template <class S>
struct Store;

template <>
struct Store<double> {
  using R = double;
  static __device__ __forceinline__ double ld(const double* p, int) { return __ldg(p); }
  static __device__ __forceinline__ double ld_cg(const double* p, int) { return __ldcg(p); }
  static __device__ __forceinline__ void st(double* p, int, double v) { *p = v; }
};

template <>
struct Store<float> {
  using R = float;
  static __device__ __forceinline__ float ld(const float* p, int) { return __ldg(p); }
  static __device__ __forceinline__ float ld_cg(const float* p, int) { return __ldcg(p); }
  static __device__ __forceinline__ void st(float* p, int, float v) { *p = v; }
};

template <>
struct Store<__half> {
  using R = float;
  static __device__ __forceinline__ float ld(const __half* p, int i) {
    return wgt<float>(i) + __half2float(__ldg(p));
  }
  static __device__ __forceinline__ float ld_cg(const __half* p, int i) {
    return wgt<float>(i) + __half2float(__ldcg(p));
  }
  static __device__ __forceinline__ void st(__half* p, int i, float v) { *p = __float2half_rn(v - wgt<float>(i)); }
};

// 16-bit storage of f_i - w_i with more precision where the shifted populations live: sign, a
// 3-bit exponent e and a 12-bit mantissa m; the value is 2^(e-9) (1 + m / 4096) for e >= 1 and
// m 2^-20 for e = 0 (evenly spaced below 2^-8), largest magnitude 2^-2 (2 - 2^-12) = 0.49994.
// IEEE half keeps 10 mantissa bits over 2^-14..65504; the shifted populations of a low-Mach flow
// stay within +-0.1, so the two exponent bits spent on that range buy two mantissa bits here: the
// step at 0.0167 (w_1 3 u at u = 0.05) is 3.8e-6 instead of 1.5e-5. Conversion: the shifted value
// is scaled by 2^-118 in one rounded FP32 fused multiply-add, so that the format's exponents are
// the FP32 exponents 0..7 (its evenly spaced range the FP32 subnormals), and its FP32 bit pattern
// is rounded to 12 mantissa bits (to nearest, ties to even) and clamped to the largest magnitude;
// decoding shifts the bits back and scales by 2^118 in the fused multiply-add that adds w_i. Values
// beyond the range saturate (a cell whose density leaves 1 +- 1/2 marks the run as diverged).
struct c16 {
  unsigned short bits;
};

namespace c16f {
constexpr float kUp = 0x1p118f;
constexpr float kDown = 0x1p-118f;
constexpr unsigned kMaxBits = 0x03fff800u;   // FP32 bits of the largest magnitude times 2^-118
// FP32 bits (times 2^-118) of a code in the low 16 bits of `c`
__device__ __forceinline__ unsigned lo_bits(unsigned c) { return ((c & 0x7fffu) << 11) | ((c & 0x8000u) << 16); }
// the same for a code in the high 16 bits
__device__ __forceinline__ unsigned hi_bits(unsigned c) { return ((c >> 5) & 0x03fff800u) | (c & 0x80000000u); }
// the code of the FP32 bits `b` of a shifted value times 2^-118
__device__ __forceinline__ unsigned code(unsigned b) {
  unsigned mag = min(b & 0x7fffffffu, kMaxBits);
  mag = (mag + 0x3ffu + ((mag >> 11) & 1u)) >> 11;
  return mag | ((b >> 16) & 0x8000u);
}
__device__ __forceinline__ float dec(unsigned c, int i) {
  return __fmaf_rn(__uint_as_float(lo_bits(c)), kUp, wgt<float>(i));
}
__device__ __forceinline__ unsigned enc(float v, int i) {
  return code(__float_as_uint(__fmaf_rn(v, kDown, -wgt<float>(i) * kDown)));
}
}  // namespace c16f

template <>
struct Store<c16> {
  using R = float;
  static __device__ __forceinline__ float ld(const c16* p, int i) {
    return c16f::dec(__ldg(reinterpret_cast<const unsigned short*>(p)), i);
  }
  static __device__ __forceinline__ float ld_cg(const c16* p, int i) {
    return c16f::dec(__ldcg(reinterpret_cast<const unsigned short*>(p)), i);
  }
  static __device__ __forceinline__ void st(c16* p, int i, float v) {
    reinterpret_cast<unsigned short*>(p)[0] = (unsigned short)c16f::enc(v, i);
  }
};

// 16-bit fixed point of f_i - w_i: the shifted value in steps of 2^-19 for the rest population and
// the diagonals and 2^-18 for the axis directions (the axis populations carry 3 u_i / 9, the largest
// shifted values of a low-Mach flow), rounded to nearest (ties to even) and clamped to the 16-bit
// range (+-0.0625 / +-0.125). Uniform absolute steps, as fine as the custom format's where the
// populations live (1.9e-6 / 3.8e-6), with conversions the hardware does in one instruction each:
// encode = one fused multiply-add (scale and subtract w_i) and a saturating float-to-int16
// conversion; decode = an int16-to-float conversion and one fused multiply-add that adds w_i.
struct q16 {
  short bits;
};

namespace q16f {
__host__ __device__ constexpr float up(int i) { return (i >= 1 && i <= 4) ? 0x1p18f : 0x1p19f; }
__host__ __device__ constexpr float down(int i) { return (i >= 1 && i <= 4) ? 0x1p-18f : 0x1p-19f; }
__device__ __forceinline__ int code(float y) { return min(max(__float2int_rn(y), -32768), 32767); }
__device__ __forceinline__ float dec(int q, int i) { return __fmaf_rn((float)q, down(i), wgt<float>(i)); }
__device__ __forceinline__ int enc(float v, int i) { return code(__fmaf_rn(v, up(i), -wgt<float>(i) * up(i))); }
}  // namespace q16f

template <>
struct Store<q16> {
  using R = float;
  static __device__ __forceinline__ float ld(const q16* p, int i) {
    return q16f::dec(__ldg(reinterpret_cast<const short*>(p)), i);
  }
  static __device__ __forceinline__ float ld_cg(const q16* p, int i) {
    return q16f::dec(__ldcg(reinterpret_cast<const short*>(p)), i);
  }
  static __device__ __forceinline__ void st(q16* p, int i, float v) {
    reinterpret_cast<short*>(p)[0] = (short)q16f::enc(v, i);
  }
};

// Storage formats that saturate instead of carrying a non-finite value.
template <class S>
struct Saturates {
  static constexpr bool value = false;
};
template <>
struct Saturates<c16> {
  static constexpr bool value = true;
};
template <>
struct Saturates<q16> {
  static constexpr bool value = true;
};

// Marks a run of a saturating storage format as diverged (the first time): a cell whose density
// left 1 +- 1/2, which a finite run at low Mach number never does.
__device__ __forceinline__ void mark_diverged(int* bad, unsigned long long* bad_t, const unsigned long long* t_now) {
  if (atomicCAS(bad, 0, 1) == 0) *bad_t = *t_now;
}

template <class R>
__device__ __forceinline__ bool density_plausible(const R* f) {
  const R r = ((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7])) + f[8];
  return fabsf((float)r - 1.0f) < 0.5f;
}

// ------------------------------------------------------------------ helpers
// The collision of storage S: the reference's operators in its operation order for FP64
// (vl_lattice.hpp), the FP32 operators with explicit multiply-adds for the narrow formats
// (vl_narrow.cuh; the forced collision keeps the generic form). ck: 0 BGK, 1 TRT, 2 forced.
template <class S>
__device__ __forceinline__ void collide_s(typename Store<S>::R* f, int ck, typename Store<S>::R op,
                                          typename Store<S>::R om, typename Store<S>::R gx, typename Store<S>::R gy) {
  if (ck == 2)
    collide_forced(f, op, om, gx, gy);
  else if (ck == 0)
    collide_bgk(f, op);
  else
    collide_trt(f, op, om);
}
template <>
__device__ __forceinline__ void collide_s<float>(float* f, int ck, float op, float om, float gx, float gy) {
  if (ck == 2)
    collide_forced(f, op, om, gx, gy);
  else if (ck == 0)
    collide_bgk_n(f, op);
  else
    collide_trt_n(f, op, om);
}
template <>
__device__ __forceinline__ void collide_s<__half>(float* f, int ck, float op, float om, float gx, float gy) {
  collide_s<float>(f, ck, op, om, gx, gy);
}
template <>
__device__ __forceinline__ void collide_s<c16>(float* f, int ck, float op, float om, float gx, float gy) {
  collide_s<float>(f, ck, op, om, gx, gy);
}
template <>
__device__ __forceinline__ void collide_s<q16>(float* f, int ck, float op, float om, float gx, float gy) {
  collide_s<float>(f, ck, op, om, gx, gy);
}
template <class R>
__device__ __forceinline__ R pick(const R* f, int i) {
  R v = f[0];
#pragma unroll
  for (int d = 1; d < 9; ++d)
    if (d == i) v = f[d];
  return v;
}

template <class R>
__device__ __forceinline__ void set_dir(R* f, int i, R v) {
#pragma unroll
  for (int d = 0; d < 9; ++d)
    if (d == i) f[d] = v;
}

// Per-step controls: in channel mode the inlet ramp and the body kick come from the uploaded
// schedule and the outlet target follows the ramp (src/cases/channel.rs:118-130).
struct Controls {
  double vs[4];
  double target;
  int has_target;
};

__device__ __forceinline__ Controls read_controls(const Ctl* c) {
  Controls k;
  const unsigned long long t = c->t;
#pragma unroll
  for (int g = 0; g < 4; ++g) k.vs[g] = c->vscale[g];
  k.target = c->target;
  k.has_target = c->has_target;
  if (c->sched_on) {
    const double v1 = t < c->sched_len ? c->sched[2 * t] : 1.0;
    const double v2 = t < c->sched_len ? c->sched[2 * t + 1] : 0.0;
    k.vs[1] = v1;
    k.vs[2] = v2;
    k.has_target = c->absorbing;
    k.target = c->u_ref * v1;
  }
  return k;
}

// ------------------------------------------------------------------ epilogue
// Pressure-drop probe (src/cases/cylinder.rs:54-59) of the state `a` recorded as step `tstep`
// of the history: probe_density (src/sim.rs:624-644) at distances 1, 2, 3 from each wall point,
// extrapolated to the wall (src/sim.rs:648-651). Block-wide; every thread must call it.
template <class S>
__device__ void record_probe(const StepParams& p, const S* __restrict__ a, long long tstep) {
  __shared__ double rho_c[kProbeCorners];
  Ctl* c = p.ctl;
  const long long rs = (long long)c->rec_start;
  if (!c->dp_on || !c->rec_cap || tstep < rs || tstep - rs >= (long long)c->rec_cap) return;
  const int tid = threadIdx.x;
  if (tid < kProbeCorners) {
    const int idx = c->probe_idx[tid];
    double r = 0.0;
    if (idx >= 0) {
      double f[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) f[i] = (double)Store<S>::ld_cg(a + (size_t)i * p.ns + idx, i);
      double jx, jy;
      moments(f, r, jx, jy);
    }
    rho_c[tid] = r;
  }
  __syncthreads();
  if (tid == 0) {
    double wall[2];
    for (int side = 0; side < 2; ++side) {
      double pd[3];
      for (int d = 0; d < 3; ++d) {
        double sum = 0.0, wsum = 0.0;
        for (int k = 0; k < 4; ++k) {
          const int s = (side * 3 + d) * 4 + k;
          if (c->probe_idx[s] < 0) continue;
          sum += c->probe_w[s] * rho_c[s];
          wsum += c->probe_w[s];
        }
        pd[d] = wsum > 0.0 ? sum / wsum : __longlong_as_double(0x7ff8000000000000ll);
      }
      wall[side] = 3.0 * pd[0] - 3.0 * pd[1] + pd[2];
    }
    c->hist[(size_t)(tstep - rs) * kRec + 9] = (1.0 / 3.0) * (wall[0] - wall[1]) / (c->u_ref * c->u_ref);
  }
  __syncthreads();
}

// Block-wide sum of `count` values spaced `stride` apart: thread t adds values t, t + kBlock, ...
// in order, then a fixed shared-memory tree. The result is valid in thread 0. Every thread calls it.
__device__ __forceinline__ double sum_partials(const double* v, int count, int stride, double* red) {
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int k = tid; k < count; k += kBlock) acc += __ldcg(v + (size_t)k * stride);
  red[tid] = acc;
  __syncthreads();
  for (int s = kBlock / 2; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  const double out = red[0];
  __syncthreads();
  return out;
}

// Runs in the last link block to finish a step: reduces the force partials in a fixed order,
// writes the step record, evaluates the pressure probe of the previous step (whose result is the
// current `a`), advances the controls and t.
template <class S>
__device__ void step_epilogue(const StepParams& p, const S* __restrict__ a, int nblocks) {
  __shared__ double red[kBlock];
  __shared__ double res[2 * kMaxGroups];
  const int tid = threadIdx.x;
  Ctl* c = p.ctl;
  const int ncomp = 2 * p.ngroups;
  for (int k = 0; k < ncomp; ++k) {
    const double v = sum_partials(p.partials + k, nblocks, 2 * kMaxGroups, red);
    if (tid == 0) res[k] = v;
  }
  __syncthreads();
  const unsigned long long t = c->t;
  const bool commit = !c->dry;
  if (commit) record_probe<S>(p, a, (long long)t - 1);
  if (tid == 0) {
    if (commit) {
      bool finite = true;
      for (int k = 0; k < 2 * kMaxGroups; ++k) {
        const double v = k < ncomp ? res[k] : 0.0;
        c->force[k] = v;
        if (!isfinite(v)) finite = false;
      }
      if (!finite && !c->nonfinite) {
        c->nonfinite = 1;
        c->nonfinite_t = t;
      }
      if (c->rec_cap && t >= c->rec_start && t - c->rec_start < c->rec_cap) {
        double* r = c->hist + (size_t)(t - c->rec_start) * kRec;
        for (int k = 0; k < 2 * kMaxGroups; ++k) r[k] = c->force[k];
        r[8] = c->drho;
        r[9] = 0.0;
      }
      if (c->sched_on) {
        const Controls k = read_controls(c);
        c->vscale[1] = k.vs[1];
        c->vscale[2] = k.vs[2];
        c->target = k.target;
        c->has_target = k.has_target;
      }
      c->t = t + 1;
    }
    c->arrive = 0;
    __threadfence();
  }
}

// Link blocks publish their force partial and count themselves; the last of the step's `nblocks`
// blocks runs the epilogue.
template <class S>
__device__ __forceinline__ void arrive(const StepParams& p, const S* __restrict__ a, int nblocks) {
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&p.ctl->arrive, 1u);
    last = prev == (unsigned)(nblocks - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    step_epilogue<S>(p, a, nblocks);
  }
}

// Records the pressure probe of the last step of a batch (its result is the current `a`).
template <class S>
__global__ void __launch_bounds__(kBlock) k_probe(const __grid_constant__ StepParams p, const S* __restrict__ a) {
  record_probe<S>(p, a, (long long)p.ctl->t - 1);
}

// ------------------------------------------------------------------ bulk kernel
// Pull + collide for the interior nodes. Block (t, y) covers the kBlock consecutive cells of tile t
// of row y. The nine population loads are issued together with the flag load, for every cell of the
// tile (wrap keeps every neighbour index inside the grid), so no load waits for the flag; only
// interior cells (flag 0) store. Boundary cells are written by the link kernel, solid cells never.
template <class S>
__device__ __forceinline__ void pull(const S* __restrict__ a, unsigned ns, int nx, int ny, int x, int y,
                                     typename Store<S>::R* f) {
  const int ym = y == 0 ? ny - 1 : y - 1;
  const int yp = y == ny - 1 ? 0 : y + 1;
  const int xm = x == 0 ? nx - 1 : x - 1;
  const int xp = x == nx - 1 ? 0 : x + 1;
  const unsigned rc = (unsigned)(y * nx), rm = (unsigned)(ym * nx), rp = (unsigned)(yp * nx);
  f[0] = Store<S>::ld(a + rc + x, 0);
  f[1] = Store<S>::ld(a + 1u * ns + rc + xm, 1);
  f[2] = Store<S>::ld(a + 2u * ns + rm + x, 2);
  f[3] = Store<S>::ld(a + 3u * ns + rc + xp, 3);
  f[4] = Store<S>::ld(a + 4u * ns + rp + x, 4);
  f[5] = Store<S>::ld(a + 5u * ns + rm + xm, 5);
  f[6] = Store<S>::ld(a + 6u * ns + rm + xp, 6);
  f[7] = Store<S>::ld(a + 7u * ns + rp + xp, 7);
  f[8] = Store<S>::ld(a + 8u * ns + rp + xm, 8);
}

//
// STAGED = 1 (the staged step): the tile also updates its boundary cells (flag 1). Their pulled
// populations come from the same coalesced row loads; each one that arrives across a link is
// replaced by the value k_links_stage computed for that link, found through the node's descriptor:
// the node's rank k in the CSR list is the warp's first rank plus the boundary cells before the
// lane (a ballot), and the link of direction j is `first + popc(mask below j)` (the links of a node
// are stored by ascending direction). Every fluid cell of the row is then written by this kernel.
template <class S, int CK, int STAGED>
__global__ void __launch_bounds__(kBlock) k_bulk(const __grid_constant__ StepParams p,
                                                 const S* __restrict__ a, S* __restrict__ b) {
  using R = typename Store<S>::R;
  const int nx = p.nx, ny = p.ny;
  // grid: x = tile of the row, y = row (from p.bulk_b0), so blocks run in row-major tile order
  const int y = (int)blockIdx.y + p.bulk_b0;
  const int x = (int)blockIdx.x * kBlock + (int)threadIdx.x;
  const int tile = y * p.tiles_per_row + (int)blockIdx.x;
  if (p.prefetch_rows && threadIdx.x == 0) {
    const int yf = y + p.prefetch_rows;
    prefetch_tile(a, p.ns, nx, ny, yf >= ny ? yf - ny : yf, (int)blockIdx.x * kBlock, kBlock);
  }
  if (!STAGED && x >= nx) return;
  const bool in = x < nx;
  const unsigned idx = (unsigned)(y * nx + x);
  int wfirst = 0;
  if (STAGED) wfirst = __ldg(p.warp_bfirst + (size_t)tile * (kBlock / 32) + (threadIdx.x >> 5));
  const uint8_t fl = in ? __ldg(p.flag + idx) : (uint8_t)2;
  R f[9];
  if (in) pull(a, p.ns, nx, ny, x, y, f);
  int k = -1;
  if (STAGED) {
    const unsigned bal = __ballot_sync(0xffffffffu, fl == 1);
    if (!in) return;
    k = wfirst + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u));
    if (fl == 1 && k < p.nb) {
      const int2 dsc = __ldg(p.bdesc + k);
      const R* __restrict__ lb = (const R*)p.lb;
#pragma unroll
      for (int d = 1; d < 9; ++d) {
        const int j = opp_of(d);
        if ((dsc.y >> j) & 1) f[d] = __ldg(lb + dsc.x + __popc((unsigned)dsc.y & ((1u << j) - 1u)));
      }
    }
  }
  collide_s<S>(f, CK, (R)p.op, (R)p.om, (R)p.gx, (R)p.gy);
  if (fl > (STAGED ? 1 : 0)) return;
  if (Saturates<S>::value && !density_plausible(f)) mark_diverged(&p.ctl->nonfinite, &p.ctl->nonfinite_t, &p.ctl->t);
#pragma unroll
  for (int i = 0; i < 9; ++i) Store<S>::st(b + (unsigned)i * p.ns + idx, i, f[i]);
  if (STAGED && fl == 1 && k < p.nb) {
    S* __restrict__ oc = (S*)p.ownc;
#pragma unroll
    for (int i = 0; i < 9; ++i) Store<S>::st(oc + (unsigned)i * p.nbs + (unsigned)k, i, f[i]);
  }
}

// ------------------------------------------------------------------ link kernel
// One thread per boundary node. The node's link records are read as three 16-byte vectors each;
// the force of each group is accumulated per thread in shared memory (in link order), then
// reduced per block by a fixed tree.
struct LinkView {
  double q, cu6, uw0, uw1, rho;
  int behind, dir, flags, vgroup, fgroup;
};

__device__ __forceinline__ LinkView load_link(const LinkRecDev* links, int l) {
  const int4* v = reinterpret_cast<const int4*>(links + l);
  const int4 w0 = __ldg(v), w1 = __ldg(v + 1), w2 = __ldg(v + 2);
  LinkView L;
  L.q = __hiloint2double(w0.y, w0.x);
  L.cu6 = __hiloint2double(w0.w, w0.z);
  L.uw0 = __hiloint2double(w1.y, w1.x);
  L.uw1 = __hiloint2double(w1.w, w1.z);
  L.rho = __hiloint2double(w2.y, w2.x);
  L.behind = w2.z;
  const unsigned packed = (unsigned)w2.w;  // dir, flags, vgroup, fgroup (little endian)
  L.dir = (int)(packed & 0xffu);
  L.flags = (int)((packed >> 8) & 0xffu);
  L.vgroup = (int)((packed >> 16) & 0xffu);
  L.fgroup = (int)(int8_t)(packed >> 24);
  return L;
}

// Outlet density offset (src/sim.rs:444-455): the velocity of every non-radiating pressure node
// from its own populations in `a`, summed sequentially in pnode order. Block-wide; every thread
// calls it and receives the result.
template <class S>
__device__ double outlet_offset(const S* __restrict__ a, unsigned ns, const int32_t* __restrict__ pnode_idx,
                                const int8_t* __restrict__ pnode_n, int np, double gx, double gy, double target,
                                double sqrt_cs2, double* s_un) {
  __shared__ double s_drho;
  const int tid = threadIdx.x;
  double sum = 0.0;
  for (int base = 0; base < np; base += kBlock) {
    const int k = base + tid;
    if (k < np) {
      const int idx = __ldg(pnode_idx + k);
      double f[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) f[i] = (double)Store<S>::ld(a + (size_t)i * ns + idx, i);
      double rho, jx, jy;
      moments(f, rho, jx, jy);
      const double ux = jx / rho - 0.5 * gx, uy = jy / rho - 0.5 * gy;
      s_un[tid] = (double)pnode_n[2 * k] * ux + (double)pnode_n[2 * k + 1] * uy;
    }
    __syncthreads();
    if (tid == 0) {
      const int m = min(kBlock, np - base);
      for (int q = 0; q < m; ++q) sum += s_un[q];
    }
    __syncthreads();
  }
  if (tid == 0) s_drho = (sum / (double)np - target) / sqrt_cs2;
  __syncthreads();
  return s_drho;
}

// The link rules of one boundary node (src/sim.rs:462-495): for link l with direction j, the
// population `back` that returns into direction i = opp(j) is handed to put(l, i, back), and the
// momentum exchanged with the link's force group is added to `acc` (component c at acc[c * kBlock]).
// Every per-link read of the reference's link pass other than the node behind the link (a[j][idx],
// a[i][idx], the node velocity) is one of the node's own post-collision populations `own`, so the
// loop touches memory only for its record and that one node.
// Whether a link's rule reads the node behind it: a wall link with q < 1/2 and a fluid node
// behind (src/sim.rs:474-477).
__device__ __forceinline__ bool uses_behind(const LinkView& L) {
  return !(L.flags & 1) && L.q < 0.5 && L.behind >= 0;
}

// The returning population of one link. `bval` is a[j][behind] (read by the caller, so that it
// can be loaded together with other links' values; any value when the rule does not use it).
template <class S>
__device__ __forceinline__ typename Store<S>::R link_back(typename Store<S>::R bval, const LinkView& L,
                                                          const typename Store<S>::R* own, const double* vs,
                                                          double drho, typename Store<S>::R gx,
                                                          typename Store<S>::R gy, double sqrt_cs2, bool& have_u,
                                                          typename Store<S>::R& ux, typename Store<S>::R& uy,
                                                          typename Store<S>::R& out, typename Store<S>::R& scale) {
  using R = typename Store<S>::R;
  const int j = L.dir;
  const int i = opp_of(j);
  out = pick(own, j);
  scale = (R)vs[L.vgroup];
  R back;
  if (!(L.flags & 1)) {
    // Wall: interpolated bounce-back with the moving-wall term (src/sim.rs:467-479).
    const R corr = (R)L.cu6 * scale;
    const R q = (R)L.q;
    if (q >= R(0.5)) {
      const R kq = R(0.5) / q;
      back = kq * (out - corr) + (R(1.0) - kq) * pick(own, i);
    } else if (L.behind >= 0) {
      back = R(2.0) * q * out + (R(1.0) - R(2.0) * q) * bval - corr;
    } else {
      back = out - corr;
    }
  } else {
    // Open boundary: anti-bounce-back around the equilibrium of the boundary density
    // (src/sim.rs:480-488), with the node's own velocity.
    if (!have_u) {
      R rho, jx, jy;
      moments(own, rho, jx, jy);
      ux = jx / rho - R(0.5) * gx;
      uy = jy / rho - R(0.5) * gy;
      have_u = true;
    }
    const R cu = R(3.0) * ((R)cx_of(j) * ux + (R)cy_of(j) * uy);
    R rho_w;
    if (L.flags & 2) {
      const R nxv = (R)((int)((L.flags >> 2) & 3) - 1), nyv = (R)((int)((L.flags >> 4) & 3) - 1);
      rho_w = (R)L.rho + (nxv * ux + nyv * uy) / (R)sqrt_cs2;
    } else {
      rho_w = (R)L.rho + (R)drho;
    }
    back = -out + R(2.0) * (R)w_of(j) * rho_w * (R(1.0) + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy));
  }
  return back;
}

// Galilean-invariant momentum exchange of one link (src/sim.rs:490-495), in FP64.
__device__ __forceinline__ void force_terms(const LinkView& L, double o, double bk, double scale, double& tx,
                                            double& ty) {
  const double wux = L.uw0 * scale, wuy = L.uw1 * scale;
  tx = (double)cx_of(L.dir) * (o + bk) - wux * (o - bk);
  ty = (double)cy_of(L.dir) * (o + bk) - wuy * (o - bk);
}

template <class S, class Put>
__device__ __forceinline__ void link_rules(const S* __restrict__ a, unsigned ns, const typename Store<S>::R* own,
                                           int first, int last, const LinkRecDev* __restrict__ links,
                                           const double* vs, double drho, double gx_, double gy_, double sqrt_cs2,
                                           double* acc, Put put) {
  using R = typename Store<S>::R;
  const R gx = (R)gx_, gy = (R)gy_;
  bool have_u = false;
  R ux = R(0), uy = R(0);
  for (int l = first; l < last; ++l) {
    const LinkView L = load_link(links, l);
    R out, scale;
    const R bval = uses_behind(L) ? Store<S>::ld(a + (unsigned)L.dir * ns + (unsigned)L.behind, L.dir) : R(0);
    const R back = link_back<S>(bval, L, own, vs, drho, gx, gy, sqrt_cs2, have_u, ux, uy, out, scale);
    put(l, opp_of(L.dir), back);
    if (L.fgroup >= 0) {
      double tx, ty;
      force_terms(L, (double)out, (double)back, (double)scale, tx, ty);
      acc[(2 * L.fgroup) * kBlock] += tx;
      acc[(2 * L.fgroup + 1) * kBlock] += ty;
    }
  }
}

// The link pass for one boundary node (src/sim.rs:456-503): the incoming populations pulled from
// the neighbours, each one that would come out of the boundary replaced by its link's rule, then
// the collision. `f` returns the post-collision populations.
template <class S>
__device__ __forceinline__ void link_node(const S* __restrict__ a, unsigned ns, int nx, int ny, int idx, int first,
                                          int last, const LinkRecDev* __restrict__ links, const double* vs,
                                          double drho, int ck, double op_, double om_, double gx_, double gy_,
                                          double sqrt_cs2, double* acc, typename Store<S>::R* f) {
  using R = typename Store<S>::R;
  const R op = (R)op_, om = (R)om_, gx = (R)gx_, gy = (R)gy_;
  const int y = idx / nx, x = idx - y * nx;
  R own[9];
  pull(a, ns, nx, ny, x, y, f);
#pragma unroll
  for (int d = 0; d < 9; ++d) own[d] = Store<S>::ld(a + (unsigned)d * ns + idx, d);
  link_rules<S>(a, ns, own, first, last, links, vs, drho, gx_, gy_, sqrt_cs2, acc,
                [&](int, int i, R back) { set_dir(f, i, back); });
  collide_s<S>(f, ck, op, om, gx, gy);
}

// Block partial of the first `ncomp` force components: fixed shuffle tree within each warp, then
// the warps in order. Written by threads 0..ncomp-1 to out[c]. Every thread calls it.
__device__ __forceinline__ void block_force_partial(const double (*s_acc)[kBlock], int ncomp, double* out) {
  __shared__ double s_red[2 * kMaxGroups][kBlock / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c = 0; c < ncomp; ++c) {
    double v = s_acc[c][tid];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) s_red[c][warp] = v;
  }
  __syncthreads();
  if (tid < ncomp) {
    double v = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) v += s_red[tid][w];
    out[tid] = v;
  }
}

#ifndef VL_LINK_MIN_BLOCKS
#define VL_LINK_MIN_BLOCKS 1
#endif
template <class S, int CK>
__global__ void __launch_bounds__(kBlock, VL_LINK_MIN_BLOCKS) k_links(const __grid_constant__ StepParams p,
                                                                    const S* __restrict__ a, S* __restrict__ b) {
  using R = typename Store<S>::R;
  __shared__ double s_un[kBlock];
  __shared__ double s_acc[2 * kMaxGroups][kBlock];
  const int tid = threadIdx.x;
  const Controls ctl = read_controls(p.ctl);
  const double drho = (ctl.has_target && p.np > 0)
                          ? outlet_offset(a, p.ns, p.pnode_idx, p.pnode_n, p.np, p.gx, p.gy, ctl.target, p.sqrt_cs2, s_un)
                          : 0.0;
  if (blockIdx.x == 0 && tid == 0 && !p.ctl->dry) p.ctl->drho = drho;
  const int ncomp = 2 * p.ngroups;
  for (int c = 0; c < ncomp; ++c) s_acc[c][tid] = 0.0;
  const int k = blockIdx.x * kBlock + tid;
  if (k < p.nb) {
    const int idx = __ldg(p.bnode_idx + k);
    R f[9];
    link_node<S>(a, p.ns, p.nx, p.ny, idx, __ldg(p.bnode_first + k), __ldg(p.bnode_first + k + 1),
                 (const LinkRecDev*)p.links, ctl.vs, drho, CK, p.op, p.om, p.gx, p.gy, p.sqrt_cs2, &s_acc[0][tid], f);
#pragma unroll
    for (int i = 0; i < 9; ++i) Store<S>::st(b + (unsigned)i * p.ns + idx, i, f[i]);
  }
  if (ncomp > 0) {
    __syncthreads();
    block_force_partial(s_acc, ncomp, p.partials + (size_t)blockIdx.x * (2 * kMaxGroups));
  }
  arrive<S>(p, a, p.nlink);
}

#ifndef VL_STAGE_PER
#define VL_STAGE_PER 1
#endif
constexpr int kStagePer = VL_STAGE_PER;  // links per thread of k_links_stage

// First kernel of the staged step: the link rules of every link, without the pull, the collision
// or the store (k_bulk<S, CK, 1> does those in its row tiles). kStagePer links per thread (blocks of
// kBlock * kStagePer links, numbered from p.link_b0, p.nlinkblk in all), so each thread's loads
// (record, the node's own populations from the compact copy p.ownc, the node behind) are one short
// chain. Writes
// the returning population of each link to p.lb; the force terms of the block's links go through
// the fixed shuffle / shared-memory tree into the block partial, the last of the p.nlinkblk blocks
// runs the end-of-step epilogue, the outlet offset is computed per block as in k_links.
template <class S>
__global__ void __launch_bounds__(kBlock) k_links_stage(const __grid_constant__ StepParams p, const S* __restrict__ a) {
  using R = typename Store<S>::R;
  __shared__ double s_un[kBlock];
  __shared__ double s_acc[2 * kMaxGroups][kBlock];
  const int tid = threadIdx.x;
  const Controls ctl = read_controls(p.ctl);
  const double drho = (ctl.has_target && p.np > 0)
                          ? outlet_offset(a, p.ns, p.pnode_idx, p.pnode_n, p.np, p.gx, p.gy, ctl.target, p.sqrt_cs2, s_un)
                          : 0.0;
  const int blk = (int)blockIdx.x + p.link_b0;
  if (blk == 0 && tid == 0 && !p.ctl->dry) p.ctl->drho = drho;
  const int ncomp = 2 * p.ngroups;
  for (int c = 0; c < ncomp; ++c) s_acc[c][tid] = 0.0;
  // Links blk * kBlock * kStagePer + tid + m * kBlock (m < kStagePer): every record first, then
  // every value the rules read, then the arithmetic, so the loads of all of a thread's links are in
  // flight together. The thread adds its links' force terms in m order.
  const LinkRecDev* __restrict__ links = (const LinkRecDev*)p.links;
  const S* __restrict__ oc = (const S*)p.ownc;
  const int lbase = blk * kBlock * kStagePer + tid;
  LinkView L[kStagePer];
  unsigned kn[kStagePer];
#pragma unroll
  for (int m = 0; m < kStagePer; ++m) {
    const int l = lbase + m * kBlock;
    if (l < p.nlinks) {
      kn[m] = (unsigned)__ldg(p.lnode + l);
      L[m] = load_link(links, l);
    }
  }
  R vj[kStagePer], vi[kStagePer], bv[kStagePer];
#pragma unroll
  for (int m = 0; m < kStagePer; ++m) {
    const int l = lbase + m * kBlock;
    if (l < p.nlinks) {
      const int j = L[m].dir, i = opp_of(j);
      vj[m] = Store<S>::ld(oc + (unsigned)j * p.nbs + kn[m], j);
      vi[m] = Store<S>::ld(oc + (unsigned)i * p.nbs + kn[m], i);
      bv[m] = uses_behind(L[m]) ? Store<S>::ld(a + (unsigned)j * p.ns + (unsigned)L[m].behind, j) : R(0);
    }
  }
#pragma unroll
  for (int m = 0; m < kStagePer; ++m) {
    const int l = lbase + m * kBlock;
    if (l < p.nlinks) {
      const int j = L[m].dir, i = opp_of(j);
      R own[9];
      if (L[m].flags & 1) {
#pragma unroll
        for (int d = 0; d < 9; ++d) own[d] = Store<S>::ld(oc + (unsigned)d * p.nbs + kn[m], d);
      } else {
#pragma unroll
        for (int d = 0; d < 9; ++d) own[d] = d == j ? vj[m] : (d == i ? vi[m] : R(0));
      }
      bool have_u = false;
      R ux = R(0), uy = R(0), out, scale;
      const R back =
          link_back<S>(bv[m], L[m], own, ctl.vs, drho, (R)p.gx, (R)p.gy, p.sqrt_cs2, have_u, ux, uy, out, scale);
      ((R*)p.lb)[l] = back;
      if (L[m].fgroup >= 0) {
        double tx, ty;
        force_terms(L[m], (double)out, (double)back, (double)scale, tx, ty);
        s_acc[2 * L[m].fgroup][tid] += tx;
        s_acc[2 * L[m].fgroup + 1][tid] += ty;
      }
    }
  }
  if (ncomp > 0) {
    __syncthreads();
    block_force_partial(s_acc, ncomp, p.partials + (size_t)blk * (2 * kMaxGroups));
  }
  arrive<S>(p, a, p.nlinkblk);
}

// The compact copy of the boundary nodes' own populations read by k_links_stage, gathered from `a`
// whenever the state was set other than by a staged step (init, upload, another schedule).
template <class S>
__global__ void k_gather_own(int nb, unsigned ns, unsigned nbs, const int32_t* __restrict__ bidx,
                             const S* __restrict__ a, S* __restrict__ oc) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
    const unsigned idx = (unsigned)__ldg(bidx + k);
#pragma unroll
    for (int d = 0; d < 9; ++d) oc[(unsigned)d * nbs + (unsigned)k] = a[(unsigned)d * ns + idx];
  }
}

// ------------------------------------------------------------------ utility kernels
// Sim::init (src/sim.rs:357-371): equilibrium of a field into both buffers; solids get (1,0,0).
template <class S>
__global__ void k_init(int n, unsigned ns, const uint8_t* __restrict__ flag, const double* __restrict__ rho,
                       const double* __restrict__ ux, const double* __restrict__ uy, double rho0, double ux0,
                       double uy0, S* __restrict__ a, S* __restrict__ b) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    double r = rho0, u = ux0, v = uy0;
    if (flag[idx] == 2) {
      r = 1.0; u = 0.0; v = 0.0;
    } else if (rho) {
      r = rho[idx]; u = ux[idx]; v = uy[idx];
    }
    double feq[9];
    equilibrium(r, u, v, feq);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      Store<S>::st(a + (size_t)i * ns + idx, i, (typename Store<S>::R)feq[i]);
      Store<S>::st(b + (size_t)i * ns + idx, i, (typename Store<S>::R)feq[i]);
    }
  }
}

// Sim::init from fields given on a coarse grid of normalised values (the warm-start network's
// output, FP32 [gh][gw][gc], device memory): lattice cell (x, y) samples the grid bilinearly at
// column (x - x0) / dx - 1/2 and row (y - y0) / dy - 1/2 (cell-centred grid, clamped at its edges),
// and channels 0-2 decode to u_x = u (1 + v0), u_y = u v1, rho = 1 + 1.5 u^2 v2; solids get
// (1, 0, 0). The equilibria go into both buffers.
template <class S>
__global__ void k_init_grid(int nx, int n, unsigned ns, const uint8_t* __restrict__ flag, const float* __restrict__ g,
                            int gh, int gw, int gc, double x0, double dx, double y0, double dy, double u,
                            S* __restrict__ a, S* __restrict__ b) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    double r = 1.0, vx = 0.0, vy = 0.0;
    if (flag[idx] != 2) {
      const int x = idx % nx, y = idx / nx;
      const double gx = ((double)x - x0) / dx - 0.5, gy = ((double)y - y0) / dy - 0.5;
      const int ix = min(max((int)floor(gx), 0), gw - 2), iy = min(max((int)floor(gy), 0), gh - 2);
      const double fx = fmin(fmax(gx - ix, 0.0), 1.0), fy = fmin(fmax(gy - iy, 0.0), 1.0);
      double v[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* p = g + ((size_t)iy * gw + ix) * gc + c;
        const double f00 = p[0], f01 = p[gc], f10 = p[(size_t)gw * gc], f11 = p[(size_t)gw * gc + gc];
        v[c] = (1.0 - fy) * ((1.0 - fx) * f00 + fx * f01) + fy * ((1.0 - fx) * f10 + fx * f11);
      }
      vx = u * (1.0 + v[0]);
      vy = u * v[1];
      r = 1.0 + 1.5 * u * u * v[2];
    }
    double feq[9];
    equilibrium(r, vx, vy, feq);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      Store<S>::st(a + (size_t)i * ns + idx, i, (typename Store<S>::R)feq[i]);
      Store<S>::st(b + (size_t)i * ns + idx, i, (typename Store<S>::R)feq[i]);
    }
  }
}

// Populations to FP64 in the reference layout (plane stride n).
template <class S>
__global__ void k_to_f64(int n, unsigned ns, const S* __restrict__ a, double* __restrict__ out) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
#pragma unroll
    for (int i = 0; i < 9; ++i) out[(size_t)i * n + idx] = (double)Store<S>::ld(a + (size_t)i * ns + idx, i);
  }
}

// FP64 populations (reference layout) into storage S.
template <class S>
__global__ void k_from_f64(int n, unsigned ns, const double* __restrict__ in, S* __restrict__ a) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
#pragma unroll
    for (int i = 0; i < 9; ++i)
      Store<S>::st(a + (size_t)i * ns + idx, i, (typename Store<S>::R)in[(size_t)i * n + idx]);
  }
}

// (rho, ux, uy) of every cell as Sim::macros computes them (src/sim.rs:527-534); solids (1,0,0).
template <class S>
__global__ void k_macros(int n, unsigned ns, const uint8_t* __restrict__ flag, double gx, double gy,
                         const S* __restrict__ a, double* __restrict__ rho, double* __restrict__ ux,
                         double* __restrict__ uy) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    if (flag[idx] == 2) {
      rho[idx] = 1.0; ux[idx] = 0.0; uy[idx] = 0.0;
      continue;
    }
    double f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = (double)Store<S>::ld(a + (size_t)i * ns + idx, i);
    double r, jx, jy;
    moments(f, r, jx, jy);
    rho[idx] = r;
    ux[idx] = jx / r - 0.5 * gx;
    uy[idx] = jy / r - 0.5 * gy;
  }
}

// Deterministic FP64 reductions over fluid cells: per-thread Neumaier sums of mass and the two
// momentum components (src/sim.rs:538-563), then a fixed pairwise tree; plus the largest speed
// with NaN propagation (src/sim.rs:566-579). One block per slot of `out` (4 doubles per block).
__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
  const double t = s + x;
  c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
  s = t;
}

template <class S>
__global__ void __launch_bounds__(kBlock) k_reduce(int n, unsigned ns, const uint8_t* __restrict__ flag,
                                                   double gx, double gy, const S* __restrict__ a,
                                                   double* __restrict__ out) {
  __shared__ double sh[7][kBlock];
  double ms = 0, mc = 0, xs = 0, xc = 0, ys = 0, yc = 0, vmax = 0.0;
  bool nan = false;
  for (int idx = blockIdx.x * kBlock + threadIdx.x; idx < n; idx += gridDim.x * kBlock) {
    if (flag[idx] == 2) continue;
    double f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = (double)Store<S>::ld(a + (size_t)i * ns + idx, i);
#pragma unroll
    for (int i = 0; i < 9; ++i) neumaier_add(ms, mc, f[i]);
#pragma unroll
    for (int i = 1; i < 9; ++i) {
      neumaier_add(xs, xc, (double)cx_of(i) * f[i]);
      neumaier_add(ys, yc, (double)cy_of(i) * f[i]);
    }
    double r, jx, jy;
    moments(f, r, jx, jy);
    const double u = jx / r - 0.5 * gx, v = jy / r - 0.5 * gy;
    const double sp = sqrt(u * u + v * v);
    if (isnan(sp)) nan = true; else vmax = fmax(vmax, sp);
  }
  const int t = threadIdx.x;
  sh[0][t] = ms; sh[1][t] = mc; sh[2][t] = xs; sh[3][t] = xc; sh[4][t] = ys; sh[5][t] = yc;
  sh[6][t] = nan ? __longlong_as_double(0x7ff8000000000000ll) : vmax;
  __syncthreads();
  for (int s = kBlock / 2; s > 0; s >>= 1) {
    if (t < s) {
      for (int k = 0; k < 3; ++k) {
        double s0 = sh[2 * k][t], c0 = sh[2 * k + 1][t];
        neumaier_add(s0, c0, sh[2 * k][t + s]);
        sh[2 * k][t] = s0;
        sh[2 * k + 1][t] = c0 + sh[2 * k + 1][t + s];
      }
      const double o = sh[6][t + s], m = sh[6][t];
      sh[6][t] = (isnan(o) || isnan(m)) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(m, o);
    }
    __syncthreads();
  }
  if (t == 0) {
    double* o = out + 7 * blockIdx.x;
    for (int k = 0; k < 7; ++k) o[k] = sh[k][0];
  }
}

// Gathers the 9 populations (as FP64) of a list of cells.
template <class S>
__global__ void k_gather(int m, unsigned ns, const int32_t* __restrict__ cells, const S* __restrict__ a,
                         double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int idx = cells[k];
#pragma unroll
  for (int i = 0; i < 9; ++i) out[9 * k + i] = (double)Store<S>::ld(a + (size_t)i * ns + idx, i);
}

}  // namespace vl
