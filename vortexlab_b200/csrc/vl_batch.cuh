// Batched step kernels: many tunnels (channels) of uneven sizes advanced together, one launch per
// kernel per step over the work of every active tunnel.
//
// All tunnels live in one arena: each tunnel's nine population planes are contiguous at its own
// offset in the two population buffers, its cells at its own offset in the flag array, and its
// boundary nodes, links and outlet nodes are concatenated into shared tables (link indices are
// global; cell indices stay local to the tunnel). A bulk work item is a tile of a tunnel: either
// 2^log2_tx cells (times the cells per thread) x ty rows, or, in the packed layout, 8 consecutive
// warp segments (32 x cells-per-thread cells of a row each) in the row-major segment order of the
// tunnel, so a tile may end in one row and go on in the next and only the last segment of each row
// can be partly past the row end. A link work item is a chunk of up to kBlock boundary nodes of a
// tunnel. The last chunk of a tunnel to finish a step runs that tunnel's epilogue (force reduction
// in the same fixed order as a single sim, force record, t + 1). The per-node arithmetic is the
// single-sim code (pull, link_node, collide), so a tunnel in a batch is bit-identical to the same
// tunnel run alone (FP64: the reference's operation order, no contraction; the narrow formats: the
// explicitly rounded FP32 operators every narrow kernel shares).
//
// The staged pairing works as for a single sim: k_batch_links<S, 1> evaluates the link rules of
// every chunk into the per-link array, then k_batch_bulk<S, 1> updates every fluid cell of its
// tiles, boundary cells included, and refreshes the compact copy of the boundary nodes' own
// populations. A warp of a tile (tiles are at least 32 cells wide) covers one 32-cell row segment,
// whose first boundary-node rank comes from the per-tunnel segment table.
#pragma once

#include "vl_device.cuh"
#include "vl_pair.cuh"

namespace vl {

struct BatchTunnel {
  int nx, ny;
  unsigned ns;                  // population plane stride of this tunnel
  int coll;                     // COLL_BGK or COLL_TRT
  unsigned long long pop_off;   // element offset of the tunnel's plane 0 in each population buffer
  unsigned long long cell_off;  // offset of the tunnel's cells in the flag array
  int b_off, nb;                // boundary nodes (global index of the first, count)
  int p_off, np;                // outlet nodes
  int chunk_off, nchunks;       // link chunks
  int seg_off, segs;            // staged step: first entry and row length (ceil(nx / 32)) in the segment table
  double op, om;
  double u_ref;
  int absorbing;
  int pad;
  unsigned long long sched_off, sched_len;
  unsigned long long steps;     // steps to run
  unsigned long long hist_off;  // first force record (2 doubles per step)
};

struct BatchState {
  unsigned long long t;
  unsigned long long nonfinite_t;
  unsigned int arrive;
  int nonfinite;
  double drho;                  // the outlet offset of the last step (an observable)
  double drho_now;              // the outlet offset of the step being taken (k_batch_outlet)
  double force[2];
};

struct BatchParams {
  const BatchTunnel* tun;
  BatchState* st;
  const int4* tiles;            // (tunnel, y0, x0, -); packed layout: (tunnel, first segment, 0, -)
  int log2_tx, ty;
  int packed;                   // tiles are 8 consecutive warp segments of a tunnel
  const int4* chunks;           // (tunnel, first boundary node, count, global chunk index)
  const int* outl;              // active tunnels with an absorbing outlet
  int noutl;
  const uint8_t* flag;
  const int32_t* bnode_idx;     // cell index local to the tunnel
  const int32_t* bnode_first;   // global link index; total_nb + 1 entries
  const void* links;
  const int32_t* pnode_idx;     // local cell index
  const int8_t* pnode_n;
  const double* sched;          // per tunnel: 2 doubles per step
  double* partials;             // 2 doubles per chunk
  double* hist;                 // 2 doubles per recorded step
  double sqrt_cs2;
  int dry;                      // timing runs: commit nothing
  // Staged step only (global boundary-node and link indices): per node {first link, link-direction
  // mask}; per 32-cell row segment of each tunnel, the boundary nodes before it; the population each
  // link returns into the fluid (arithmetic type); the nodes' own populations (stored type, 9 planes
  // of stride nbs).
  const int2* bdesc;
  const int32_t* seg_bfirst;
  void* lb;
  void* ownc;
  unsigned nbs;
  // narrow storage with every row length even: the bulk kernel is the two-cell form and a tile is
  // 2 * 2^log2_tx cells wide
  int pairs;
  int ntiles;                   // tiles in the list
  int prefetch_tiles;           // a bulk block prefetches into the L2 the tile this far ahead (0: none)
};

// Packed layout: row and first cell of warp segment `w` of tile `td` (segments of `seg` cells;
// a row holds ceil(nx / seg) of them). Past the tunnel's last segment y comes out >= ny.
__device__ __forceinline__ void packed_seg(const int4& td, int nx, int seg, int w, int& y, int& x0) {
  const int nseg = (nx + seg - 1) / seg;
  const int g = td.y + w;
  y = g / nseg;
  x0 = (g - y * nseg) * seg;
}

// Threads of a bulk block ask the L2 for the rows of tile `k` of the list (one plane row each);
// `width`: the tile's width in cells, or in the packed layout the segment's.
template <class S>
__device__ __forceinline__ void batch_prefetch(const BatchParams& p, const S* A, int k, int width) {
  // packed layout: the tile's 8 segments are one stretch of the tunnel's rows laid end to end, so
  // they cover contiguous spans of at most three rows where a row holds 4 or more segments (the
  // spans of any further rows are not asked for: this is a hint)
  const int rows = p.packed ? 3 : p.ty;
  if (k >= p.ntiles || (int)threadIdx.x >= 9 * rows) return;
  const int4 td = __ldg(p.tiles + k);
  const BatchTunnel& T = p.tun[td.x];
  const int i = (int)threadIdx.x % 9, j = (int)threadIdx.x / 9;
  int y = td.y + j, x0 = td.z, end = x0 + width;
  if (p.packed) {
    int y0, xf, yl, xl;
    packed_seg(td, T.nx, width, 0, y0, xf);
    packed_seg(td, T.nx, width, kBlock / 32 - 1, yl, xl);
    y = y0 + j;
    if (y > yl) return;
    x0 = j == 0 ? xf : 0;
    end = y == yl ? xl + width : T.nx;
  }
  if (y >= T.ny) return;
  const int ym = y == 0 ? T.ny - 1 : y - 1, yp = y == T.ny - 1 ? 0 : y + 1;
  const int r = (i == 2 || i == 5 || i == 6) ? ym : ((i == 4 || i == 7 || i == 8) ? yp : y);
  end = min(end, T.nx);
  if (end <= x0) return;
  prefetch_l2(A + T.pop_off + (size_t)i * T.ns + (size_t)r * T.nx + x0, (size_t)(end - x0) * sizeof(S));
}

// Controls of a tunnel at its step t (src/cases/channel.rs:118-130).
__device__ __forceinline__ void tunnel_controls(const BatchParams& p, const BatchTunnel& T, unsigned long long t,
                                                double* vs, double& target) {
  double v1 = 1.0, v2 = 0.0;
  if (t < T.sched_len) {
    v1 = p.sched[T.sched_off + 2 * t];
    v2 = p.sched[T.sched_off + 2 * t + 1];
  }
  vs[0] = 1.0;
  vs[1] = v1;
  vs[2] = v2;
  vs[3] = 1.0;
  target = T.u_ref * v1;
}

template <class S, int STAGED>
__global__ void __launch_bounds__(kBlock) k_batch_bulk(const __grid_constant__ BatchParams p, const S* __restrict__ A,
                                                       S* __restrict__ B) {
  using R = typename Store<S>::R;
  // Only tunnels that are active for the whole launch are in the tile list (the host rebuilds it
  // when a tunnel finishes), so the tile never checks the tunnel's t, which the link kernel's
  // epilogue may advance concurrently.
  if (p.prefetch_tiles) batch_prefetch(p, A, (int)blockIdx.x + p.prefetch_tiles, p.packed ? 32 : 1 << p.log2_tx);
  const int4 td = __ldg(p.tiles + blockIdx.x);
  const BatchTunnel& T = p.tun[td.x];
  const int nx = T.nx, ny = T.ny;
  int x, y;
  if (p.packed) {
    packed_seg(td, nx, 32, (int)(threadIdx.x >> 5), y, x);
    x += (int)(threadIdx.x & 31u);
  } else {
    x = td.z + (int)(threadIdx.x & ((1u << p.log2_tx) - 1u));
    y = td.y + (int)(threadIdx.x >> p.log2_tx);
  }
  const bool in = x < nx && y < ny;
  if (!STAGED && !in) return;
  const S* a = A + T.pop_off;
  S* b = B + T.pop_off;
  const unsigned idx = (unsigned)(y * nx + x);
  int gfirst = 0;
  if (STAGED && in) gfirst = __ldg(p.seg_bfirst + T.seg_off + y * T.segs + (x >> 5));
  const uint8_t fl = in ? __ldg(p.flag + T.cell_off + idx) : (uint8_t)2;
  R f[9];
  if (in) pull(a, T.ns, nx, ny, x, y, f);
  int g = -1;
  if (STAGED) {
    const unsigned bal = __ballot_sync(0xffffffffu, fl == 1);
    if (!in) return;
    g = gfirst + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u));
    if (fl == 1 && g < T.b_off + T.nb) {
      const int2 dsc = __ldg(p.bdesc + g);
      const R* __restrict__ lb = (const R*)p.lb;
#pragma unroll
      for (int d = 1; d < 9; ++d) {
        const int j = opp_of(d);
        if ((dsc.y >> j) & 1) f[d] = __ldg(lb + dsc.x + __popc((unsigned)dsc.y & ((1u << j) - 1u)));
      }
    }
  }
  collide_s<S>(f, T.coll == COLL_BGK ? 0 : 1, (R)T.op, (R)T.om, R(0), R(0));
  if (fl > (STAGED ? 1 : 0)) return;
  if (Saturates<S>::value && !density_plausible(f))
    mark_diverged(&p.st[td.x].nonfinite, &p.st[td.x].nonfinite_t, &p.st[td.x].t);
#pragma unroll
  for (int i = 0; i < 9; ++i) Store<S>::st(b + (unsigned)i * T.ns + idx, i, f[i]);
  if (STAGED && fl == 1 && g < T.b_off + T.nb) {
    S* __restrict__ oc = (S*)p.ownc;
#pragma unroll
    for (int i = 0; i < 9; ++i) Store<S>::st(oc + (unsigned)i * p.nbs + (unsigned)g, i, f[i]);
  }
}

// The two-cell form of k_batch_bulk for narrow storage (every tunnel's row length even): a tile is
// 2 * 2^log2_tx cells x ty rows, thread t of the tile updates the pair at 2 (t mod 2^log2_tx) of
// row t / 2^log2_tx; a warp covers 64 cells of one row (2^log2_tx >= 32).
// Resident blocks per SM the two-cell batch kernel is compiled for: FP32 5 (48 registers, a few
// spilled; left to itself the compiler takes 76-80 registers, 3 blocks per SM, and the batch
// streams 13 % slower), 16-bit 4.
#ifndef VL_BATCH_PAIR_MIN_BLOCKS
#define VL_BATCH_PAIR_MIN_BLOCKS 5
#endif
template <class S>
constexpr int batch_pair_min_blocks() {
  return sizeof(S) == 4 ? VL_BATCH_PAIR_MIN_BLOCKS : 4;
}
template <class S, int STAGED>
__global__ void __launch_bounds__(kBlock, batch_pair_min_blocks<S>()) k_batch_bulk2(const __grid_constant__ BatchParams p, const S* __restrict__ A,
                                                        S* __restrict__ B) {
  if (p.prefetch_tiles) batch_prefetch(p, A, (int)blockIdx.x + p.prefetch_tiles, p.packed ? 64 : 2 << p.log2_tx);
  const int4 td = __ldg(p.tiles + blockIdx.x);
  const BatchTunnel& T = p.tun[td.x];
  PairTask t;
  t.nx = T.nx;
  t.ny = T.ny;
  if (p.packed) {
    packed_seg(td, t.nx, 64, (int)(threadIdx.x >> 5), t.y, t.xw);
  } else {
    t.y = td.y + (int)(threadIdx.x >> p.log2_tx);
    t.xw = td.z + 2 * (int)((threadIdx.x & ((1u << p.log2_tx) - 1u)) & ~31u);
  }
  if (t.y >= t.ny || t.xw >= t.nx) return;   // uniform over the warp
  t.ns = T.ns;
  t.flag = p.flag + T.cell_off;
  t.ck = T.coll == COLL_BGK ? 0 : 1;
  t.op = (float)T.op;
  t.om = (float)T.om;
  t.wfirst = STAGED ? __ldg(p.seg_bfirst + T.seg_off + t.y * T.segs + (t.xw >> 5)) : 0;
  t.kend = T.b_off + T.nb;
  t.bdesc = p.bdesc;
  t.lb = (const float*)p.lb;
  t.ownc = p.ownc;
  t.nbs = p.nbs;
  t.bad = &p.st[td.x].nonfinite;
  t.bad_t = &p.st[td.x].nonfinite_t;
  t.t_now = &p.st[td.x].t;
  group_update<S, 2, STAGED>(t, A + T.pop_off, B + T.pop_off);
}

// STAGED = 1: the link rules only (k_links_stage for a chunk): own populations from the compact
// copy, the returning populations to the per-link array, no pull, collision or store.
// The outlet density offset of each active absorbing tunnel at its current step, once per tunnel
// (src/sim.rs:425-440; the sequential sum in outlet-node order of the reference), for every link
// chunk of that tunnel to read; launched on the link kernel's stream just before it.
template <class S>
__global__ void __launch_bounds__(kBlock) k_batch_outlet(const __grid_constant__ BatchParams p, const S* __restrict__ A) {
  __shared__ double s_un[kBlock];
  const int k = __ldg(p.outl + blockIdx.x);
  const BatchTunnel& T = p.tun[k];
  BatchState* st = &p.st[k];
  const unsigned long long t = st->t;
  if (t >= T.steps) return;
  double vs[4], target;
  tunnel_controls(p, T, t, vs, target);
  const double drho = outlet_offset(A + T.pop_off, T.ns, p.pnode_idx + T.p_off, p.pnode_n + 2 * T.p_off, T.np, 0.0,
                                    0.0, target, p.sqrt_cs2, s_un);
  if (threadIdx.x == 0) st->drho_now = drho;
}

template <class S, int STAGED>
__global__ void __launch_bounds__(kBlock) k_batch_links(const __grid_constant__ BatchParams p, const S* __restrict__ A,
                                                        S* __restrict__ B) {
  using R = typename Store<S>::R;
  __shared__ double s_acc[2][kBlock];
  __shared__ double red[kBlock];
  __shared__ int last;
  const int tid = threadIdx.x;
  const int4 cd = __ldg(p.chunks + blockIdx.x);
  const BatchTunnel& T = p.tun[cd.x];
  BatchState* st = &p.st[cd.x];
  const unsigned long long t = st->t;
  if (t >= T.steps) return;
  const S* a = A + T.pop_off;
  S* b = B + T.pop_off;
  double vs[4], target;
  tunnel_controls(p, T, t, vs, target);
  const double drho = (T.absorbing && T.np > 0) ? st->drho_now : 0.0;   // k_batch_outlet, just before
  if (cd.w == T.chunk_off && tid == 0 && !p.dry) st->drho = drho;
  s_acc[0][tid] = 0.0;
  s_acc[1][tid] = 0.0;
  if (tid < cd.z && STAGED) {
    const int g = cd.y + tid;
    const S* __restrict__ oc = (const S*)p.ownc;
    R own[9];
#pragma unroll
    for (int d = 0; d < 9; ++d) own[d] = Store<S>::ld(oc + (unsigned)d * p.nbs + (unsigned)g, d);
    R* __restrict__ lb = (R*)p.lb;
    link_rules<S>(a, T.ns, own, __ldg(p.bnode_first + g), __ldg(p.bnode_first + g + 1), (const LinkRecDev*)p.links,
                  vs, drho, 0.0, 0.0, p.sqrt_cs2, &s_acc[0][tid], [&](int l, int, R back) { lb[l] = back; });
  } else if (tid < cd.z) {
    const int g = cd.y + tid;
    const int idx = __ldg(p.bnode_idx + g);
    R f[9];
    link_node<S>(a, T.ns, T.nx, T.ny, idx, __ldg(p.bnode_first + g), __ldg(p.bnode_first + g + 1),
                 (const LinkRecDev*)p.links, vs, drho, T.coll, T.op, T.om, 0.0, 0.0, p.sqrt_cs2, &s_acc[0][tid], f);
#pragma unroll
    for (int i = 0; i < 9; ++i) Store<S>::st(b + (unsigned)i * T.ns + idx, i, f[i]);
  }
  __syncthreads();
  block_force_partial(s_acc, 2, p.partials + 2 * (size_t)cd.w);
  // The last chunk of this tunnel reduces the tunnel's partials and advances its step.
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    last = atomicAdd(&st->arrive, 1u) == (unsigned)(T.nchunks - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double fx = sum_partials(p.partials + 2 * (size_t)T.chunk_off, T.nchunks, 2, red);
  const double fy = sum_partials(p.partials + 2 * (size_t)T.chunk_off + 1, T.nchunks, 2, red);
  if (tid == 0) {
    if (!p.dry) {
      st->force[0] = fx;
      st->force[1] = fy;
      if (!(isfinite(fx) && isfinite(fy)) && !st->nonfinite) {
        st->nonfinite = 1;
        st->nonfinite_t = t;
      }
      p.hist[2 * (T.hist_off + t)] = fx;
      p.hist[2 * (T.hist_off + t) + 1] = fy;
      st->t = t + 1;
    }
    st->arrive = 0;
    __threadfence();
  }
}

// The compact copy of the boundary nodes' own populations of the chunks' tunnels, gathered from
// `a` (one block per link chunk).
template <class S>
__global__ void __launch_bounds__(kBlock) k_batch_gather_own(const __grid_constant__ BatchParams p, const S* __restrict__ A) {
  const int4 cd = __ldg(p.chunks + blockIdx.x);
  if ((int)threadIdx.x >= cd.z) return;
  const BatchTunnel& T = p.tun[cd.x];
  const int g = cd.y + (int)threadIdx.x;
  const unsigned idx = (unsigned)__ldg(p.bnode_idx + g);
  const S* a = A + T.pop_off;
  S* oc = (S*)p.ownc;
#pragma unroll
  for (int d = 0; d < 9; ++d) oc[(unsigned)d * p.nbs + (unsigned)g] = a[(unsigned)d * T.ns + idx];
}

}  // namespace vl
