// The multi-cell bulk kernels of the narrow storage formats (FP32 and 16-bit populations).
//
// Each thread updates V neighbouring cells of a row (V = 2 or 4), x0 = V * (thread of the row tile)
// .. x0 + V - 1, so that every population plane is read and written as one vector per thread (8 or
// 16 bytes for FP32, 4 or 8 for the 16-bit formats), and the collision runs on packed FP32 pairs
// (vl_narrow.cuh). A warp covers 32 V cells of one row; a block of kBlock threads kBlock V cells.
//
// Pull (src/sim.rs:700-735): the planes that stream along y only (0, 2, 4) are the vector at x0 of
// the row above, the row itself or the row below. The planes that arrive from x - 1 (1, 5, 8) need
// the cells x0 - 1 .. x0 + V - 2: the last value of the neighbouring lane's vector (a warp shuffle)
// and the first V - 1 of the thread's own; lane 0 reads its x0 - 1 from memory (wrapping to nx - 1
// at the row start). The planes from x + 1 (3, 6, 7) need x0 + 1 .. x0 + V likewise, lane 31 and the
// row's last group reading x0 + V from memory (wrapping to 0). The row length must be a multiple of
// V (every group starts on a multiple of V, so every vector is aligned); other rows use a smaller V
// or the one-cell kernel.
//
// STAGED = 1 (the staged step) also updates the boundary cells, exactly as the one-cell kernel
// does: a cell's rank in the boundary-node list is its warp's first rank (the table the one-cell
// kernel uses, indexed by the warp's first 32-cell slot) plus the boundary cells before it in the
// warp (one ballot per cell position of the group), and its links' returning populations replace
// the pulled ones.
#pragma once

#include <cuda_fp16.h>

#include "vl_device.cuh"
#include "vl_narrow.cuh"

namespace vl {

// ------------------------------------------------------------------ 16-bit pair codecs
// A 32-bit word holds two cells' 16-bit values (the first cell in the low half).
template <class S>
struct Codec16;

// IEEE half of f_i - w_i (the shifted form): a pair is one __half2.
template <>
struct Codec16<__half> {
  static __device__ __forceinline__ float2 dec(int i, unsigned w) {
    __half2 h;
    *reinterpret_cast<unsigned*>(&h) = w;
    const float2 v = __half22float2(h);
    const float wi = wgt<float>(i);
    return __fadd2_rn(v, make_float2(wi, wi));
  }
  static __device__ __forceinline__ unsigned enc(int i, float2 f) {
    const float wi = wgt<float>(i);
    const __half2 h = __float22half2_rn(__fadd2_rn(f, make_float2(-wi, -wi)));
    return *reinterpret_cast<const unsigned*>(&h);
  }
};

// The custom 16-bit format (c16, vl_device.cuh): the two codes of a word decode to FP32 bit
// patterns scaled by 2^-118, and one packed fused multiply-add scales them back and adds w_i; the
// encoding is the packed fused multiply-add that subtracts w_i and scales, then the rounding of each
// FP32 bit pattern to a 16-bit code.
template <>
struct Codec16<c16> {
  static __device__ __forceinline__ float2 dec(int i, unsigned w) {
    const float2 x = make_float2(__uint_as_float(c16f::lo_bits(w)), __uint_as_float(c16f::hi_bits(w)));
    const float wi = wgt<float>(i);
    return __ffma2_rn(x, make_float2(c16f::kUp, c16f::kUp), make_float2(wi, wi));
  }
  static __device__ __forceinline__ unsigned enc(int i, float2 f) {
    const float sw = -wgt<float>(i) * c16f::kDown;
    const float2 y = __ffma2_rn(f, make_float2(c16f::kDown, c16f::kDown), make_float2(sw, sw));
    return c16f::code(__float_as_uint(y.x)) | (c16f::code(__float_as_uint(y.y)) << 16);
  }
};

// The 16-bit fixed-point format (q16, vl_device.cuh): the two codes of a word convert to FP32
// exactly and one packed fused multiply-add scales them and adds w_i; encoding is the packed fused
// multiply-add that scales and subtracts w_i, then a saturating conversion of each to int16.
template <>
struct Codec16<q16> {
  static __device__ __forceinline__ float2 dec(int i, unsigned w) {
    const float2 x = make_float2((float)(int)(short)(w & 0xffffu), (float)((int)w >> 16));
    const float d = q16f::down(i), wi = wgt<float>(i);
    return __ffma2_rn(x, make_float2(d, d), make_float2(wi, wi));
  }
  static __device__ __forceinline__ unsigned enc(int i, float2 f) {
    const float u = q16f::up(i), sw = -wgt<float>(i) * u;
    const float2 y = __ffma2_rn(f, make_float2(u, u), make_float2(sw, sw));
    return ((unsigned)q16f::code(y.x) & 0xffffu) | ((unsigned)q16f::code(y.y) << 16);
  }
};

// ------------------------------------------------------------------ vector access per format
// `Word` holds a thread's V stored values; dec / left / right give the V / 2 FP32 pairs of the
// aligned group, of the group shifted one cell left (x0 - 1 ..) and one cell right (x0 + 1 ..);
// `edge` selects the value at `ep` instead of the neighbouring lane's.
template <class S, int V>
struct GroupIO;

template <>
struct GroupIO<float, 2> {
  using Word = float2;
  template <bool SM>
  static __device__ __forceinline__ Word ld(const float* p) {
#ifdef VL_LD_L2_256B
    if (!SM) {
      float2 w;
      asm("ld.global.nc.L2::256B.v2.f32 {%0, %1}, [%2];" : "=f"(w.x), "=f"(w.y) : "l"(p));
      return w;
    }
#endif
    return SM ? *reinterpret_cast<const float2*>(p) : __ldg(reinterpret_cast<const float2*>(p));
  }
  static __device__ __forceinline__ void st(float* p, Word w) { *reinterpret_cast<float2*>(p) = w; }
  static __device__ __forceinline__ void dec(int, Word w, float2* o) { o[0] = w; }
  static __device__ __forceinline__ void left(int, Word v, bool edge, const float* ep, float2* o) {
    float up = __shfl_up_sync(0xffffffffu, v.y, 1);
    if (edge) up = *ep;
    o[0] = make_float2(up, v.x);
  }
  static __device__ __forceinline__ void right(int, Word v, bool edge, const float* ep, float2* o) {
    float dn = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (edge) dn = *ep;
    o[0] = make_float2(v.y, dn);
  }
  static __device__ __forceinline__ Word enc(int, const float2* f) { return f[0]; }
};

template <>
struct GroupIO<float, 4> {
  using Word = float4;
  template <bool SM>
  static __device__ __forceinline__ Word ld(const float* p) {
    return SM ? *reinterpret_cast<const float4*>(p) : __ldg(reinterpret_cast<const float4*>(p));
  }
  static __device__ __forceinline__ void st(float* p, Word w) { *reinterpret_cast<float4*>(p) = w; }
  static __device__ __forceinline__ void dec(int, Word w, float2* o) {
    o[0] = make_float2(w.x, w.y);
    o[1] = make_float2(w.z, w.w);
  }
  static __device__ __forceinline__ void left(int, Word v, bool edge, const float* ep, float2* o) {
    float up = __shfl_up_sync(0xffffffffu, v.w, 1);
    if (edge) up = *ep;
    o[0] = make_float2(up, v.x);
    o[1] = make_float2(v.y, v.z);
  }
  static __device__ __forceinline__ void right(int, Word v, bool edge, const float* ep, float2* o) {
    float dn = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (edge) dn = *ep;
    o[0] = make_float2(v.y, v.z);
    o[1] = make_float2(v.w, dn);
  }
  static __device__ __forceinline__ Word enc(int, const float2* f) { return make_float4(f[0].x, f[0].y, f[1].x, f[1].y); }
};

// One stored 16-bit value (a generic load: the pointer may be in global or shared memory).
template <class S>
__device__ __forceinline__ unsigned ld16(const S* p) {
  return (unsigned)*reinterpret_cast<const unsigned short*>(p);
}

template <class S>
struct GroupIO<S, 2> {
  using Word = unsigned;
  using C = Codec16<S>;
  template <bool SM>
  static __device__ __forceinline__ Word ld(const S* p) {
    return SM ? *reinterpret_cast<const unsigned*>(p) : __ldg(reinterpret_cast<const unsigned*>(p));
  }
  static __device__ __forceinline__ void st(S* p, Word w) { *reinterpret_cast<unsigned*>(p) = w; }
  static __device__ __forceinline__ void dec(int i, Word w, float2* o) { o[0] = C::dec(i, w); }
  // low half: the previous lane's high half (or the value at `ep`); high half: the own low half
  static __device__ __forceinline__ void left(int i, Word v, bool edge, const S* ep, float2* o) {
    unsigned up = __shfl_up_sync(0xffffffffu, v, 1);
    if (edge) up = ld16(ep) << 16;
    o[0] = C::dec(i, __byte_perm(up, v, 0x5432));
  }
  // low half: the own high half; high half: the next lane's low half (or the value at `ep`)
  static __device__ __forceinline__ void right(int i, Word v, bool edge, const S* ep, float2* o) {
    unsigned dn = __shfl_down_sync(0xffffffffu, v, 1);
    if (edge) dn = ld16(ep);
    o[0] = C::dec(i, __byte_perm(v, dn, 0x5432));
  }
  static __device__ __forceinline__ Word enc(int i, const float2* f) { return C::enc(i, f[0]); }
};

template <class S>
struct GroupIO<S, 4> {
  using Word = uint2;
  using C = Codec16<S>;
  template <bool SM>
  static __device__ __forceinline__ Word ld(const S* p) {
    return SM ? *reinterpret_cast<const uint2*>(p) : __ldg(reinterpret_cast<const uint2*>(p));
  }
  static __device__ __forceinline__ void st(S* p, Word w) { *reinterpret_cast<uint2*>(p) = w; }
  static __device__ __forceinline__ void dec(int i, Word w, float2* o) {
    o[0] = C::dec(i, w.x);
    o[1] = C::dec(i, w.y);
  }
  static __device__ __forceinline__ void left(int i, Word v, bool edge, const S* ep, float2* o) {
    unsigned up = __shfl_up_sync(0xffffffffu, v.y, 1);
    if (edge) up = ld16(ep) << 16;
    o[0] = C::dec(i, __byte_perm(up, v.x, 0x5432));
    o[1] = C::dec(i, __byte_perm(v.x, v.y, 0x5432));
  }
  static __device__ __forceinline__ void right(int i, Word v, bool edge, const S* ep, float2* o) {
    unsigned dn = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (edge) dn = ld16(ep);
    o[0] = C::dec(i, __byte_perm(v.x, v.y, 0x5432));
    o[1] = C::dec(i, __byte_perm(v.y, dn, 0x5432));
  }
  static __device__ __forceinline__ Word enc(int i, const float2* f) { return make_uint2(C::enc(i, f[0]), C::enc(i, f[1])); }
};

// The flags of a thread's V cells, one per byte.
template <int V>
__device__ __forceinline__ unsigned ld_flags(const uint8_t* p) {
  if (V == 2) return (unsigned)__ldg(reinterpret_cast<const unsigned short*>(p));
  return __ldg(reinterpret_cast<const unsigned*>(p));
}

// One warp's share of a row: the group x0 .. x0 + V - 1 of every lane, x0 = t.xw + V * lane.
struct PairTask {
  int nx, ny, y, xw;            // grid, row, the warp's first cell (xw < nx)
  unsigned ns;                  // plane stride
  const uint8_t* flag;          // the domain's flags
  int ck;                       // 0 BGK, 1 TRT
  float op, om;
  // STAGED: the CSR rank of the warp's first boundary cell, the end of the valid ranks, the node
  // descriptors, the per-link returning populations and the compact copy of the boundary nodes'
  // populations (9 planes of stride nbs)
  int wfirst, kend;
  const int2* bdesc;
  const float* lb;
  void* ownc;
  unsigned nbs;
  // saturating formats: the run's divergence flag, the step it records, and the current step
  int* bad;
  unsigned long long* bad_t;
  const unsigned long long* t_now;
  // shared-memory sources (bulk-copy fed kernel): plane i of the row is at stage + i * seg, its
  // element 0 holding cell x0t - halo
  const void* stage;
  int seg, x0t, halo;
};

// The pull of plane i for the thread's group: `src` is where the source row's values are read
// (global memory, or a shared-memory copy indexed by the same x), `grow` the source row in global
// memory (read at the periodic wrap).
template <class S, int V, int SHIFT, bool SM>
__device__ __forceinline__ void pull_group(const S* __restrict__ src, const S* __restrict__ grow, int i, int x0, int xl,
                                           int nx, int lane, bool in, float2 (*f)[9]) {
  using IO = GroupIO<S, V>;
  float2 o[V / 2];
  const typename IO::Word v = IO::template ld<SM>(src + xl);
  if (SHIFT == 0)
    IO::dec(i, v, o);
  else if (SHIFT < 0)
    IO::left(i, v, lane == 0, x0 == 0 ? grow + (nx - 1) : src + (x0 - 1), o);
  else
    IO::right(i, v, in && (lane == 31 || x0 + V >= nx), x0 + V >= nx ? grow : src + (x0 + V), o);
#pragma unroll
  for (int p = 0; p < V / 2; ++p) f[p][i] = o[p];
}

__device__ __forceinline__ float& cell_of(float2 (*f)[9], int c, int i) {
  return (c & 1) ? f[c >> 1][i].y : f[c >> 1][i].x;
}

template <class S, int V, int STAGED, bool SM = false>
__device__ __forceinline__ void group_update(const PairTask& t, const S* __restrict__ a, S* __restrict__ b) {
  using IO = GroupIO<S, V>;
  const int nx = t.nx, ny = t.ny, y = t.y;
  const int lane = (int)(threadIdx.x & 31u);
  const int x0 = t.xw + V * lane;
  const bool in = x0 < nx;
  const int xl = in ? x0 : nx - V;
  const int ym = y == 0 ? ny - 1 : y - 1;
  const int yp = y == ny - 1 ? 0 : y + 1;
  const unsigned ns = t.ns;
  const unsigned rc = (unsigned)(y * nx), rm = (unsigned)(ym * nx), rp = (unsigned)(yp * nx);
  const unsigned flw = in ? ld_flags<V>(t.flag + rc + x0) : 0x02020202u;
  int fl[V];
#pragma unroll
  for (int c = 0; c < V; ++c) fl[c] = (int)((flw >> (8 * c)) & 0xffu);
  float2 f[V / 2][9];
  const S* g[9] = {a + rc, a + 1u * ns + rc, a + 2u * ns + rm, a + 3u * ns + rc, a + 4u * ns + rp,
                   a + 5u * ns + rm, a + 6u * ns + rm, a + 7u * ns + rp, a + 8u * ns + rp};
  const S* sr[9];
#pragma unroll
  for (int i = 0; i < 9; ++i)
    sr[i] = SM ? (const S*)t.stage + (i * t.seg + t.halo - t.x0t) : g[i];
  pull_group<S, V, 0, SM>(sr[0], g[0], 0, x0, xl, nx, lane, in, f);
  pull_group<S, V, -1, SM>(sr[1], g[1], 1, x0, xl, nx, lane, in, f);
  pull_group<S, V, 0, SM>(sr[2], g[2], 2, x0, xl, nx, lane, in, f);
  pull_group<S, V, 1, SM>(sr[3], g[3], 3, x0, xl, nx, lane, in, f);
  pull_group<S, V, 0, SM>(sr[4], g[4], 4, x0, xl, nx, lane, in, f);
  pull_group<S, V, -1, SM>(sr[5], g[5], 5, x0, xl, nx, lane, in, f);
  pull_group<S, V, 1, SM>(sr[6], g[6], 6, x0, xl, nx, lane, in, f);
  pull_group<S, V, 1, SM>(sr[7], g[7], 7, x0, xl, nx, lane, in, f);
  pull_group<S, V, -1, SM>(sr[8], g[8], 8, x0, xl, nx, lane, in, f);
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
  const unsigned idx = rc + (unsigned)x0;
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

// Resident blocks per SM the register allocation targets: 16-bit storage 5 (V = 2) or 3 (V = 4);
// FP32 5 (V = 2: 48 registers, no spills; 4 blocks measured 0.2 % slower, 6 blocks spill and ran
// 2 % slower) or 2 (its V = 4 threads keep 144 bytes of loads in flight each).
#ifndef VL_F32_PAIR_MIN_BLOCKS
#define VL_F32_PAIR_MIN_BLOCKS 5
#endif
template <class S, int V>
constexpr int group_min_blocks() {
  return sizeof(S) == 4 ? (V == 2 ? VL_F32_PAIR_MIN_BLOCKS : 2) : (V == 2 ? 5 : 3);
}

// One sim: block (t, y) updates the V * kBlock cells of tile t of row y (from p.bulk_b0).
template <class S, int V, int CK, int STAGED>
__global__ void __launch_bounds__(kBlock, group_min_blocks<S, V>()) k_bulkv(const __grid_constant__ StepParams p,
                                                                                  const S* __restrict__ a,
                                                                                  S* __restrict__ b) {
  PairTask t;
  t.nx = p.nx;
  t.ny = p.ny;
  t.y = (int)blockIdx.y + p.bulk_b0;
  t.xw = (int)blockIdx.x * (V * kBlock) + (int)(threadIdx.x >> 5) * (32 * V);
  if (p.prefetch_rows && threadIdx.x == 0) {
    const int yf = t.y + p.prefetch_rows;
    prefetch_tile(a, p.ns, t.nx, t.ny, yf >= t.ny ? yf - t.ny : yf, (int)blockIdx.x * (V * kBlock), V * kBlock);
  }
  if (t.xw >= t.nx) return;   // the whole warp is past the row end
  t.ns = p.ns;
  t.flag = p.flag;
  t.ck = CK;
  t.op = (float)p.op;
  t.om = (float)p.om;
  t.wfirst = STAGED ? __ldg(p.warp_bfirst + (size_t)t.y * (size_t)(p.tiles_per_row * (kBlock / 32)) + (t.xw >> 5)) : 0;
  t.kend = p.nb;
  t.bdesc = p.bdesc;
  t.lb = (const float*)p.lb;
  t.ownc = p.ownc;
  t.nbs = p.nbs;
  t.bad = &p.ctl->nonfinite;
  t.bad_t = &p.ctl->nonfinite_t;
  t.t_now = &p.ctl->t;
  group_update<S, V, STAGED>(t, a, b);
}

}  // namespace vl
