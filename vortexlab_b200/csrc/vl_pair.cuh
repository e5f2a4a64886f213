// The two-cell bulk kernel of the narrow storage formats (FP32 and 16-bit populations).
//
// Each thread updates two neighbouring cells of a row, x0 = 2 * (thread of the row tile) and
// x0 + 1, so that every population plane is read and written as one 8-byte (FP32) or 4-byte
// (16-bit) vector per thread, and the collision runs on packed FP32 pairs (vl_narrow.cuh). A warp
// covers 64 cells of one row; a block of kBlock threads 2 * kBlock cells.
//
// Pull (src/sim.rs:700-735): the planes that stream along y only (0, 2, 4) are the vector at x0 of
// the row above, the row itself or the row below. The planes that arrive from x - 1 (1, 5, 8) need
// the pair (x0 - 1, x0): the second half of the neighbouring lane's vector (a warp shuffle) and the
// first half of the thread's own; lane 0 reads its x0 - 1 from memory (wrapping to nx - 1 at the row
// start). The planes from x + 1 (3, 6, 7) need (x0 + 1, x0 + 2) likewise, lane 31 and the row's last
// pair reading x0 + 2 from memory (wrapping to 0). The row length must be even (every pair starts on
// an even cell index, so every vector is aligned); odd rows use the one-cell kernel.
//
// STAGED = 1 (the staged step) also updates the boundary cells, exactly as the one-cell kernel
// does: a cell's rank in the boundary-node list is its warp's first rank (the table the one-cell
// kernel uses, indexed by the warp's first 32-cell slot) plus the boundary cells before it in the
// warp (two ballots: first cells of the pairs, second cells), and its links' returning populations
// replace the pulled ones.
#pragma once

#include <cuda_fp16.h>

#include "vl_device.cuh"
#include "vl_narrow.cuh"

namespace vl {

// Vector access to the stored populations of a pair of cells, per storage format. `Word` is the
// stored pair (8 bytes for FP32, 4 for 16-bit formats); `Elem` one stored value.
template <class S>
struct PairIO;

template <>
struct PairIO<float> {
  using Word = float2;
  using Elem = float;
  static __device__ __forceinline__ Word ld(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
  static __device__ __forceinline__ Elem ld1(const float* p) { return __ldg(p); }
  static __device__ __forceinline__ void st(float* p, Word w) { *reinterpret_cast<float2*>(p) = w; }
  // (x0 - 1, x0): the previous lane's second value, or at `edge` the value at `ep`
  static __device__ __forceinline__ Word left(Word v, bool edge, const float* ep) {
    float up = __shfl_up_sync(0xffffffffu, v.y, 1);
    if (edge) up = __ldg(ep);
    return make_float2(up, v.x);
  }
  // (x0 + 1, x0 + 2): the next lane's first value, or at `edge` the value at `ep`
  static __device__ __forceinline__ Word right(Word v, bool edge, const float* ep) {
    float dn = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (edge) dn = __ldg(ep);
    return make_float2(v.y, dn);
  }
  static __device__ __forceinline__ float2 dec(int, Word w) { return w; }
  static __device__ __forceinline__ Word enc(int, float2 f) { return f; }
};

// The word moves of the 16-bit formats: a pair is one 32-bit word, the first cell in the low half.
template <class S>
struct PairIO16 {
  using Word = unsigned;
  using Elem = unsigned;   // the 16-bit value in the low half
  static __device__ __forceinline__ Word ld(const S* p) { return __ldg(reinterpret_cast<const unsigned*>(p)); }
  static __device__ __forceinline__ Elem ld1(const S* p) {
    return (unsigned)__ldg(reinterpret_cast<const unsigned short*>(p));
  }
  static __device__ __forceinline__ void st(S* p, Word w) { *reinterpret_cast<unsigned*>(p) = w; }
  // the low half of the result is the previous lane's high half (or the value at `ep`), the high
  // half the thread's low half
  static __device__ __forceinline__ Word left(Word v, bool edge, const S* ep) {
    unsigned up = __shfl_up_sync(0xffffffffu, v, 1);
    if (edge) up = ld1(ep) << 16;
    return __byte_perm(up, v, 0x5432);
  }
  // the low half is the thread's high half, the high half the next lane's low half (or `ep`)
  static __device__ __forceinline__ Word right(Word v, bool edge, const S* ep) {
    unsigned dn = __shfl_down_sync(0xffffffffu, v, 1);
    if (edge) dn = ld1(ep);
    return __byte_perm(v, dn, 0x5432);
  }
};

// IEEE half of f_i - w_i (the shifted form): a pair is one __half2.
template <>
struct PairIO<__half> : PairIO16<__half> {
  static __device__ __forceinline__ float2 dec(int i, Word w) {
    __half2 h;
    *reinterpret_cast<unsigned*>(&h) = w;
    const float2 v = __half22float2(h);
    const float wi = wgt<float>(i);
    return __fadd2_rn(v, make_float2(wi, wi));
  }
  static __device__ __forceinline__ Word enc(int i, float2 f) {
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
struct PairIO<c16> : PairIO16<c16> {
  static __device__ __forceinline__ float2 dec(int i, Word w) {
    const float2 x = make_float2(__uint_as_float(c16f::lo_bits(w)), __uint_as_float(c16f::hi_bits(w)));
    const float wi = wgt<float>(i);
    return __ffma2_rn(x, make_float2(c16f::kUp, c16f::kUp), make_float2(wi, wi));
  }
  static __device__ __forceinline__ Word enc(int i, float2 f) {
    const float sw = -wgt<float>(i) * c16f::kDown;
    const float2 y = __ffma2_rn(f, make_float2(c16f::kDown, c16f::kDown), make_float2(sw, sw));
    return c16f::code(__float_as_uint(y.x)) | (c16f::code(__float_as_uint(y.y)) << 16);
  }
};

// The pull of one plane for the pair (x0, x0 + 1) of a row. `row` points at the plane's row the
// population streams from; SHIFT = -1 the population arrives from x - 1, +1 from x + 1, 0 along y.
// `xl` is x0 clamped into the row (lanes past the row end load a valid pair and discard it).
template <class S, int SHIFT>
__device__ __forceinline__ float2 pull_pair(const S* __restrict__ row, int i, int x0, int xl, int nx, int lane,
                                            bool in) {
  using IO = PairIO<S>;
  const typename IO::Word v = IO::ld(row + xl);
  if (SHIFT == 0) return IO::dec(i, v);
  if (SHIFT < 0) return IO::dec(i, IO::left(v, lane == 0, row + (x0 == 0 ? nx - 1 : x0 - 1)));
  return IO::dec(i, IO::right(v, in && (lane == 31 || x0 + 2 >= nx), row + (x0 + 2 >= nx ? 0 : x0 + 2)));
}

// One warp's share of a row: the pair (x0, x0 + 1) of every lane, x0 = t.xw + 2 * lane.
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
};

template <class S, int STAGED>
__device__ __forceinline__ void pair_update(const PairTask& t, const S* __restrict__ a, S* __restrict__ b) {
  using IO = PairIO<S>;
  const int nx = t.nx, ny = t.ny, y = t.y;
  const int lane = (int)(threadIdx.x & 31u);
  const int x0 = t.xw + 2 * lane;
  const bool in = x0 < nx;
  const int xl = in ? x0 : nx - 2;
  const int ym = y == 0 ? ny - 1 : y - 1;
  const int yp = y == ny - 1 ? 0 : y + 1;
  const unsigned ns = t.ns;
  const unsigned rc = (unsigned)(y * nx), rm = (unsigned)(ym * nx), rp = (unsigned)(yp * nx);
  const unsigned short fl2 =
      in ? __ldg(reinterpret_cast<const unsigned short*>(t.flag + rc + x0)) : (unsigned short)0x0202;
  const int fl0 = fl2 & 0xff, fl1 = fl2 >> 8;
  float2 f[9];
  f[0] = pull_pair<S, 0>(a + rc, 0, x0, xl, nx, lane, in);
  f[1] = pull_pair<S, -1>(a + 1u * ns + rc, 1, x0, xl, nx, lane, in);
  f[2] = pull_pair<S, 0>(a + 2u * ns + rm, 2, x0, xl, nx, lane, in);
  f[3] = pull_pair<S, 1>(a + 3u * ns + rc, 3, x0, xl, nx, lane, in);
  f[4] = pull_pair<S, 0>(a + 4u * ns + rp, 4, x0, xl, nx, lane, in);
  f[5] = pull_pair<S, -1>(a + 5u * ns + rm, 5, x0, xl, nx, lane, in);
  f[6] = pull_pair<S, 1>(a + 6u * ns + rm, 6, x0, xl, nx, lane, in);
  f[7] = pull_pair<S, 1>(a + 7u * ns + rp, 7, x0, xl, nx, lane, in);
  f[8] = pull_pair<S, -1>(a + 8u * ns + rp, 8, x0, xl, nx, lane, in);
  int k0 = -1, k1 = -1;
  if (STAGED) {
    const unsigned b0 = __ballot_sync(0xffffffffu, in && fl0 == 1);
    const unsigned b1 = __ballot_sync(0xffffffffu, in && fl1 == 1);
    const unsigned lt = (1u << lane) - 1u;
    k0 = t.wfirst + __popc(b0 & lt) + __popc(b1 & lt);
    k1 = k0 + (fl0 == 1 ? 1 : 0);
    if (in && fl0 == 1 && k0 < t.kend) {
      const int2 dsc = __ldg(t.bdesc + k0);
#pragma unroll
      for (int d = 1; d < 9; ++d) {
        const int j = opp_of(d);
        if ((dsc.y >> j) & 1) f[d].x = __ldg(t.lb + dsc.x + __popc((unsigned)dsc.y & ((1u << j) - 1u)));
      }
    }
    if (in && fl1 == 1 && k1 < t.kend) {
      const int2 dsc = __ldg(t.bdesc + k1);
#pragma unroll
      for (int d = 1; d < 9; ++d) {
        const int j = opp_of(d);
        if ((dsc.y >> j) & 1) f[d].y = __ldg(t.lb + dsc.x + __popc((unsigned)dsc.y & ((1u << j) - 1u)));
      }
    }
  }
  if (!in) return;
  const float2 rho = t.ck == 0 ? collide_bgk_n(f, t.op) : collide_trt_n(f, t.op, t.om);
  const unsigned idx = rc + (unsigned)x0;
  const bool s0 = fl0 <= STAGED, s1 = fl1 <= STAGED;
  if (Saturates<S>::value) {
    const bool ok0 = fabsf(rho.x - 1.0f) < 0.5f, ok1 = fabsf(rho.y - 1.0f) < 0.5f;
    if ((s0 && !ok0) || (s1 && !ok1)) mark_diverged(t.bad, t.bad_t, t.t_now);
  }
  if (s0 && s1) {
#pragma unroll
    for (int i = 0; i < 9; ++i) IO::st(b + (unsigned)i * ns + idx, IO::enc(i, f[i]));
  } else if (s0 || s1) {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const float v = s0 ? f[i].x : f[i].y;
      Store<S>::st(b + (unsigned)i * ns + idx + (s0 ? 0u : 1u), i, v);
    }
  }
  if (STAGED) {
    S* __restrict__ oc = (S*)t.ownc;
    if (fl0 == 1 && k0 < t.kend) {
#pragma unroll
      for (int i = 0; i < 9; ++i) Store<S>::st(oc + (unsigned)i * t.nbs + (unsigned)k0, i, f[i].x);
    }
    if (fl1 == 1 && k1 < t.kend) {
#pragma unroll
      for (int i = 0; i < 9; ++i) Store<S>::st(oc + (unsigned)i * t.nbs + (unsigned)k1, i, f[i].y);
    }
  }
}

// One sim: block (t, y) updates the 2 * kBlock cells of tile t of row y (from p.bulk_b0).
#ifndef VL_PAIR_MIN_BLOCKS
#define VL_PAIR_MIN_BLOCKS 5
#endif
template <class S, int CK, int STAGED>
__global__ void __launch_bounds__(kBlock, VL_PAIR_MIN_BLOCKS) k_bulk2(const __grid_constant__ StepParams p, const S* __restrict__ a,
                                                  S* __restrict__ b) {
  PairTask t;
  t.nx = p.nx;
  t.ny = p.ny;
  t.y = (int)blockIdx.y + p.bulk_b0;
  t.xw = (int)blockIdx.x * (2 * kBlock) + (int)(threadIdx.x >> 5) * 64;
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
  pair_update<S, STAGED>(t, a, b);
}

}  // namespace vl
