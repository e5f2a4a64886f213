// Collision arithmetic of the narrow-storage kernels (FP32 and 16-bit population storage).
//
// The collision runs in FP32 with every rounding spelled out: adds, multiplies and fused
// multiply-adds are the round-to-nearest intrinsics, which the compiler neither contracts nor
// reorders. The operators are written once over V = float (one cell) or float2 (two cells, one
// packed FADD2 / FMUL2 / FFMA2 instruction of Blackwell's FP32 pipe per operation). Each lane of
// the packed form performs exactly the operations of the scalar form, so a cell's new populations
// do not depend on which kernel updated it (the two-cell bulk kernel, the one-cell bulk kernel for
// odd row lengths, the link kernel or the batched kernels).
//
// The physics and the operation sequence follow the reference's operators (src/lattice.rs:59-156:
// moments, second-order equilibrium, BGK, TRT with the rest population relaxed towards
// rho - sum of the moving equilibria); only the association of sums and the fusing of
// multiply-adds differ, which the FP64 path (vl_lattice.hpp) does not allow itself.
#pragma once

#include <cuda_runtime.h>

#include "vl_lattice.hpp"

namespace vl {

template <class V>
struct NOps;

template <>
struct NOps<float> {
  static __device__ __forceinline__ float s(float x) { return x; }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ float rcp(float a) { return __frcp_rn(a); }
  static __device__ __forceinline__ float neg(float a) { return -a; }
};

template <>
struct NOps<float2> {
  static __device__ __forceinline__ float2 s(float x) { return make_float2(x, x); }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
  static __device__ __forceinline__ float2 sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
  static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
  static __device__ __forceinline__ float2 rcp(float2 a) { return make_float2(__frcp_rn(a.x), __frcp_rn(a.y)); }
  static __device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
};

// rho, jx, jy (src/lattice.rs:59-64), summed pairwise.
template <class V>
__device__ __forceinline__ void moments_n(const V* f, V& rho, V& jx, V& jy) {
  using O = NOps<V>;
  const V s13 = O::add(f[1], f[3]), s24 = O::add(f[2], f[4]), s57 = O::add(f[5], f[7]), s68 = O::add(f[6], f[8]);
  rho = O::add(O::add(O::add(f[0], s13), s24), O::add(s57, s68));
  const V d13 = O::sub(f[1], f[3]), d24 = O::sub(f[2], f[4]), d57 = O::sub(f[5], f[7]), d68 = O::sub(f[6], f[8]);
  jx = O::sub(O::add(d13, d57), d68);   // f1 - f3 + f5 - f7 - (f6 - f8)
  jy = O::add(O::add(d24, d57), d68);   // f2 - f4 + f5 - f7 + (f6 - f8)
}

// The shared part of both collisions: rho, the velocity, 3 u, and `base` = 1 - 1.5 |u|^2.
template <class V>
struct NMacro {
  V rho, ux3, uy3, base;
};

template <class V>
__device__ __forceinline__ NMacro<V> macro_n(const V* f) {
  using O = NOps<V>;
  V rho, jx, jy;
  moments_n(f, rho, jx, jy);
  const V inv = O::rcp(rho);
  const V ux = O::mul(jx, inv), uy = O::mul(jy, inv);
  const V usq = O::fma(uy, uy, O::mul(ux, ux));
  NMacro<V> m;
  m.rho = rho;
  m.ux3 = O::mul(O::s(3.0f), ux);
  m.uy3 = O::mul(O::s(3.0f), uy);
  m.base = O::fma(O::s(-1.5f), usq, O::s(1.0f));
  return m;
}

// c.u * 3 of the four directions 1, 2, 5, 6 (their opposites 3, 4, 7, 8 have the negated value).
template <class V>
__device__ __forceinline__ void cu_n(const NMacro<V>& m, V* cu) {
  using O = NOps<V>;
  cu[0] = m.ux3;
  cu[1] = m.uy3;
  cu[2] = O::add(m.ux3, m.uy3);
  cu[3] = O::sub(m.uy3, m.ux3);
}

// BGK (src/lattice.rs:80-95): f_i -= omega (f_i - feq_i); the rest population relaxes towards
// rho - sum of the moving equilibria. Returns rho.
template <class V>
__device__ __forceinline__ V collide_bgk_n(V* f, float omega) {
  using O = NOps<V>;
  const NMacro<V> m = macro_n(f);
  V cu[4];
  cu_n(m, cu);
  const V wr1 = O::mul(O::s((float)(1.0 / 9.0)), m.rho), wr5 = O::mul(O::s((float)(1.0 / 36.0)), m.rho);
  const V nom = O::s(-omega);
  V moving = O::s(0.0f);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int a = p < 2 ? p + 1 : p + 3;   // 1, 2, 5, 6
    const int b = p < 2 ? p + 3 : p + 5;   // 3, 4, 7, 8
    const V wr = p < 2 ? wr1 : wr5;
    const V sym = O::fma(O::mul(O::s(0.5f), cu[p]), cu[p], m.base);   // 1 + cu^2 / 2 - 1.5 u^2
    const V ea = O::mul(wr, O::add(sym, cu[p]));
    const V eb = O::mul(wr, O::sub(sym, cu[p]));
    f[a] = O::fma(nom, O::sub(f[a], ea), f[a]);
    f[b] = O::fma(nom, O::sub(f[b], eb), f[b]);
    moving = O::add(moving, O::add(ea, eb));
  }
  f[0] = O::fma(nom, O::sub(f[0], O::sub(m.rho, moving)), f[0]);
  return m.rho;
}

// TRT on the pairs (1,3), (2,4), (5,7), (6,8) (src/lattice.rs:100-119): the symmetric part relaxes
// at op, the antisymmetric part at om; the rest population as in BGK at op. Returns rho.
template <class V>
__device__ __forceinline__ V collide_trt_n(V* f, float op_, float om_) {
  using O = NOps<V>;
  const NMacro<V> m = macro_n(f);
  V cu[4];
  cu_n(m, cu);
  const V wr1 = O::mul(O::s((float)(1.0 / 9.0)), m.rho), wr5 = O::mul(O::s((float)(1.0 / 36.0)), m.rho);
  const V op = O::s(op_), om = O::s(om_);
  V moving = O::s(0.0f);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int a = p < 2 ? p + 1 : p + 3;
    const int b = p < 2 ? p + 3 : p + 5;
    const V wr = p < 2 ? wr1 : wr5;
    const V eq = O::mul(wr, O::fma(O::mul(O::s(0.5f), cu[p]), cu[p], m.base));
    const V dp = O::mul(op, O::fma(O::s(0.5f), O::add(f[a], f[b]), O::neg(eq)));
    const V dm = O::mul(om, O::fma(O::s(0.5f), O::sub(f[a], f[b]), O::neg(O::mul(wr, cu[p]))));
    const V fa = f[a], fb = f[b];
    f[a] = O::sub(O::sub(fa, dp), dm);
    f[b] = O::add(O::sub(fb, dp), dm);
    moving = O::fma(O::s(2.0f), eq, moving);
  }
  f[0] = O::fma(O::s(-op_), O::sub(f[0], O::sub(m.rho, moving)), f[0]);
  return m.rho;
}

}  // namespace vl
