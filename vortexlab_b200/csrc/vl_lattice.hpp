// D2Q9 lattice constants and collision operators, for host (g++) and device (nvcc) code.
//
// The operators are templated on the arithmetic type R (double for the FP64 path, float for the
// reduced-precision paths). For R = double and a translation unit compiled without FMA
// contraction (nvcc -fmad=false, g++ -ffp-contract=off) each operator performs exactly the
// floating-point operations of the reference, in the same order, so results are bit-identical:
//   moments           src/lattice.rs:59-64
//   equilibrium       src/lattice.rs:68-76
//   collide_bgk       src/lattice.rs:80-95
//   collide_trt       src/lattice.rs:100-119
//   collide_forced    src/lattice.rs:127-156
// The rest population is relaxed towards `rho - sum of moving equilibria`, as in the reference,
// which keeps the equilibrium summing to rho to the last bit.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define VL_HD __host__ __device__ __forceinline__
#else
#define VL_HD inline
#endif

namespace vl {

enum { COLL_BGK = 0, COLL_TRT = 1 };
enum { PREC_F64 = 0, PREC_F32 = 1, PREC_F16S = 2 };

// Direction numbering (src/lattice.rs:3-11):   6 2 5 / 3 0 1 / 7 4 8
VL_HD constexpr int cx_of(int j) { return (int)((0x20919u >> (2 * j)) & 3u) - 1; }  // 0,1,0,-1,0,1,-1,-1,1
VL_HD constexpr int cy_of(int j) { return (int)((0x02865u >> (2 * j)) & 3u) - 1; }  // 0,0,1,0,-1,1,1,-1,-1
VL_HD constexpr int opp_of(int j) { return j == 0 ? 0 : (j < 5 ? ((j + 1) & 3) + 1 : ((j - 3) & 3) + 5); }
VL_HD constexpr double w_of(int j) { return j == 0 ? 4.0 / 9.0 : (j < 5 ? 1.0 / 9.0 : 1.0 / 36.0); }

constexpr int kCX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
constexpr int kCY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};

template <class R>
struct Lat {
  static constexpr R W0 = R(4.0 / 9.0);
  static constexpr R W1 = R(1.0 / 9.0);
  static constexpr R W5 = R(1.0 / 36.0);
};

template <class R>
VL_HD void moments(const R* f, R& rho, R& jx, R& jy) {
  rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
  jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
}

template <class R>
VL_HD R wgt(int i) {
  return i == 0 ? Lat<R>::W0 : (i < 5 ? Lat<R>::W1 : Lat<R>::W5);
}

template <class R>
VL_HD void equilibrium(R rho, R ux, R uy, R* out) {
  const R usq = R(1.5) * (ux * ux + uy * uy);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const R cu = R(3.0) * (R(cx_of(i)) * ux + R(cy_of(i)) * uy);
    out[i] = wgt<R>(i) * rho * (R(1.0) + cu + R(0.5) * cu * cu - usq);
  }
}

template <class R>
VL_HD void collide_bgk(R* f, R omega) {
  R rho, jx, jy;
  moments(f, rho, jx, jy);
  const R inv = R(1.0) / rho;
  R feq[9];
  equilibrium(rho, jx * inv, jy * inv, feq);
  R moving = R(0.0);
#pragma unroll
  for (int i = 1; i < 9; ++i) {
    f[i] = f[i] - omega * (f[i] - feq[i]);
    moving += feq[i];
  }
  f[0] = f[0] - omega * (f[0] - (rho - moving));
}

// TRT pairs (1,3), (2,4), (5,7), (6,8) in that order (src/lattice.rs:24).
template <class R>
VL_HD void collide_trt(R* f, R op, R om) {
  R rho, jx, jy;
  moments(f, rho, jx, jy);
  const R inv = R(1.0) / rho;
  const R ux = jx * inv, uy = jy * inv;
  const R usq = R(1.5) * (ux * ux + uy * uy);
  R moving = R(0.0);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int a = p < 2 ? p + 1 : p + 3;
    const int b = p < 2 ? p + 3 : p + 5;
    const R cu = R(3.0) * (R(cx_of(a)) * ux + R(cy_of(a)) * uy);
    const R wr = wgt<R>(a) * rho;
    const R eq = wr * (R(1.0) + R(0.5) * cu * cu - usq);
    const R dp = op * (R(0.5) * (f[a] + f[b]) - eq);
    const R dm = om * (R(0.5) * (f[a] - f[b]) - wr * cu);
    const R fa = f[a], fb = f[b];
    f[a] = fa - dp - dm;
    f[b] = fb - dp + dm;
    moving += R(2.0) * eq;
  }
  f[0] = f[0] - op * (f[0] - (rho - moving));
}

template <class R>
VL_HD void collide_forced(R* f, R op, R om, R gx, R gy) {
  R rho, jx, jy;
  moments(f, rho, jx, jy);
  const R inv = R(1.0) / rho;
  const R ux = jx * inv + R(0.5) * gx, uy = jy * inv + R(0.5) * gy;
  const R fx = rho * gx, fy = rho * gy;
  const R usq = R(1.5) * (ux * ux + uy * uy);
  const R uf = R(3.0) * (ux * fx + uy * fy);
  const R kp = R(1.0) - R(0.5) * op, km = R(1.0) - R(0.5) * om;
  R moving = R(0.0), source = R(0.0);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int a = p < 2 ? p + 1 : p + 3;
    const int b = p < 2 ? p + 3 : p + 5;
    const R cx = R(cx_of(a)), cy = R(cy_of(a));
    const R cu = R(3.0) * (cx * ux + cy * uy);
    const R cf = R(3.0) * (cx * fx + cy * fy);
    const R wr = wgt<R>(a) * rho;
    const R eq = wr * (R(1.0) + R(0.5) * cu * cu - usq);
    const R dp = op * (R(0.5) * (f[a] + f[b]) - eq);
    const R dm = om * (R(0.5) * (f[a] - f[b]) - wr * cu);
    const R sp = kp * wgt<R>(a) * (cu * cf - uf);
    const R sm = km * wgt<R>(a) * cf;
    const R fa = f[a], fb = f[b];
    f[a] = fa - dp - dm + sp + sm;
    f[b] = fb - dp + dm + sp - sm;
    moving += R(2.0) * eq;
    source += R(2.0) * sp;
  }
  f[0] = f[0] - op * (f[0] - (rho - moving)) - source;
}

// Collision dispatch of Sim::step (src/sim.rs:407-413): forced if a body acceleration is set,
// else BGK or TRT.
template <class R>
VL_HD void collide(R* f, int coll, bool forced, R op, R om, R gx, R gy) {
  if (forced)
    collide_forced(f, op, om, gx, gy);
  else if (coll == COLL_BGK)
    collide_bgk(f, op);
  else
    collide_trt(f, op, om);
}

}  // namespace vl
