// ORACLE — test infrastructure only. Storage-rounding study on the oracle's CPU solver: the
// Schafer-Turek 2D-2 rig (src/cases/cylinder.rs:35-50, TRT 3/16, u_mean 0.05, Re 100) with every
// population re-stored after each step as w_i + round(f_i - w_i) in a 16-bit format, the collision
// and everything else in FP64. It separates the physics of a storage format from any GPU kernel:
//
//   make -C oracle storage_rounding && oracle/storage_rounding N MODE [units window]
//
// MODE 0: FP64 (no rounding); 1: IEEE half; 2: the custom 16-bit format of the GPU path (sign,
// 3-bit exponent, 12-bit mantissa, exponent bias 9: 2^(e-9) (1 + m/4096), m 2^-20 below 2^-8,
// saturating at 0.49994); 3: 16-bit fixed point with a step of 2^-18; 4: 16-bit fixed point with
// steps 2^-19 (rest), 2^-18 (axis directions), 2^-19 (diagonals). Prints c_D max / mean,
// c_L max / min, St (dominant lift frequency) over the last `window` convective units and the
// total mass.
#include "vl_oracle.cpp"

#include <cstdio>
#include <cstdlib>

namespace {

const double kW[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};

// The custom format: (f - w) 2^-118 as FP32 (its evenly spaced range lands on the FP32
// subnormals), the FP32 bits rounded to 12 mantissa bits (ties to even) and clamped.
double round_custom(double d) {
  float y = (float)d * 0x1p-118f;
  uint32_t b;
  std::memcpy(&b, &y, 4);
  const uint32_t sign = b & 0x80000000u, maxb = 0x03fff800u;
  uint32_t mag = std::min(b & 0x7fffffffu, maxb);
  mag = (mag + 0x3ffu + ((mag >> 11) & 1u)) & ~0x7ffu;
  mag = std::min(mag, maxb);
  const uint32_t o = sign | mag;
  float z;
  std::memcpy(&z, &o, 4);
  return (double)(z * 0x1p118f);
}

double round_fixed(double d, int k) {
  const double q = std::min(std::max(std::nearbyint(std::ldexp(d, k)), -32768.0), 32767.0);
  return std::ldexp(q, -k);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s N MODE [units window]\n", argv[0]);
    return 2;
  }
  const int n = std::atoi(argv[1]), mode = std::atoi(argv[2]);
  const double units = argc > 3 ? std::atof(argv[3]) : 100.0, window = argc > 4 ? std::atof(argv[4]) : 20.0;
  const double u = 0.05, re = 100.0, nf = n, c0 = 0.5 + 2.0 * nf;
  auto* body = new Circle();
  body->cx = c0;
  body->cy = c0;
  body->r = 0.5 * nf;
  std::string err;
  Channel* ch = channel_new(22 * n + 2, 41 * n / 10 + 2, 0, u, u * nf / re, 1, 3.0 / 16.0, body,
                            (uint64_t)(8.0 * nf / u), nullptr, 8, &err);
  if (!ch) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 1;
  }
  Sim& s = *ch->sim;
  const uint64_t steps = (uint64_t)(units * nf / u);
  std::vector<double> cd(steps), cl(steps);
  const size_t nt = s.pool->threads();
  for (uint64_t k = 0; k < steps; ++k) {
    ch->step();
    if (mode != 0) {
      double* pa = s.a.data();
      const size_t N = s.n;
      s.pool->run([&](size_t th) {
        for (int i = 0; i < 9; ++i)
          for (size_t idx = th * N / nt; idx < (th + 1) * N / nt; ++idx) {
            const double d = pa[i * N + idx] - kW[i];
            const double q = mode == 1   ? (double)(_Float16)(float)d
                             : mode == 2 ? round_custom(d)
                             : mode == 3 ? round_fixed(d, 18)
                                         : round_fixed(d, i == 0 ? 19 : (i < 5 ? 18 : 19));
            pa[i * N + idx] = kW[i] + q;
          }
      });
    }
    const double c = 2.0 / (u * u * nf);
    cd[k] = c * s.force[0];
    cl[k] = c * s.force[1];
  }
  const uint64_t w0 = steps - (uint64_t)(window * nf / u);
  double cdmax = -1e300, clmax = -1e300, clmin = 1e300, cdsum = 0.0;
  for (uint64_t k = w0; k < steps; ++k) {
    cdmax = std::max(cdmax, cd[k]);
    clmax = std::max(clmax, cl[k]);
    clmin = std::min(clmin, cl[k]);
    cdsum += cd[k];
  }
  double f, amp;
  dominant_frequency(cl.data() + w0, steps - w0, 1.0, &f, &amp);
  std::printf("n=%d mode=%d cd_max=%.5f cd_mean=%.5f cl_max=%.5f cl_min=%.5f St=%.5f mass=%.9f\n", n, mode, cdmax,
              cdsum / (double)(steps - w0), clmax, clmin, f * nf / u, total_mass(s));
  return 0;
}
