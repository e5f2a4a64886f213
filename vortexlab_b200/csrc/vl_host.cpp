// Host-side domain compiler, shapes and signal analysis (compiled by g++ with
// -ffp-contract=off so that link geometry and analysis match the reference bit for bit).
#include "vl_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>

namespace vl {

// ------------------------------------------------------------------ shapes
// Square section of side d with a corner treatment, optionally rotated (src/geometry.rs:215-261).
// The top-right corner profile (offsets in units of d, counter-clockwise) is repeated at the
// four corners by quarter turns.
std::unique_ptr<Shape> make_section(int corner, double b, double cx, double cy, double d, double angle) {
  std::unique_ptr<Shape> base;
  if (corner == 2) {  // rounded
    auto r = std::make_unique<RoundedSquareShape>();
    r->cx = cx; r->cy = cy; r->half = 0.5 * d; r->r = b * d;
    base = std::move(r);
  } else {
    std::vector<std::pair<double, double>> prof;
    switch (corner) {
      case 1: prof = {{0.0, -b}, {-b, 0.0}}; break;
      case 3: prof = {{0.0, -b}, {-b, -b}, {-b, 0.0}}; break;
      case 4: prof = {{0.0, -2.0 * b}, {-b, -2.0 * b}, {-b, -b}, {-2.0 * b, -b}, {-2.0 * b, 0.0}}; break;
      default: prof = {{0.0, 0.0}}; break;
    }
    auto poly = std::make_unique<PolygonShape>();
    const double h = 0.5 * d;
    for (int quarter = 0; quarter < 4; ++quarter) {
      for (const auto& pr : prof) {
        const double x = h + pr.first * d, y = h + pr.second * d;
        double rx = x, ry = y;
        if (quarter == 1) { rx = -y; ry = x; }
        else if (quarter == 2) { rx = -x; ry = -y; }
        else if (quarter == 3) { rx = y; ry = -x; }
        poly->vx.push_back(cx + rx);
        poly->vy.push_back(cy + ry);
      }
    }
    base = std::move(poly);
  }
  if (angle == 0.0) return base;
  auto rot = std::make_unique<RotatedShape>();
  rot->inner = std::move(base); rot->cx = cx; rot->cy = cy; rot->angle = angle;
  return rot;
}

// Star-convex polygon: vertex k at angle phase + 2 pi k / n and distance radii[k] from the centre.
std::unique_ptr<Shape> make_star(double cx, double cy, const double* radii, size_t nvert, double phase) {
  auto poly = std::make_unique<PolygonShape>();
  for (size_t k = 0; k < nvert; ++k) {
    const double th = phase + 2.0 * M_PI * (double)k / (double)nvert;
    poly->vx.push_back(cx + radii[k] * std::cos(th));
    poly->vy.push_back(cy + radii[k] * std::sin(th));
  }
  return poly;
}

// Bisection for the fraction of a fluid-to-solid link that lies in the fluid
// (src/geometry.rs:268-279): 40 halvings, clamped to [1e-9, 1].
double cut_fraction(const Shape& s, double x, double y, double dx, double dy) {
  double lo = 0.0, hi = 1.0;
  for (int it = 0; it < 40; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (s.inside(x + mid * dx, y + mid * dy)) hi = mid; else lo = mid;
  }
  const double q = 0.5 * (lo + hi);
  return std::min(std::max(q, 1e-9), 1.0);
}

void DiskUnionShape::index() {
  double x0 = 0, x1 = 0, y0 = 0, y1 = 0;
  for (size_t k = 0; k < r.size(); ++k) {
    const double a = cx[k] - r[k], b = cx[k] + r[k], c = cy[k] - r[k], d = cy[k] + r[k];
    if (k == 0 || a < x0) x0 = a;
    if (k == 0 || b > x1) x1 = b;
    if (k == 0 || c < y0) y0 = c;
    if (k == 0 || d > y1) y1 = d;
  }
  gx0 = (long)std::floor(x0 / cell) - 1;
  gy0 = (long)std::floor(y0 / cell) - 1;
  gw = (long)std::floor(x1 / cell) - gx0 + 2;
  gh = (long)std::floor(y1 / cell) - gy0 + 2;
  bucket.assign((size_t)(gw * gh), {});
  for (size_t k = 0; k < r.size(); ++k) {
    const long i0 = (long)std::floor((cx[k] - r[k]) / cell) - gx0, i1 = (long)std::floor((cx[k] + r[k]) / cell) - gx0;
    const long j0 = (long)std::floor((cy[k] - r[k]) / cell) - gy0, j1 = (long)std::floor((cy[k] + r[k]) / cell) - gy0;
    for (long j = j0; j <= j1; ++j)
      for (long i = i0; i <= i1; ++i) bucket[(size_t)(j * gw + i)].push_back((int32_t)k);
  }
}

bool DiskUnionShape::inside(double x, double y) const {
  const long i = (long)std::floor(x / cell) - gx0, j = (long)std::floor(y / cell) - gy0;
  if (i < 0 || j < 0 || i >= gw || j >= gh) return false;
  for (int32_t k : bucket[(size_t)(j * gw + i)]) {
    const double dx = x - cx[k], dy = y - cy[k];
    if (dx * dx + dy * dy < r[k] * r[k]) return true;
  }
  return false;
}

// src/geometry.rs:99-115
bool bounding_box(const Shape& s, double reach, double step, double* out) {
  const size_t n = (size_t)std::ceil(2.0 * reach / step);
  double x0 = std::numeric_limits<double>::max(), x1 = std::numeric_limits<double>::lowest();
  double y0 = x0, y1 = x1;
  for (size_t j = 0; j <= n; ++j) {
    const double y = -reach + (double)j * step;
    for (size_t i = 0; i <= n; ++i) {
      const double x = -reach + (double)i * step;
      if (!s.inside(x, y)) continue;
      x0 = std::fmin(x0, x); x1 = std::fmax(x1, x);
      y0 = std::fmin(y0, y); y1 = std::fmax(y1, y);
    }
  }
  if (!(x0 <= x1)) return false;
  out[0] = x0 - 0.5 * step; out[1] = x1 + 0.5 * step;
  out[2] = y0 - 0.5 * step; out[3] = y1 + 0.5 * step;
  return true;
}

void WallVelocity::at(double x, double y, double& ux, double& uy) const {
  switch (kind) {
    case VEL_CONST: ux = p[0]; uy = p[1]; return;
    case VEL_PARABOLIC: {  // src/cases/channel.rs:80-83
      const double u_mean = p[0], h = p[1];
      const double s = std::min(std::max(y - 0.5, 0.0), h);
      ux = 6.0 * u_mean * s * (h - s) / (h * h);
      uy = 0.0;
      return;
    }
    case VEL_ROTATION: ux = -(y - p[1]); uy = x - p[0]; return;  // src/cases/channel.rs:104
    default: ux = 0.0; uy = 0.0; return;
  }
}

// ------------------------------------------------------------------ domain compiler
// Scans the cells in y-major, x order. A fluid cell whose neighbour along direction j is not
// fluid owns one link per such j (j = 1..8 ascending); the link order defines the force
// accumulation order. Mirrors the classification of src/sim.rs:243-328.
bool compile_domain(const DomainSpec& spec, CompiledDomain& out, std::string& err) {
  const size_t nx = spec.nx, ny = spec.ny, n = nx * ny;
  if (!(spec.tau > 0.5)) { err = "tau must exceed 1/2 (viscosity must be positive)"; return false; }
  if (n > (size_t)std::numeric_limits<int32_t>::max() / 2) { err = "grid too large for int32 cell indices"; return false; }
  const long lnx = (long)nx, lny = (long)ny;
  // Neighbour with periodic wrap; -1 if it leaves a non-periodic domain.
  auto neighbour = [&](long x, long y) -> long {
    if (x < 0 || x >= lnx) {
      if (!spec.periodic_x) return -1;
      x = ((x % lnx) + lnx) % lnx;
    }
    if (y < 0 || y >= lny) {
      if (!spec.periodic_y) return -1;
      y = ((y % lny) + lny) % lny;
    }
    return y * lnx + x;
  };
  auto is_open = [&](long c) {
    if (c < 0) return false;
    const KindTag t = spec.kinds[spec.paint[(size_t)c]].tag;
    return t == KIND_PRESSURE || t == KIND_RADIATING;
  };

  out = CompiledDomain();
  out.nx = nx; out.ny = ny; out.n = n;
  out.periodic_x = spec.periodic_x; out.periodic_y = spec.periodic_y;
  out.collision = spec.collision;
  out.accel[0] = spec.accel[0]; out.accel[1] = spec.accel[1];
  // Collision::omegas (src/lattice.rs:39-44)
  out.op = 1.0 / spec.tau;
  out.om = spec.collision == COLL_BGK ? 1.0 / spec.tau : 1.0 / (0.5 + spec.magic / (spec.tau - 0.5));
  out.flag.assign(n, 2);
  out.bnode_first.push_back(0);
  int ngroups = 0;

  for (long y = 0; y < lny; ++y) {
    for (long x = 0; x < lnx; ++x) {
      const long idx = y * lnx + x;
      if (spec.paint[(size_t)idx] != 0) continue;
      out.fluid_nodes += 1;
      const size_t before = out.links.size();
      for (int j = 1; j < 9; ++j) {
        const long cx = cx_of(j), cy = cy_of(j);
        const long tgt = neighbour(x + cx, y + cy);
        if (tgt < 0) {
          char buf[192];
          snprintf(buf, sizeof buf,
                   "fluid cell (%ld,%ld) touches a non-periodic edge; close the domain with wall or pressure cells", x, y);
          err = buf;
          return false;
        }
        const uint8_t kid = spec.paint[(size_t)tgt];
        if (kid == 0) continue;
        const CellKind& kind = spec.kinds[kid];
        LinkRec L;
        std::memset(&L, 0, sizeof L);
        L.dir = (uint8_t)j;
        L.q = 0.5;
        L.rho = 1.0;
        L.fgroup = -1;
        const long back = neighbour(x - cx, y - cy);
        L.behind = (back >= 0 && spec.paint[(size_t)back] == 0) ? (int32_t)back : -1;
        if (kind.tag == KIND_PRESSURE || kind.tag == KIND_RADIATING) {
          const bool radiating = kind.tag == KIND_RADIATING;
          L.rho = kind.rho;
          // Outward normal: along x if the cell beside the node in x is open boundary too,
          // otherwise along y (src/sim.rs:292-297).
          int nxv = 0, nyv = 0;
          if (is_open(neighbour(x + cx, y))) nxv = (int)cx; else nyv = (int)cy;
          L.flags = (uint8_t)(1u | (radiating ? 2u : 0u) | ((unsigned)(nxv + 1) << 2) | ((unsigned)(nyv + 1) << 4));
          if (!radiating && (out.pnode_idx.empty() || out.pnode_idx.back() != (int32_t)idx)) {
            out.pnode_idx.push_back((int32_t)idx);
            out.pnode_nx.push_back((int8_t)nxv);
            out.pnode_ny.push_back((int8_t)nyv);
          }
        } else if (kind.tag == KIND_WALL) {
          if (kind.vgroup < 0 || kind.vgroup >= 4) { err = "wall vgroup must be below 4"; return false; }
          L.vgroup = (uint8_t)kind.vgroup;
          L.flags = (uint8_t)((1u << 2) | (1u << 4));
          if (kind.shape) L.q = cut_fraction(*kind.shape, (double)x, (double)y, (double)cx, (double)cy);
          if (kind.velocity.kind != VEL_NONE) {
            const double wx = (double)x + L.q * (double)cx, wy = (double)y + L.q * (double)cy;
            kind.velocity.at(wx, wy, L.uw[0], L.uw[1]);
            L.cu6 = 6.0 * w_of(j) * ((double)cx * L.uw[0] + (double)cy * L.uw[1]);
          }
          if (kind.fgroup >= 0) {
            if (kind.fgroup >= 4) { err = "force group must be below 4 (VL_MAX_FGROUPS)"; return false; }
            L.fgroup = (int8_t)kind.fgroup;
            ngroups = std::max(ngroups, kind.fgroup + 1);
          }
        }
        out.links.push_back(L);
      }
      if (out.links.size() > before) {
        out.flag[(size_t)idx] = 1;
        out.bnode_idx.push_back((int32_t)idx);
        out.bnode_first.push_back((int32_t)out.links.size());
      } else {
        out.flag[(size_t)idx] = 0;
      }
    }
  }
  if (out.links.size() > (size_t)std::numeric_limits<int32_t>::max()) { err = "too many links"; return false; }
  out.ngroups = ngroups;
  return true;
}

// ------------------------------------------------------------------ signal (src/signal.rs)
// Radix-2 decimation-in-time FFT, forward sign (src/signal.rs:6-43).
void fft_inplace(double* re, double* im, size_t n) {
  size_t j = 0;
  for (size_t i = 1; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j |= bit;
    if (i < j) { std::swap(re[i], re[j]); std::swap(im[i], im[j]); }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const double ang = -2.0 * M_PI / (double)len;
    const double wr = std::cos(ang), wi = std::sin(ang);
    for (size_t start = 0; start < n; start += len) {
      double cr = 1.0, ci = 0.0;
      const size_t half = len / 2;
      for (size_t k = 0; k < half; ++k) {
        const size_t a = start + k, b = a + half;
        const double tr = re[b] * cr - im[b] * ci, ti = re[b] * ci + im[b] * cr;
        re[b] = re[a] - tr;
        im[b] = im[a] - ti;
        re[a] += tr;
        im[a] += ti;
        const double ncr = cr * wr - ci * wi;
        ci = cr * wi + ci * wr;
        cr = ncr;
      }
    }
  }
}

double series_mean(const double* x, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += x[i];
  return s / (double)n;
}

double series_rms(const double* x, size_t n) {
  const double m = series_mean(x, n);
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += (x[i] - m) * (x[i] - m);
  return std::sqrt(s / (double)n);
}

// Hann-windowed, mean-removed, zero-padded amplitude spectrum (src/signal.rs:74-88), then the
// strongest bin refined by a parabola through the log-amplitudes (src/signal.rs:92-107).
void dominant_frequency(const double* x, size_t n, double dt, double& freq, double& amp) {
  const double m = series_mean(x, n);
  size_t size = 1;
  while (size < n * 8) size <<= 1;
  std::vector<double> re(size, 0.0), im(size, 0.0);
  for (size_t i = 0; i < n; ++i) {
    const double w = 0.5 - 0.5 * std::cos(2.0 * M_PI * (double)i / (double)n);
    re[i] = (x[i] - m) * w;
  }
  fft_inplace(re.data(), im.data(), size);
  const double scale = 4.0 / (double)n;
  const size_t ns = size / 2;
  std::vector<double> fr(ns), am(ns);
  for (size_t k = 0; k < ns; ++k) {
    fr[k] = (double)k / ((double)size * dt);
    am[k] = scale * std::sqrt(re[k] * re[k] + im[k] * im[k]);
  }
  size_t k = 1;
  for (size_t i = 1; i + 1 < ns; ++i)
    if (am[i] > am[k]) k = i;
  if (k == 0 || k + 1 >= ns || am[k] <= 0.0 || am[k - 1] <= 0.0 || am[k + 1] <= 0.0) {
    freq = fr[k]; amp = am[k];
    return;
  }
  const double a = std::log(am[k - 1]), b = std::log(am[k]), c = std::log(am[k + 1]);
  const double shift = 0.5 * (a - c) / (a - 2.0 * b + c);
  const double df = fr[1] - fr[0];
  freq = fr[k] + shift * df;
  amp = std::exp(b - 0.25 * (a - c) * shift);
}

// Local maxima above the mean, refined by a parabola (src/signal.rs:111-123).
size_t find_peaks(const double* x, size_t n, double* pos, double* val, size_t cap) {
  const double m = series_mean(x, n);
  size_t cnt = 0;
  for (size_t i = 1; i + 1 < n; ++i) {
    if (!(x[i] > m && x[i] > x[i - 1] && x[i] >= x[i + 1])) continue;
    const double a = x[i - 1], b = x[i], c = x[i + 1];
    const double denom = a - 2.0 * b + c;
    const double shift = denom != 0.0 ? 0.5 * (a - c) / denom : 0.0;
    if (cnt < cap) { pos[cnt] = (double)i + shift; val[cnt] = b - 0.25 * (a - c) * shift; }
    ++cnt;
  }
  return cnt;
}

// Mean spacing of upward mean-crossings (src/signal.rs:127-140).
bool crossing_frequency(const double* x, size_t n, double dt, double& out) {
  const double m = series_mean(x, n);
  double first = 0.0, last = 0.0;
  size_t count = 0;
  for (size_t i = 1; i < n; ++i) {
    const double a = x[i - 1] - m, b = x[i] - m;
    if (a < 0.0 && b >= 0.0) {
      const double t = (double)(i - 1) + a / (a - b);
      if (count == 0) first = t;
      last = t;
      ++count;
    }
  }
  if (count < 2) return false;
  out = (double)(count - 1) / ((last - first) * dt);
  return true;
}

// src/signal.rs:143-147
double sample_at(const double* x, size_t n, double pos) {
  const size_t i = std::min((size_t)std::floor(pos), n - 2);
  const double f = pos - (double)i;
  return x[i] * (1.0 - f) + x[i + 1] * f;
}

}  // namespace vl
