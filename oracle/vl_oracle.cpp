// ORACLE — test infrastructure only. Not part of the product.
//
// A plain C++17 restatement of the reference's FP64 CPU path (vortexlab, a Rust crate that
// cannot be compiled here: no cargo/rustc in the image). Only tests/, the smoke check and the
// CPU-baseline leg of bench.py load this library, and only as the checker / timed CPU baseline.
//
// Every function follows the reference expression by expression (same operand order, same
// association), and the library is compiled with -O3 -ffp-contract=off and without fast-math,
// so that its FP64 results are bit-identical to the reference's (which runs on aarch64 Rust,
// where LLVM never contracts a*b+c into an FMA).
//
// Parity pins (checked by tests/test_oracle_golden.py):
//   * state hash 6b6814b976bbbaff after cylinder::bench(n=40, u_mean=0.05, TRT 3/16), 3000 steps
//   * state hash c93e26bfa33474ee after cylinder::bench(n=80, ...), 1000 steps
//     (docs/report/index.html:59, commands Makefile:42-43)
//   * the unit tests of src/lattice.rs:184-288, src/geometry.rs:298-357, src/signal.rs:351-405
//   * the solver invariants of tests/solver.rs.
//
// Files restated: src/lattice.rs:16-156, src/sim.rs:33-735, src/geometry.rs:11-279,
// src/pool.rs (row split only), src/cases/mod.rs:10-18, src/cases/channel.rs:22-189,
// src/cases/cylinder.rs:18-232, src/cases/tunnel.rs:11-67, src/cases/poiseuille.rs:11-21,
// src/signal.rs:6-147.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace vlo {

// ---------------------------------------------------------------- lattice (src/lattice.rs:16-24)
constexpr int Q = 9;
constexpr int CX[Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
constexpr int CY[Q] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const double W[Q] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                            1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
constexpr int OPP[Q] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const double CS2 = 1.0 / 3.0;
constexpr int PAIRS[4][2] = {{1, 3}, {2, 4}, {5, 7}, {6, 8}};

enum Collision { BGK = 0, TRT = 1 };

// src/lattice.rs:39-44
static void omegas(int coll, double magic, double tau, double* op, double* om) {
  if (coll == BGK) {
    *op = 1.0 / tau;
    *om = 1.0 / tau;
  } else {
    *op = 1.0 / tau;
    *om = 1.0 / (0.5 + magic / (tau - 0.5));
  }
}

// src/lattice.rs:53-55
static double tau_for(double nu) { return nu / CS2 + 0.5; }

// src/lattice.rs:59-64
static inline void moments(const double* f, double* rho, double* jx, double* jy) {
  *rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  *jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
  *jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
}

// src/lattice.rs:68-76
static inline void equilibrium(double rho, double ux, double uy, double* out) {
  double usq = 1.5 * (ux * ux + uy * uy);
  for (int i = 0; i < Q; ++i) {
    double cu = 3.0 * ((double)CX[i] * ux + (double)CY[i] * uy);
    out[i] = W[i] * rho * (1.0 + cu + 0.5 * cu * cu - usq);
  }
}

// src/lattice.rs:80-95
static inline void collide_bgk(const double* f, double omega, double* out) {
  double rho, jx, jy;
  moments(f, &rho, &jx, &jy);
  double inv = 1.0 / rho;
  double feq[Q];
  equilibrium(rho, jx * inv, jy * inv, feq);
  double moving = 0.0;
  for (int i = 1; i < Q; ++i) {
    out[i] = f[i] - omega * (f[i] - feq[i]);
    moving += feq[i];
  }
  out[0] = f[0] - omega * (f[0] - (rho - moving));
}

// src/lattice.rs:100-119
static inline void collide_trt(const double* f, double op, double om, double* out) {
  double rho, jx, jy;
  moments(f, &rho, &jx, &jy);
  double inv = 1.0 / rho;
  double ux = jx * inv, uy = jy * inv;
  double usq = 1.5 * (ux * ux + uy * uy);
  double moving = 0.0;
  for (int p = 0; p < 4; ++p) {
    int a = PAIRS[p][0], b = PAIRS[p][1];
    double cu = 3.0 * ((double)CX[a] * ux + (double)CY[a] * uy);
    double wr = W[a] * rho;
    double eq = wr * (1.0 + 0.5 * cu * cu - usq);
    double dp = op * (0.5 * (f[a] + f[b]) - eq);
    double dm = om * (0.5 * (f[a] - f[b]) - wr * cu);
    out[a] = f[a] - dp - dm;
    out[b] = f[b] - dp + dm;
    moving += 2.0 * eq;
  }
  out[0] = f[0] - op * (f[0] - (rho - moving));
}

// src/lattice.rs:127-156
static inline void collide_forced(const double* f, double op, double om, double gx, double gy,
                                  double* out) {
  double rho, jx, jy;
  moments(f, &rho, &jx, &jy);
  double inv = 1.0 / rho;
  double ux = jx * inv + 0.5 * gx, uy = jy * inv + 0.5 * gy;
  double fx = rho * gx, fy = rho * gy;
  double usq = 1.5 * (ux * ux + uy * uy);
  double uf = 3.0 * (ux * fx + uy * fy);
  double kp = 1.0 - 0.5 * op, km = 1.0 - 0.5 * om;
  double moving = 0.0, source = 0.0;
  for (int p = 0; p < 4; ++p) {
    int a = PAIRS[p][0], b = PAIRS[p][1];
    double cx = (double)CX[a], cy = (double)CY[a];
    double cu = 3.0 * (cx * ux + cy * uy);
    double cf = 3.0 * (cx * fx + cy * fy);
    double wr = W[a] * rho;
    double eq = wr * (1.0 + 0.5 * cu * cu - usq);
    double dp = op * (0.5 * (f[a] + f[b]) - eq);
    double dm = om * (0.5 * (f[a] - f[b]) - wr * cu);
    double sp = kp * W[a] * (cu * cf - uf);
    double sm = km * W[a] * cf;
    out[a] = f[a] - dp - dm + sp + sm;
    out[b] = f[b] - dp + dm + sp - sm;
    moving += 2.0 * eq;
    source += 2.0 * sp;
  }
  out[0] = f[0] - op * (f[0] - (rho - moving)) - source;
}

// ---------------------------------------------------------------- geometry (src/geometry.rs)
struct Shape {
  virtual ~Shape() {}
  virtual bool inside(double x, double y) const = 0;
};

// src/geometry.rs:16-27
struct Circle : Shape {
  double cx, cy, r;
  bool inside(double x, double y) const override {
    double dx = x - cx, dy = y - cy;
    return dx * dx + dy * dy < r * r;
  }
};

// src/geometry.rs:30-49
struct Polygon : Shape {
  std::vector<double> px, py;
  bool inside(double x, double y) const override {
    size_t n = px.size();
    bool in = false;
    size_t j = n - 1;
    for (size_t i = 0; i < n; ++i) {
      double xi = px[i], yi = py[i], xj = px[j], yj = py[j];
      if (((yi > y) != (yj > y)) && x < (xj - xi) * (y - yi) / (yj - yi) + xi) in = !in;
      j = i;
    }
    return in;
  }
};

// src/geometry.rs:52-66
struct RoundedSquare : Shape {
  double cx, cy, half, r;
  bool inside(double x, double y) const override {
    double core = half - r;
    double dx = std::fmax(std::fabs(x - cx) - core, 0.0);
    double dy = std::fmax(std::fabs(y - cy) - core, 0.0);
    return std::fabs(x - cx) < half && std::fabs(y - cy) < half && dx * dx + dy * dy < r * r;
  }
};

// src/geometry.rs:69-82
struct Rotated : Shape {
  std::unique_ptr<Shape> inner;
  double cx, cy, angle;
  bool inside(double x, double y) const override {
    double s = std::sin(angle), c = std::cos(angle);
    double dx = x - cx, dy = y - cy;
    return inner->inside(cx + c * dx + s * dy, cy - s * dx + c * dy);
  }
};

// src/geometry.rs:85-95
struct Translated : Shape {
  std::unique_ptr<Shape> inner;
  double dx, dy;
  bool inside(double x, double y) const override { return inner->inside(x - dx, y - dy); }
};

// src/cases/poiseuille.rs:12-21: everything outside the band y0 < y < y1.
struct OutsideBand : Shape {
  double y0, y1;
  bool inside(double, double y) const override { return y <= y0 || y >= y1; }
};

// Axis-aligned ellipse with semi-axes (a, b). Not in the reference (a new body class for the
// batched tunnels); defined here so the product's ellipse can be checked.
struct Ellipse : Shape {
  double cx, cy, a, b;
  bool inside(double x, double y) const override {
    double u = (x - cx) / a, v = (y - cy) / b;
    return u * u + v * v < 1.0;
  }
};

// Union of disks: inside if any Circle (src/geometry.rs:22-27) contains the point. Plain scan over
// the disks whose bounding box contains the point (a sorted sweep on x keeps it fast).
struct DiskUnion : Shape {
  std::vector<double> cx, cy, r;
  std::vector<size_t> order;  // by cx - r
  double rmax = 0.0;
  void prepare() {
    order.resize(cx.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cx[a] - r[a] < cx[b] - r[b]; });
    for (double v : r) rmax = std::max(rmax, v);
  }
  bool inside(double x, double y) const override {
    // first disk whose left edge could be at or left of x
    size_t lo = 0, hi = order.size();
    while (lo < hi) {
      size_t mid = (lo + hi) / 2;
      if (cx[order[mid]] - r[order[mid]] <= x) lo = mid + 1; else hi = mid;
    }
    for (size_t m = lo; m-- > 0;) {
      size_t k = order[m];
      if (cx[k] + rmax < x - rmax) break;
      double dx = x - cx[k], dy = y - cy[k];
      if (dx * dx + dy * dy < r[k] * r[k]) return true;
    }
    return false;
  }
};

// src/geometry.rs:120-185
struct Bitmap : Shape {
  size_t w = 0, h = 0;
  std::vector<float> level;
  double x0 = 0, y0 = 0, scale = 1;
  double at(long i, long j) const {
    if (i < 0 || j < 0 || i >= (long)w || j >= (long)h) return 0.0;
    return (double)level[(size_t)j * w + (size_t)i];
  }
  double sample(double x, double y) const {
    double px = (x - x0) / scale - 0.5;
    double py = (double)h - (y - y0) / scale - 0.5;
    double i = std::floor(px), j = std::floor(py);
    double fx = px - i, fy = py - j;
    long ii = (long)i, jj = (long)j;
    return (1.0 - fx) * (1.0 - fy) * at(ii, jj) + fx * (1.0 - fy) * at(ii + 1, jj) +
           (1.0 - fx) * fy * at(ii, jj + 1) + fx * fy * at(ii + 1, jj + 1);
  }
  bool inside(double x, double y) const override { return sample(x, y) > 0.5; }
};

// src/geometry.rs:189-248 (corner profiles and square sections)
enum Corner { SHARP = 0, CHAMFERED = 1, ROUNDED = 2, RECESSED = 3, DOUBLE_RECESSED = 4 };

static std::vector<std::pair<double, double>> corner_profile(int corner, double b) {
  switch (corner) {
    case CHAMFERED: return {{0.0, -b}, {-b, 0.0}};
    case RECESSED: return {{0.0, -b}, {-b, -b}, {-b, 0.0}};
    case DOUBLE_RECESSED:
      return {{0.0, -2.0 * b}, {-b, -2.0 * b}, {-b, -b}, {-2.0 * b, -b}, {-2.0 * b, 0.0}};
    default: return {{0.0, 0.0}};
  }
}

static std::unique_ptr<Shape> section(int corner, double b, double cx, double cy, double d,
                                      double angle) {
  std::unique_ptr<Shape> base;
  if (corner == ROUNDED) {
    auto r = std::make_unique<RoundedSquare>();
    r->cx = cx; r->cy = cy; r->half = 0.5 * d; r->r = b * d;
    base = std::move(r);
  } else {
    auto p = std::make_unique<Polygon>();
    double h = 0.5 * d;
    auto prof = corner_profile(corner, b);
    for (int k = 0; k < 4; ++k) {
      for (auto& pr : prof) {
        double x = h + pr.first * d, y = h + pr.second * d;
        double rx, ry;
        switch (k) {
          case 0: rx = x; ry = y; break;
          case 1: rx = -y; ry = x; break;
          case 2: rx = -x; ry = -y; break;
          default: rx = y; ry = -x; break;
        }
        p->px.push_back(cx + rx);
        p->py.push_back(cy + ry);
      }
    }
    base = std::move(p);
  }
  if (angle == 0.0) return base;
  auto r = std::make_unique<Rotated>();
  r->inner = std::move(base); r->cx = cx; r->cy = cy; r->angle = angle;
  return r;
}

// src/geometry.rs:268-279
static double cut_fraction(const Shape& s, double x, double y, double dx, double dy) {
  double lo = 0.0, hi = 1.0;
  for (int k = 0; k < 40; ++k) {
    double mid = 0.5 * (lo + hi);
    if (s.inside(x + mid * dx, y + mid * dy)) hi = mid; else lo = mid;
  }
  double q = 0.5 * (lo + hi);
  return q < 1e-9 ? 1e-9 : (q > 1.0 ? 1.0 : q);
}

// src/geometry.rs:99-115
static bool bounding_box(const Shape& s, double reach, double step, double* out) {
  size_t n = (size_t)std::ceil(2.0 * reach / step);
  double x0 = std::numeric_limits<double>::max(), x1 = std::numeric_limits<double>::lowest();
  double y0 = std::numeric_limits<double>::max(), y1 = std::numeric_limits<double>::lowest();
  for (size_t j = 0; j <= n; ++j) {
    double y = -reach + (double)j * step;
    for (size_t i = 0; i <= n; ++i) {
      double x = -reach + (double)i * step;
      if (s.inside(x, y)) {
        x0 = std::fmin(x0, x); x1 = std::fmax(x1, x);
        y0 = std::fmin(y0, y); y1 = std::fmax(y1, y);
      }
    }
  }
  if (!(x0 <= x1)) return false;
  out[0] = x0 - 0.5 * step; out[1] = x1 + 0.5 * step;
  out[2] = y0 - 0.5 * step; out[3] = y1 + 0.5 * step;
  return true;
}

// ---------------------------------------------------------------- wall velocity
// The reference takes a closure `Fn(x, y) -> [f64; 2]` (src/sim.rs:34). The closures its cases
// use are restated as tagged data:
enum VelKind { VEL_NONE = 0, VEL_CONST = 1, VEL_PARABOLIC = 2, VEL_ROTATION = 3 };
struct Velocity {
  int kind = VEL_NONE;
  double p[4] = {0, 0, 0, 0};
  void eval(double x, double y, double* u) const {
    switch (kind) {
      case VEL_CONST: u[0] = p[0]; u[1] = p[1]; return;
      case VEL_PARABOLIC: {
        // src/cases/channel.rs:77-85: s = (y - 0.5).clamp(0, h); 6 u_mean s (h - s) / h^2
        double u_mean = p[0], h = p[1];
        double s = y - 0.5;
        if (s < 0.0) s = 0.0;
        if (s > h) s = h;
        u[0] = 6.0 * u_mean * s * (h - s) / (h * h);
        u[1] = 0.0;
        return;
      }
      case VEL_ROTATION:
        // src/cases/channel.rs:104: [-(y - cy), x - cx]
        u[0] = -(y - p[1]); u[1] = x - p[0];
        return;
      default: u[0] = 0.0; u[1] = 0.0; return;
    }
  }
};

// ---------------------------------------------------------------- pool (src/pool.rs, row split)
// Persistent workers woken by a generation counter; run(f) calls f(t) for t in 0..threads.
class Pool {
 public:
  explicit Pool(size_t threads) : nt_(threads < 1 ? 1 : threads) {
    for (size_t t = 1; t < nt_; ++t) workers_.emplace_back([this, t] { loop(t); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }
  size_t threads() const { return nt_; }
  void run(const std::function<void(size_t)>& f) {
    if (nt_ == 1) { f(0); return; }
    {
      std::lock_guard<std::mutex> g(m_);
      job_ = &f;
      pending_ = nt_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    f(0);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [this] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(size_t t) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(size_t)>* job;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        job = job_;
      }
      (*job)(t);
      {
        std::lock_guard<std::mutex> g(m_);
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }
  size_t nt_;
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(size_t)>* job_ = nullptr;
  size_t pending_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// ---------------------------------------------------------------- sim (src/sim.rs)
enum KindTag { K_FLUID = 0, K_WALL = 1, K_PRESSURE = 2, K_RADIATING = 3 };
struct Kind {
  int tag = K_FLUID;
  Velocity vel;
  int vgroup = 0;
  long fgroup = -1;
  std::unique_ptr<Shape> shape;
  double rho = 1.0;
};

constexpr uint8_t FLUID = 0;
constexpr int VGROUPS = 4;
constexpr size_t NONE = std::numeric_limits<size_t>::max();

struct Builder {
  size_t nx, ny;
  bool periodic_x = false, periodic_y = false;
  double tau = 1.0;
  int collision = TRT;
  double magic = 3.0 / 16.0;
  double accel[2] = {0.0, 0.0};
  std::vector<Kind> kinds;
  std::vector<uint8_t> cell;
  std::string error;
};

struct Link {
  uint8_t dir, kind, vgroup;
  double q;
  size_t behind, fgroup;
  double uw[2], cu6, rho;
  int8_t normal[2];
  bool radiating;
};

struct BNode {
  size_t idx;
  size_t src[Q];
  size_t first, last;
};

struct PNode {
  size_t idx;
  int8_t nx, ny;
};

struct Sim {
  size_t nx, ny, n;
  bool periodic[2];
  std::vector<double> a, b;
  std::vector<uint8_t> flag;
  std::vector<BNode> bnodes;
  std::vector<Link> links;
  double op, om;
  int collision;
  double accel[2];
  std::unique_ptr<Pool> pool;
  double vscale[VGROUPS] = {1.0, 1.0, 1.0, 1.0};
  std::vector<double> force;  // [ngroups][2]
  bool has_target = false;
  double target = 0.0;
  double outlet_density_offset = 0.0;
  std::vector<PNode> pnodes;
  uint64_t t = 0;
  size_t fluid_nodes = 0;

  void init_fn(const std::function<void(size_t, size_t, double*)>& field);
  void step();
  void link_pass();
  void pops(size_t idx, double* f) const {
    for (int i = 0; i < Q; ++i) f[i] = a[i * n + idx];
  }
  void velocity_at(size_t idx, double* ux, double* uy) const {
    double f[Q], rho, jx, jy;
    pops(idx, f);
    moments(f, &rho, &jx, &jy);
    *ux = jx / rho - 0.5 * accel[0];
    *uy = jy / rho - 0.5 * accel[1];
  }
};

// src/sim.rs:219-354
static Sim* build_sim(Builder& bd, size_t threads) {
  size_t nx = bd.nx, ny = bd.ny, n = nx * ny;
  if (!(bd.tau > 0.5)) { bd.error = "tau must exceed 1/2 (viscosity must be positive)"; return nullptr; }
  auto wrap = [&](long x, long y, size_t* out) -> bool {
    if (x < 0 || x >= (long)nx) {
      if (!bd.periodic_x) return false;
      x = ((x % (long)nx) + (long)nx) % (long)nx;
    }
    if (y < 0 || y >= (long)ny) {
      if (!bd.periodic_y) return false;
      y = ((y % (long)ny) + (long)ny) % (long)ny;
    }
    *out = (size_t)y * nx + (size_t)x;
    return true;
  };
  auto s = std::make_unique<Sim>();
  s->flag.assign(n, 2);
  size_t ngroups = 0;
  for (size_t y = 0; y < ny; ++y) {
    for (size_t x = 0; x < nx; ++x) {
      size_t idx = y * nx + x;
      if (bd.cell[idx] != FLUID) continue;
      s->fluid_nodes += 1;
      size_t first = s->links.size();
      BNode bn;
      bn.idx = idx;
      for (int i = 0; i < Q; ++i) bn.src[i] = idx;
      for (int j = 1; j < Q; ++j) {
        long cx = CX[j], cy = CY[j];
        size_t target;
        if (!wrap((long)x + cx, (long)y + cy, &target)) {
          char buf[160];
          snprintf(buf, sizeof buf,
                   "fluid cell (%zu,%zu) touches a non-periodic edge; close the domain with wall or pressure cells",
                   x, y);
          bd.error = buf;
          return nullptr;
        }
        bn.src[OPP[j]] = target;
        uint8_t kind = bd.cell[target];
        if (kind == FLUID) continue;
        size_t bi;
        size_t behind = NONE;
        if (wrap((long)x - cx, (long)y - cy, &bi) && bd.cell[bi] == FLUID) behind = bi;
        Link l;
        l.dir = (uint8_t)j; l.kind = 0; l.vgroup = 0; l.q = 0.5; l.behind = behind;
        l.fgroup = NONE; l.uw[0] = 0.0; l.uw[1] = 0.0; l.cu6 = 0.0; l.rho = 1.0;
        l.normal[0] = 0; l.normal[1] = 0; l.radiating = false;
        const Kind& k = bd.kinds[kind];
        if (k.tag == K_PRESSURE || k.tag == K_RADIATING) {
          l.kind = 1;
          l.rho = k.rho;
          l.radiating = k.tag == K_RADIATING;
          size_t si;
          bool open = wrap((long)x + cx, (long)y, &si) &&
                      (bd.kinds[bd.cell[si]].tag == K_PRESSURE || bd.kinds[bd.cell[si]].tag == K_RADIATING);
          if (open) { l.normal[0] = (int8_t)cx; l.normal[1] = 0; }
          else { l.normal[0] = 0; l.normal[1] = (int8_t)cy; }
          if (!l.radiating && (s->pnodes.empty() || s->pnodes.back().idx != idx))
            s->pnodes.push_back(PNode{idx, l.normal[0], l.normal[1]});
        } else {
          if (k.vgroup >= VGROUPS) { bd.error = "vgroup out of range"; return nullptr; }
          l.vgroup = (uint8_t)k.vgroup;
          if (k.shape) l.q = cut_fraction(*k.shape, (double)x, (double)y, (double)cx, (double)cy);
          if (k.vel.kind != VEL_NONE) {
            double wx = (double)x + l.q * (double)cx, wy = (double)y + l.q * (double)cy;
            k.vel.eval(wx, wy, l.uw);
            l.cu6 = 6.0 * W[j] * ((double)cx * l.uw[0] + (double)cy * l.uw[1]);
          }
          if (k.fgroup >= 0) {
            l.fgroup = (size_t)k.fgroup;
            ngroups = std::max(ngroups, (size_t)k.fgroup + 1);
          }
        }
        s->links.push_back(l);
      }
      if (s->links.size() > first) {
        s->flag[idx] = 1;
        bn.first = first;
        bn.last = s->links.size();
        s->bnodes.push_back(bn);
      } else {
        s->flag[idx] = 0;
      }
    }
  }
  s->nx = nx; s->ny = ny; s->n = n;
  s->periodic[0] = bd.periodic_x; s->periodic[1] = bd.periodic_y;
  s->a.assign(Q * n, 0.0);
  s->b.assign(Q * n, 0.0);
  omegas(bd.collision, bd.magic, bd.tau, &s->op, &s->om);
  s->collision = bd.collision;
  s->accel[0] = bd.accel[0]; s->accel[1] = bd.accel[1];
  s->pool = std::make_unique<Pool>(threads);
  s->force.assign(2 * ngroups, 0.0);
  s->init_fn([](size_t, size_t, double* r) { r[0] = 1.0; r[1] = 0.0; r[2] = 0.0; });
  return s.release();
}

// src/sim.rs:357-371
void Sim::init_fn(const std::function<void(size_t, size_t, double*)>& field) {
  for (size_t y = 0; y < ny; ++y) {
    for (size_t x = 0; x < nx; ++x) {
      size_t idx = y * nx + x;
      double r[3];
      if (flag[idx] == 2) { r[0] = 1.0; r[1] = 0.0; r[2] = 0.0; }
      else field(x, y, r);
      double feq[Q];
      equilibrium(r[0], r[1], r[2], feq);
      for (int i = 0; i < Q; ++i) { a[i * n + idx] = feq[i]; b[i * n + idx] = feq[i]; }
    }
  }
  t = 0;
}

// src/sim.rs:700-735
template <class C>
static inline void row(const double* a, double* b, const uint8_t* flag, size_t n, size_t nx,
                       size_t ny, size_t y, const C& collide) {
  size_t ym = y == 0 ? ny - 1 : y - 1;
  size_t yp = y == ny - 1 ? 0 : y + 1;
  size_t base = y * nx, bm = ym * nx, bp = yp * nx;
  for (size_t x = 0; x < nx; ++x) {
    if (flag[base + x] != 0) continue;
    size_t xm = x == 0 ? nx - 1 : x - 1;
    size_t xp = x == nx - 1 ? 0 : x + 1;
    double f[Q] = {a[base + x],        a[n + base + xm],     a[2 * n + bm + x],
                   a[3 * n + base + xp], a[4 * n + bp + x],     a[5 * n + bm + xm],
                   a[6 * n + bm + xp],   a[7 * n + bp + xp],    a[8 * n + bp + xm]};
    double o[Q];
    collide(f, o);
    for (int i = 0; i < Q; ++i) b[i * n + base + x] = o[i];
  }
}

// src/sim.rs:391-420
void Sim::step() {
  double gx = accel[0], gy = accel[1];
  bool forced = gx != 0.0 || gy != 0.0;
  const double* pa = a.data();
  double* pb = b.data();
  const uint8_t* fl = flag.data();
  size_t nt = pool->threads();
  double op_ = op, om_ = om;
  int coll = collision;
  size_t n_ = n, nx_ = nx, ny_ = ny;
  pool->run([&](size_t th) {
    for (size_t y = th * ny_ / nt; y < (th + 1) * ny_ / nt; ++y) {
      if (forced)
        row(pa, pb, fl, n_, nx_, ny_, y,
            [&](const double* f, double* o) { collide_forced(f, op_, om_, gx, gy, o); });
      else if (coll == BGK)
        row(pa, pb, fl, n_, nx_, ny_, y, [&](const double* f, double* o) { collide_bgk(f, op_, o); });
      else
        row(pa, pb, fl, n_, nx_, ny_, y,
            [&](const double* f, double* o) { collide_trt(f, op_, om_, o); });
    }
  });
  link_pass();
  std::swap(a, b);
  t += 1;
}

// src/sim.rs:425-508
void Sim::link_pass() {
  double gx = accel[0], gy = accel[1];
  for (auto& v : force) v = 0.0;
  double drho = 0.0;
  if (has_target && !pnodes.empty()) {
    double sum = 0.0;
    for (auto& p : pnodes) {
      double ux, uy;
      velocity_at(p.idx, &ux, &uy);
      sum += (double)p.nx * ux + (double)p.ny * uy;
    }
    drho = (sum / (double)pnodes.size() - target) / std::sqrt(CS2);
  }
  outlet_density_offset = drho;
  for (auto& bn : bnodes) {
    size_t idx = bn.idx;
    double f[Q];
    for (int i = 0; i < Q; ++i) f[i] = a[i * n + bn.src[i]];
    for (size_t li = bn.first; li < bn.last; ++li) {
      const Link& l = links[li];
      int j = l.dir;
      int i = OPP[j];
      double out = a[j * n + idx];
      double scale = vscale[l.vgroup];
      double back;
      if (l.kind == 0) {
        double corr = l.cu6 * scale;
        if (l.q >= 0.5) {
          double k = 0.5 / l.q;
          back = k * (out - corr) + (1.0 - k) * a[i * n + idx];
        } else if (l.behind != NONE) {
          back = 2.0 * l.q * out + (1.0 - 2.0 * l.q) * a[j * n + l.behind] - corr;
        } else {
          back = out - corr;
        }
      } else {
        double ux, uy;
        velocity_at(idx, &ux, &uy);
        double cu = 3.0 * ((double)CX[j] * ux + (double)CY[j] * uy);
        double rho_w = l.radiating
                           ? l.rho + ((double)l.normal[0] * ux + (double)l.normal[1] * uy) / std::sqrt(CS2)
                           : l.rho + drho;
        back = -out + 2.0 * W[j] * rho_w * (1.0 + 0.5 * cu * cu - 1.5 * (ux * ux + uy * uy));
      }
      f[i] = back;
      if (l.fgroup != NONE) {
        double ux = l.uw[0] * scale, uy = l.uw[1] * scale;
        double* g = &force[2 * l.fgroup];
        g[0] += (double)CX[j] * (out + back) - ux * (out - back);
        g[1] += (double)CY[j] * (out + back) - uy * (out - back);
      }
    }
    double o[Q];
    if (gx != 0.0 || gy != 0.0) collide_forced(f, op, om, gx, gy, o);
    else if (collision == BGK) collide_bgk(f, op, o);
    else collide_trt(f, op, om, o);
    for (int i = 0; i < Q; ++i) b[i * n + idx] = o[i];
  }
}

// Kahan-Babuska-Neumaier summation (src/sim.rs:676-691)
struct Neumaier {
  double sum = 0.0, comp = 0.0;
  void add(double x) {
    double t = sum + x;
    comp += std::fabs(sum) >= std::fabs(x) ? (sum - t) + x : (x - t) + sum;
    sum = t;
  }
  double value() const { return sum + comp; }
};

// src/sim.rs:538-548
static double total_mass(const Sim& s) {
  Neumaier m;
  for (size_t idx = 0; idx < s.n; ++idx)
    if (s.flag[idx] != 2)
      for (int i = 0; i < Q; ++i) m.add(s.a[i * s.n + idx]);
  return m.value();
}

// src/sim.rs:551-563
static void total_momentum(const Sim& s, double* out) {
  Neumaier px, py;
  for (size_t idx = 0; idx < s.n; ++idx)
    if (s.flag[idx] != 2)
      for (int i = 1; i < Q; ++i) {
        double f = s.a[i * s.n + idx];
        px.add((double)CX[i] * f);
        py.add((double)CY[i] * f);
      }
  out[0] = px.value();
  out[1] = py.value();
}

// src/sim.rs:566-579
static double max_speed(const Sim& s) {
  double m = 0.0;
  for (size_t idx = 0; idx < s.n; ++idx) {
    if (s.flag[idx] == 2) continue;
    double ux, uy;
    s.velocity_at(idx, &ux, &uy);
    double v = std::sqrt(ux * ux + uy * uy);
    if (std::isnan(v)) return std::nan("");
    m = std::fmax(m, v);
  }
  return m;
}

// src/sim.rs:527-534
static void macros(const Sim& s, size_t x, size_t y, double* out) {
  size_t idx = y * s.nx + x;
  if (s.flag[idx] == 2) { out[0] = 1.0; out[1] = 0.0; out[2] = 0.0; return; }
  double f[Q], rho, jx, jy;
  s.pops(idx, f);
  moments(f, &rho, &jx, &jy);
  out[0] = rho;
  out[1] = jx / rho - 0.5 * s.accel[0];
  out[2] = jy / rho - 0.5 * s.accel[1];
}

// src/sim.rs:582-620
static void vorticity(const Sim& s, float* w) {
  size_t nx = s.nx, ny = s.ny;
  std::vector<double> ux(s.n, 0.0), uy(s.n, 0.0);
  for (size_t idx = 0; idx < s.n; ++idx)
    if (s.flag[idx] != 2) s.velocity_at(idx, &ux[idx], &uy[idx]);
  for (size_t i = 0; i < s.n; ++i) w[i] = 0.0f;
  auto fluid = [&](long x, long y) {
    return x >= 0 && y >= 0 && x < (long)nx && y < (long)ny && s.flag[(size_t)y * nx + (size_t)x] != 2;
  };
  for (long y = 0; y < (long)ny; ++y) {
    for (long x = 0; x < (long)nx; ++x) {
      if (!fluid(x, y)) continue;
      auto diff = [&](long dx, long dy, int comp) -> double {
        auto get = [&](long xx, long yy) {
          size_t k = (size_t)yy * nx + (size_t)xx;
          return comp == 0 ? ux[k] : uy[k];
        };
        bool p = fluid(x + dx, y + dy), m = fluid(x - dx, y - dy);
        if (p && m) return 0.5 * (get(x + dx, y + dy) - get(x - dx, y - dy));
        if (p) return get(x + dx, y + dy) - get(x, y);
        if (m) return get(x, y) - get(x - dx, y - dy);
        return 0.0;
      };
      w[(size_t)y * nx + (size_t)x] = (float)(diff(1, 0, 1) - diff(0, 1, 0));
    }
  }
}

// src/sim.rs:624-644
static double probe_density(const Sim& s, double x, double y) {
  double i = std::floor(x), j = std::floor(y);
  double fx = x - i, fy = y - j;
  double sum = 0.0, wsum = 0.0;
  const long di[4] = {0, 1, 0, 1}, dj[4] = {0, 0, 1, 1};
  const double w[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
  for (int k = 0; k < 4; ++k) {
    long xi = (long)i + di[k], yj = (long)j + dj[k];
    if (xi < 0 || yj < 0 || xi >= (long)s.nx || yj >= (long)s.ny) continue;
    size_t idx = (size_t)yj * s.nx + (size_t)xi;
    if (s.flag[idx] != 2 && w[k] > 0.0) {
      double f[Q], rho, jx, jy;
      s.pops(idx, f);
      moments(f, &rho, &jx, &jy);
      sum += w[k] * rho;
      wsum += w[k];
    }
  }
  return wsum > 0.0 ? sum / wsum : std::nan("");
}

// src/sim.rs:648-651
static double probe_density_at_wall(const Sim& s, double x, double y, double nx, double ny) {
  auto p = [&](double d) { return probe_density(s, x + d * nx, y + d * ny); };
  return 3.0 * p(1.0) - 3.0 * p(2.0) + p(3.0);
}

// src/sim.rs:654-668
static uint64_t state_hash(const Sim& s) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t idx = 0; idx < s.n; ++idx) {
    if (s.flag[idx] == 2) continue;
    for (int i = 0; i < Q; ++i) {
      uint64_t bits;
      double v = s.a[i * s.n + idx];
      std::memcpy(&bits, &v, 8);
      for (int k = 0; k < 8; ++k) {
        h ^= (bits >> (8 * k)) & 0xff;
        h *= 0x100000001b3ull;
      }
    }
  }
  return h;
}

// ---------------------------------------------------------------- cases
// src/cases/mod.rs:11-18
static double ramp(uint64_t t, uint64_t steps) {
  if (steps == 0 || t >= steps) return 1.0;
  double s = (double)t / (double)steps;
  return s * s * (3.0 - 2.0 * s);
}

enum Inflow { PARABOLIC = 0, UNIFORM = 1, UNIFORM_OPEN = 2 };

struct Kick {
  double cx, cy, omega;
  uint64_t start, duration;
};

struct Channel {
  std::unique_ptr<Sim> sim;
  uint64_t ramp_steps = 0;
  bool has_kick = false;
  Kick kick{};
  double u_ref = 0.0;
  bool absorbing_outlet = true;

  // src/cases/channel.rs:118-130
  void step() {
    uint64_t t = sim->t;
    sim->vscale[1] = ramp(t, ramp_steps);
    sim->has_target = absorbing_outlet;
    sim->target = u_ref * sim->vscale[1];
    double v2 = 0.0;
    if (has_kick && t >= kick.start && t < kick.start + kick.duration) {
      double s = (double)(t - kick.start) / (double)kick.duration;
      double sn = std::sin(M_PI * s);
      double sg = std::sin(2.0 * M_PI * s);
      v2 = kick.omega * (sn * sn) * std::copysign(1.0, sg);
    }
    sim->vscale[2] = v2;
    sim->step();
  }
};

// src/cases/channel.rs:71-116
static Channel* channel_new(size_t nx, size_t ny, int inflow, double u, double nu, int collision,
                            double magic, Shape* body, uint64_t ramp_steps, const Kick* kick,
                            size_t threads, std::string* err) {
  double h = (double)(ny - 2);
  Builder b;
  b.nx = nx; b.ny = ny;
  b.kinds.emplace_back();
  b.cell.assign(nx * ny, FLUID);
  b.tau = tau_for(nu);
  b.collision = collision;
  b.magic = magic;
  auto add = [&](Kind&& k) {
    b.kinds.push_back(std::move(k));
    return (uint8_t)(b.kinds.size() - 1);
  };
  auto fill = [&](size_t x0, size_t x1, size_t y0, size_t y1, uint8_t k) {
    for (size_t y = y0; y <= y1; ++y)
      for (size_t x = x0; x <= x1; ++x) b.cell[y * nx + x] = k;
  };
  Velocity prof;
  if (inflow == PARABOLIC) { prof.kind = VEL_PARABOLIC; prof.p[0] = u; prof.p[1] = h; }
  else { prof.kind = VEL_CONST; prof.p[0] = u; prof.p[1] = 0.0; }
  Kind inlet; inlet.tag = K_WALL; inlet.vel = prof; inlet.vgroup = 1;
  uint8_t k_in = add(std::move(inlet));
  Kind outlet; outlet.tag = K_PRESSURE; outlet.rho = 1.0;
  uint8_t k_out = add(std::move(outlet));
  Kind walls;
  if (inflow == PARABOLIC) { walls.tag = K_WALL; }
  else if (inflow == UNIFORM) {
    walls.tag = K_WALL; walls.vel.kind = VEL_CONST; walls.vel.p[0] = u; walls.vel.p[1] = 0.0; walls.vgroup = 1;
  } else { walls.tag = K_RADIATING; walls.rho = 1.0; }
  uint8_t k_w = add(std::move(walls));
  fill(0, 0, 0, ny - 1, k_in);
  fill(nx - 1, nx - 1, 0, ny - 1, k_out);
  fill(1, nx - 2, 0, 0, k_w);
  fill(1, nx - 2, ny - 1, ny - 1, k_w);
  if (inflow == PARABOLIC || inflow == UNIFORM) {
    fill(0, nx - 1, 0, 0, k_w);
    fill(0, nx - 1, ny - 1, ny - 1, k_w);
  }
  Kind bodyk; bodyk.tag = K_WALL; bodyk.vgroup = 2; bodyk.fgroup = 0;
  bodyk.shape.reset(body);
  if (kick) { bodyk.vel.kind = VEL_ROTATION; bodyk.vel.p[0] = kick->cx; bodyk.vel.p[1] = kick->cy; }
  uint8_t k_b = add(std::move(bodyk));
  {
    const Shape& sh = *b.kinds[k_b].shape;
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x)
        if (sh.inside((double)x, (double)y)) b.cell[y * nx + x] = k_b;
  }
  Sim* s = build_sim(b, threads);
  if (!s) { *err = b.error; return nullptr; }
  if (ramp_steps == 0) {
    Velocity pv = prof;
    s->init_fn([&](size_t, size_t y, double* r) {
      double uu[2];
      pv.eval(0.0, (double)y, uu);
      r[0] = 1.0; r[1] = uu[0]; r[2] = 0.0;
    });
  }
  auto ch = new Channel();
  ch->sim.reset(s);
  ch->ramp_steps = ramp_steps;
  if (kick) { ch->has_kick = true; ch->kick = *kick; }
  ch->u_ref = u;
  ch->absorbing_outlet = true;
  return ch;
}

// ---------------------------------------------------------------- signal (src/signal.rs)
static void fft(double* re, double* im, size_t n) {
  size_t j = 0;
  for (size_t i = 1; i < n; ++i) {
    size_t bit = n >> 1;
    while (j & bit) { j ^= bit; bit >>= 1; }
    j |= bit;
    if (i < j) { std::swap(re[i], re[j]); std::swap(im[i], im[j]); }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    double ang = -2.0 * M_PI / (double)len;
    double wr = std::cos(ang), wi = std::sin(ang);
    for (size_t start = 0; start < n; start += len) {
      double cr = 1.0, ci = 0.0;
      for (size_t k = 0; k < len / 2; ++k) {
        size_t a = start + k, b = start + k + len / 2;
        double tr = re[b] * cr - im[b] * ci, ti = re[b] * ci + im[b] * cr;
        re[b] = re[a] - tr;
        im[b] = im[a] - ti;
        re[a] += tr;
        im[a] += ti;
        double ncr = cr * wr - ci * wi;
        ci = cr * wi + ci * wr;
        cr = ncr;
      }
    }
  }
}

static double mean(const double* x, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += x[i];
  return s / (double)n;
}

static double rms(const double* x, size_t n) {
  double m = mean(x, n), s = 0.0;
  for (size_t i = 0; i < n; ++i) s += (x[i] - m) * (x[i] - m);
  return std::sqrt(s / (double)n);
}

static size_t next_pow2(size_t v) {
  size_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

// src/signal.rs:74-88
static std::vector<std::pair<double, double>> spectrum(const double* x, size_t n, double dt, size_t pad) {
  double m = mean(x, n);
  size_t size = next_pow2(n * std::max<size_t>(pad, 1));
  std::vector<double> re(size, 0.0), im(size, 0.0);
  for (size_t i = 0; i < n; ++i) {
    double w = 0.5 - 0.5 * std::cos(2.0 * M_PI * (double)i / (double)n);
    re[i] = (x[i] - m) * w;
  }
  fft(re.data(), im.data(), size);
  double scale = 4.0 / (double)n;
  std::vector<std::pair<double, double>> out(size / 2);
  for (size_t k = 0; k < size / 2; ++k)
    out[k] = {(double)k / ((double)size * dt), scale * std::sqrt(re[k] * re[k] + im[k] * im[k])};
  return out;
}

// src/signal.rs:92-107
static void dominant_frequency(const double* x, size_t n, double dt, double* f, double* amp) {
  auto s = spectrum(x, n, dt, 8);
  size_t k = 1;
  for (size_t i = 1; i + 1 < s.size(); ++i)
    if (s[i].second > s[k].second) k = i;
  if (k == 0 || k + 1 >= s.size() || s[k].second <= 0.0 || s[k - 1].second <= 0.0 ||
      s[k + 1].second <= 0.0) {
    *f = s[k].first; *amp = s[k].second;
    return;
  }
  double a = std::log(s[k - 1].second), b = std::log(s[k].second), c = std::log(s[k + 1].second);
  double shift = 0.5 * (a - c) / (a - 2.0 * b + c);
  double df = s[1].first - s[0].first;
  *f = s[k].first + shift * df;
  *amp = std::exp(b - 0.25 * (a - c) * shift);
}

// src/signal.rs:111-123
static size_t peaks(const double* x, size_t n, double* pos, double* val, size_t cap) {
  double m = mean(x, n);
  size_t cnt = 0;
  for (size_t i = 1; i + 1 < n; ++i) {
    if (x[i] > m && x[i] > x[i - 1] && x[i] >= x[i + 1]) {
      double a = x[i - 1], b = x[i], c = x[i + 1];
      double denom = a - 2.0 * b + c;
      double shift = denom != 0.0 ? 0.5 * (a - c) / denom : 0.0;
      if (cnt < cap) { pos[cnt] = (double)i + shift; val[cnt] = b - 0.25 * (a - c) * shift; }
      ++cnt;
    }
  }
  return cnt;
}

// src/signal.rs:127-140
static bool crossing_frequency(const double* x, size_t n, double dt, double* out) {
  double m = mean(x, n);
  std::vector<double> times;
  for (size_t i = 1; i < n; ++i) {
    double a = x[i - 1] - m, b = x[i] - m;
    if (a < 0.0 && b >= 0.0) times.push_back((double)(i - 1) + a / (a - b));
  }
  if (times.size() < 2) return false;
  *out = (double)(times.size() - 1) / ((times.back() - times.front()) * dt);
  return true;
}

// src/signal.rs:143-147
static double sample_at(const double* x, size_t n, double pos) {
  size_t i = std::min((size_t)std::floor(pos), n - 2);
  double f = pos - (double)i;
  return x[i] * (1.0 - f) + x[i + 1] * f;
}

}  // namespace vlo

// ================================================================ C API (ctypes)
using namespace vlo;

static thread_local std::string g_err;

extern "C" {

const char* vlo_last_error() { return g_err.c_str(); }

// ---- lattice unit functions
void vlo_equilibrium(double rho, double ux, double uy, double* out) { equilibrium(rho, ux, uy, out); }
void vlo_moments(const double* f, double* out) { moments(f, &out[0], &out[1], &out[2]); }
void vlo_collide_bgk(const double* f, double omega, double* out) { collide_bgk(f, omega, out); }
void vlo_collide_trt(const double* f, double op, double om, double* out) { collide_trt(f, op, om, out); }
void vlo_collide_forced(const double* f, double op, double om, double gx, double gy, double* out) {
  collide_forced(f, op, om, gx, gy, out);
}
void vlo_omegas(int coll, double magic, double tau, double* out) { omegas(coll, magic, tau, &out[0], &out[1]); }
double vlo_tau_for(double nu) { return tau_for(nu); }

// ---- shapes (the returned handle owns the shape; wrappers take ownership of `inner`)
void* vlo_shape_circle(double cx, double cy, double r) {
  auto s = new Circle(); s->cx = cx; s->cy = cy; s->r = r; return (Shape*)s;
}
void* vlo_shape_polygon(const double* xy, int n) {
  auto s = new Polygon();
  for (int i = 0; i < n; ++i) { s->px.push_back(xy[2 * i]); s->py.push_back(xy[2 * i + 1]); }
  return (Shape*)s;
}
void* vlo_shape_rounded_square(double cx, double cy, double half, double r) {
  auto s = new RoundedSquare(); s->cx = cx; s->cy = cy; s->half = half; s->r = r; return (Shape*)s;
}
void* vlo_shape_rotated(void* inner, double cx, double cy, double angle) {
  auto s = new Rotated(); s->inner.reset((Shape*)inner); s->cx = cx; s->cy = cy; s->angle = angle;
  return (Shape*)s;
}
void* vlo_shape_translated(void* inner, double dx, double dy) {
  auto s = new Translated(); s->inner.reset((Shape*)inner); s->dx = dx; s->dy = dy; return (Shape*)s;
}
void* vlo_shape_outside_band(double y0, double y1) {
  auto s = new OutsideBand(); s->y0 = y0; s->y1 = y1; return (Shape*)s;
}
// The star-convex polygon of the batched-tunnel workload (no counterpart in the reference's
// shapes): vertex k at angle phase + 2 pi k / n, distance radii[k] from (cx, cy).
void* vlo_shape_star(double cx, double cy, const double* radii, int n, double phase) {
  auto s = new Polygon();
  for (int k = 0; k < n; ++k) {
    const double th = phase + 2.0 * M_PI * (double)k / (double)n;
    s->px.push_back(cx + radii[k] * std::cos(th));
    s->py.push_back(cy + radii[k] * std::sin(th));
  }
  return (Shape*)s;
}
void* vlo_shape_ellipse(double cx, double cy, double a, double b) {
  auto s = new Ellipse(); s->cx = cx; s->cy = cy; s->a = a; s->b = b; return (Shape*)s;
}
void* vlo_shape_section(int corner, double b, double cx, double cy, double d, double angle) {
  return (Shape*)section(corner, b, cx, cy, d, angle).release();
}
void* vlo_shape_bitmap(size_t w, size_t h, const float* level, double x0, double y0, double scale) {
  auto s = new Bitmap(); s->w = w; s->h = h; s->level.assign(level, level + w * h);
  s->x0 = x0; s->y0 = y0; s->scale = scale; return (Shape*)s;
}
void* vlo_shape_disks(const double* cxcyr, size_t n) {
  auto s = new DiskUnion();
  for (size_t k = 0; k < n; ++k) { s->cx.push_back(cxcyr[3 * k]); s->cy.push_back(cxcyr[3 * k + 1]); s->r.push_back(cxcyr[3 * k + 2]); }
  s->prepare();
  return (Shape*)s;
}
void vlo_shape_free(void* s) { delete (Shape*)s; }
int vlo_shape_inside(void* s, double x, double y) { return ((Shape*)s)->inside(x, y) ? 1 : 0; }
double vlo_cut_fraction(void* s, double x, double y, double dx, double dy) {
  return cut_fraction(*(Shape*)s, x, y, dx, dy);
}
int vlo_bounding_box(void* s, double reach, double step, double* out) {
  return bounding_box(*(Shape*)s, reach, step, out) ? 1 : 0;
}

// ---- builder (src/sim.rs:84-136)
void* vlo_builder_new(size_t nx, size_t ny) {
  if (nx < 3 || ny < 3) { g_err = "grid must be at least 3 x 3"; return nullptr; }
  auto b = new Builder();
  b->nx = nx; b->ny = ny;
  b->kinds.emplace_back();
  b->cell.assign(nx * ny, FLUID);
  return b;
}
void vlo_builder_free(void* b) { delete (Builder*)b; }
void vlo_builder_config(void* bp, int px, int py, double tau, int coll, double magic, double gx, double gy) {
  auto b = (Builder*)bp;
  b->periodic_x = px != 0; b->periodic_y = py != 0; b->tau = tau; b->collision = coll;
  b->magic = magic; b->accel[0] = gx; b->accel[1] = gy;
}
static int add_kind(Builder* b, Kind&& k) {
  if (b->kinds.size() >= 255) { g_err = "too many kinds"; return -1; }
  b->kinds.push_back(std::move(k));
  return (int)b->kinds.size() - 1;
}
// vel: kind + 4 params; fgroup < 0 = none; shape may be NULL (ownership taken).
int vlo_builder_add_wall(void* bp, int vel_kind, const double* vel, int vgroup, long fgroup, void* shape) {
  Kind k; k.tag = K_WALL; k.vel.kind = vel_kind;
  if (vel) for (int i = 0; i < 4; ++i) k.vel.p[i] = vel[i];
  k.vgroup = vgroup; k.fgroup = fgroup; k.shape.reset((Shape*)shape);
  return add_kind((Builder*)bp, std::move(k));
}
int vlo_builder_add_pressure(void* bp, double rho) {
  Kind k; k.tag = K_PRESSURE; k.rho = rho; return add_kind((Builder*)bp, std::move(k));
}
int vlo_builder_add_radiating(void* bp, double rho) {
  Kind k; k.tag = K_RADIATING; k.rho = rho; return add_kind((Builder*)bp, std::move(k));
}
void vlo_builder_fill_rect(void* bp, size_t x0, size_t x1, size_t y0, size_t y1, int kind) {
  auto b = (Builder*)bp;
  for (size_t y = y0; y <= y1; ++y)
    for (size_t x = x0; x <= x1; ++x) b->cell[y * b->nx + x] = (uint8_t)kind;
}
int vlo_builder_fill_shape(void* bp, int kind) {
  auto b = (Builder*)bp;
  const Kind& k = b->kinds[kind];
  if (k.tag != K_WALL || !k.shape) { g_err = "fill_shape needs a wall kind with an outline"; return -1; }
  for (size_t y = 0; y < b->ny; ++y)
    for (size_t x = 0; x < b->nx; ++x)
      if (k.shape->inside((double)x, (double)y)) b->cell[y * b->nx + x] = (uint8_t)kind;
  return 0;
}
// Consumes the builder (freed whether or not the build succeeds).
void* vlo_sim_build(void* bp, size_t threads) {
  auto b = (Builder*)bp;
  Sim* s = build_sim(*b, threads);
  if (!s) g_err = b->error;
  delete b;
  return s;
}

// ---- sim
void vlo_sim_free(void* s) { delete (Sim*)s; }
size_t vlo_sim_nx(void* s) { return ((Sim*)s)->nx; }
size_t vlo_sim_ny(void* s) { return ((Sim*)s)->ny; }
size_t vlo_sim_fluid_nodes(void* s) { return ((Sim*)s)->fluid_nodes; }
size_t vlo_sim_link_count(void* s) { return ((Sim*)s)->links.size(); }
size_t vlo_sim_bnode_count(void* s) { return ((Sim*)s)->bnodes.size(); }
size_t vlo_sim_pnode_count(void* s) { return ((Sim*)s)->pnodes.size(); }
size_t vlo_sim_threads(void* s) { return ((Sim*)s)->pool->threads(); }
// Replaces the worker pool (the same row split over another thread count; results do not depend
// on it, tests/solver.rs:270-291).
void vlo_sim_set_threads(void* s, size_t threads) { ((Sim*)s)->pool = std::make_unique<Pool>(threads); }
int vlo_sim_ngroups(void* s) { return (int)(((Sim*)s)->force.size() / 2); }
uint64_t vlo_sim_t(void* s) { return ((Sim*)s)->t; }
void vlo_sim_flags(void* s, uint8_t* out) {
  auto p = (Sim*)s; std::memcpy(out, p->flag.data(), p->n);
}
// Field init from arrays of n = nx*ny values (x fastest).
// Link list of Sim::from_builder in the same encoding as the product's vl_builder_link_table.
void vlo_sim_link_table(void* sp, int32_t* bnode_idx, int32_t* bnode_first, double* link_f64, int32_t* link_i32) {
  auto s = (Sim*)sp;
  for (size_t k = 0; k < s->bnodes.size(); ++k) {
    if (bnode_idx) bnode_idx[k] = (int32_t)s->bnodes[k].idx;
    if (bnode_first) { bnode_first[k] = (int32_t)s->bnodes[k].first; bnode_first[k + 1] = (int32_t)s->bnodes[k].last; }
  }
  for (size_t k = 0; k < s->links.size(); ++k) {
    const Link& L = s->links[k];
    if (link_f64) {
      double* o = link_f64 + 5 * k;
      o[0] = L.q; o[1] = L.cu6; o[2] = L.uw[0]; o[3] = L.uw[1]; o[4] = L.rho;
    }
    if (link_i32) {
      int32_t* o = link_i32 + 7 * k;
      o[0] = L.dir; o[1] = L.kind; o[2] = L.radiating ? 1 : 0; o[3] = L.vgroup;
      o[4] = L.fgroup == NONE ? -1 : (int32_t)L.fgroup;
      o[5] = L.behind == NONE ? -1 : (int32_t)L.behind;
      o[6] = L.normal[0] + 3 * (L.normal[1] + 1) + 1;
    }
  }
}
void vlo_sim_init_arrays(void* sp, const double* rho, const double* ux, const double* uy) {
  auto s = (Sim*)sp;
  s->init_fn([&](size_t x, size_t y, double* r) {
    size_t k = y * s->nx + x;
    r[0] = rho[k]; r[1] = ux[k]; r[2] = uy[k];
  });
}
void vlo_sim_step(void* sp, uint64_t steps) {
  auto s = (Sim*)sp;
  for (uint64_t k = 0; k < steps; ++k) s->step();
}
void vlo_sim_set_vscale(void* sp, int g, double v) { ((Sim*)sp)->vscale[g] = v; }
double vlo_sim_get_vscale(void* sp, int g) { return ((Sim*)sp)->vscale[g]; }
void vlo_sim_set_outflow_target(void* sp, int has, double v) {
  auto s = (Sim*)sp; s->has_target = has != 0; s->target = v;
}
double vlo_sim_outlet_density_offset(void* sp) { return ((Sim*)sp)->outlet_density_offset; }
void vlo_sim_force(void* sp, double* out) {
  auto s = (Sim*)sp; std::memcpy(out, s->force.data(), s->force.size() * sizeof(double));
}
void vlo_sim_get_f(void* sp, double* out) {
  auto s = (Sim*)sp; std::memcpy(out, s->a.data(), s->a.size() * sizeof(double));
}
void vlo_sim_set_f(void* sp, const double* in) {
  auto s = (Sim*)sp; std::memcpy(s->a.data(), in, s->a.size() * sizeof(double));
}
void vlo_sim_macros(void* sp, size_t x, size_t y, double* out) { macros(*(Sim*)sp, x, y, out); }
double vlo_sim_total_mass(void* sp) { return total_mass(*(Sim*)sp); }
void vlo_sim_total_momentum(void* sp, double* out) { total_momentum(*(Sim*)sp, out); }
double vlo_sim_max_speed(void* sp) { return max_speed(*(Sim*)sp); }
void vlo_sim_vorticity(void* sp, float* out) { vorticity(*(Sim*)sp, out); }
double vlo_sim_probe_density(void* sp, double x, double y) { return probe_density(*(Sim*)sp, x, y); }
double vlo_sim_probe_density_at_wall(void* sp, double x, double y, double nx, double ny) {
  return probe_density_at_wall(*(Sim*)sp, x, y, nx, ny);
}
uint64_t vlo_sim_state_hash(void* sp) { return state_hash(*(Sim*)sp); }
double vlo_ramp(uint64_t t, uint64_t steps) { return ramp(t, steps); }

// ---- channel (src/cases/channel.rs); kick = {cx, cy, omega, start, duration} or NULL
void* vlo_channel_new(size_t nx, size_t ny, int inflow, double u, double nu, int coll, double magic,
                      void* body, uint64_t ramp_steps, const double* kick, size_t threads) {
  Kick k{};
  if (kick) { k.cx = kick[0]; k.cy = kick[1]; k.omega = kick[2]; k.start = (uint64_t)kick[3]; k.duration = (uint64_t)kick[4]; }
  std::string err;
  Channel* ch = channel_new(nx, ny, inflow, u, nu, coll, magic, (Shape*)body, ramp_steps, kick ? &k : nullptr, threads, &err);
  if (!ch) g_err = err;
  return ch;
}
void vlo_channel_free(void* c) { delete (Channel*)c; }
void* vlo_channel_sim(void* c) { return ((Channel*)c)->sim.get(); }
void vlo_channel_set_absorbing(void* c, int on) { ((Channel*)c)->absorbing_outlet = on != 0; }
double vlo_channel_u_ref(void* c) { return ((Channel*)c)->u_ref; }
// Runs `steps` Channel::step calls. If `force_hist` is non-null it receives force[0] (fx, fy)
// after each step. If `dp_hist` is non-null it receives the cylinder pressure drop of
// src/cases/cylinder.rs:54-59 for a body centred at (xc, yc) with radius r.
void vlo_channel_run(void* c, uint64_t steps, double* force_hist, double* dp_hist, double xc,
                     double yc, double r) {
  auto ch = (Channel*)c;
  for (uint64_t k = 0; k < steps; ++k) {
    ch->step();
    if (force_hist) {
      if (ch->sim->force.size() >= 2) { force_hist[2 * k] = ch->sim->force[0]; force_hist[2 * k + 1] = ch->sim->force[1]; }
      else { force_hist[2 * k] = 0.0; force_hist[2 * k + 1] = 0.0; }
    }
    if (dp_hist) {
      double front = probe_density_at_wall(*ch->sim, xc - r, yc, -1.0, 0.0);
      double back = probe_density_at_wall(*ch->sim, xc + r, yc, 1.0, 0.0);
      dp_hist[k] = CS2 * (front - back) / (ch->u_ref * ch->u_ref);
    }
  }
}

// ---- signal
void vlo_fft(double* re, double* im, size_t n) { fft(re, im, n); }
double vlo_mean(const double* x, size_t n) { return mean(x, n); }
double vlo_rms(const double* x, size_t n) { return rms(x, n); }
void vlo_dominant_frequency(const double* x, size_t n, double dt, double* out) {
  dominant_frequency(x, n, dt, &out[0], &out[1]);
}
size_t vlo_peaks(const double* x, size_t n, double* pos, double* val, size_t cap) {
  return peaks(x, n, pos, val, cap);
}
int vlo_crossing_frequency(const double* x, size_t n, double dt, double* out) {
  return crossing_frequency(x, n, dt, out) ? 1 : 0;
}
double vlo_sample_at(const double* x, size_t n, double pos) { return sample_at(x, n, pos); }

}  // extern "C"
