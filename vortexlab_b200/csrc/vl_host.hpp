// Host-side model of a vortexlab domain: shapes, wall kinds, the cell painter and the compiler
// that turns painted cells into the device tables the step kernels read.
//
// Everything here runs once per domain on the host. The arithmetic that decides link geometry
// (cut fractions, wall velocities, the 6 w (c . u_w) correction) follows the reference operation
// by operation so that the uploaded tables are bit-identical to the reference's link list
// (src/sim.rs:219-354); the layout of those tables is this project's own (packed 48-byte link
// records, int32 indices, boundary nodes as a CSR list).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "vl_lattice.hpp"

namespace vl {

// ------------------------------------------------------------------ shapes (src/geometry.rs)
struct Shape {
  virtual ~Shape() = default;
  virtual bool inside(double x, double y) const = 0;
};

// src/geometry.rs:16-27
struct CircleShape final : Shape {
  double cx, cy, r;
  CircleShape(double cx_, double cy_, double r_) : cx(cx_), cy(cy_), r(r_) {}
  bool inside(double x, double y) const override {
    const double dx = x - cx, dy = y - cy;
    return dx * dx + dy * dy < r * r;
  }
};

// src/geometry.rs:30-49 (even-odd rule)
struct PolygonShape final : Shape {
  std::vector<double> vx, vy;
  bool inside(double x, double y) const override {
    const size_t n = vx.size();
    bool in = false;
    for (size_t i = 0, j = n - 1; i < n; j = i++) {
      const double xi = vx[i], yi = vy[i], xj = vx[j], yj = vy[j];
      if ((yi > y) != (yj > y) && x < (xj - xi) * (y - yi) / (yj - yi) + xi) in = !in;
    }
    return in;
  }
};

// src/geometry.rs:52-66
struct RoundedSquareShape final : Shape {
  double cx, cy, half, r;
  bool inside(double x, double y) const override {
    const double ax = std::fabs(x - cx), ay = std::fabs(y - cy);
    const double core = half - r;
    const double dx = std::fmax(ax - core, 0.0), dy = std::fmax(ay - core, 0.0);
    return ax < half && ay < half && dx * dx + dy * dy < r * r;
  }
};

// src/geometry.rs:69-82
struct RotatedShape final : Shape {
  std::unique_ptr<Shape> inner;
  double cx, cy, angle;
  bool inside(double x, double y) const override {
    const double s = std::sin(angle), c = std::cos(angle);
    const double dx = x - cx, dy = y - cy;
    return inner->inside(cx + c * dx + s * dy, cy - s * dx + c * dy);
  }
};

// src/geometry.rs:85-95
struct TranslatedShape final : Shape {
  std::unique_ptr<Shape> inner;
  double dx, dy;
  bool inside(double x, double y) const override { return inner->inside(x - dx, y - dy); }
};

// src/cases/poiseuille.rs:12-21
struct OutsideBandShape final : Shape {
  double y0, y1;
  bool inside(double, double y) const override { return y <= y0 || y >= y1; }
};

// Axis-aligned ellipse (batched-tunnel bodies; no reference counterpart).
struct EllipseShape final : Shape {
  double cx, cy, a, b;
  bool inside(double x, double y) const override {
    const double u = (x - cx) / a, v = (y - cy) / b;
    return u * u + v * v < 1.0;
  }
};

// src/geometry.rs:120-185: 0.5 contour of a bilinearly interpolated grey-level picture.
struct BitmapShape final : Shape {
  size_t w = 0, h = 0;
  std::vector<float> level;
  double x0 = 0, y0 = 0, scale = 1;
  double pixel(long i, long j) const {
    if (i < 0 || j < 0 || i >= (long)w || j >= (long)h) return 0.0;
    return (double)level[(size_t)j * w + (size_t)i];
  }
  bool inside(double x, double y) const override {
    const double px = (x - x0) / scale - 0.5;
    const double py = (double)h - (y - y0) / scale - 0.5;
    const double fi = std::floor(px), fj = std::floor(py);
    const double fx = px - fi, fy = py - fj;
    const long i = (long)fi, j = (long)fj;
    const double v = (1.0 - fx) * (1.0 - fy) * pixel(i, j) + fx * (1.0 - fy) * pixel(i + 1, j) +
                     (1.0 - fx) * fy * pixel(i, j + 1) + fx * fy * pixel(i + 1, j + 1);
    return v > 0.5;
  }
};

// Union of many disks (the solid obstacles of the periodic throughput box). A point is inside if
// any disk contains it, with the disk test of CircleShape; disks are bucketed on a coarse grid so
// that a query looks at the few disks near the point only. The answer does not depend on the
// bucketing or on the disk order.
struct DiskUnionShape final : Shape {
  std::vector<double> cx, cy, r;
  double cell = 32.0;
  long gx0 = 0, gy0 = 0, gw = 0, gh = 0;
  std::vector<std::vector<int32_t>> bucket;
  void index();
  bool inside(double x, double y) const override;
};

std::unique_ptr<Shape> make_section(int corner, double b, double cx, double cy, double d, double angle);
std::unique_ptr<Shape> make_star(double cx, double cy, const double* radii, size_t nvert, double phase);
double cut_fraction(const Shape& s, double x, double y, double dx, double dy);
bool bounding_box(const Shape& s, double reach, double step, double* out);

// ------------------------------------------------------------------ wall velocity
enum { VEL_NONE = 0, VEL_CONST = 1, VEL_PARABOLIC = 2, VEL_ROTATION = 3 };
struct WallVelocity {
  int kind = VEL_NONE;
  double p[4] = {0, 0, 0, 0};
  void at(double x, double y, double& ux, double& uy) const;
};

// ------------------------------------------------------------------ cell kinds / builder
enum KindTag : uint8_t { KIND_FLUID = 0, KIND_WALL = 1, KIND_PRESSURE = 2, KIND_RADIATING = 3 };
struct CellKind {
  KindTag tag = KIND_FLUID;
  WallVelocity velocity;
  int vgroup = 0;
  int fgroup = -1;
  std::unique_ptr<Shape> shape;
  double rho = 1.0;
};

struct DomainSpec {
  size_t nx = 0, ny = 0;
  bool periodic_x = false, periodic_y = false;
  double tau = 1.0;
  int collision = COLL_TRT;
  double magic = 3.0 / 16.0;
  double accel[2] = {0.0, 0.0};
  std::vector<CellKind> kinds;   // kinds[0] is fluid
  std::vector<uint8_t> paint;    // kind id per cell
};

// ------------------------------------------------------------------ compiled domain
// One boundary link as the device reads it. 48 bytes, 16-byte aligned, loaded as three 16-byte
// vectors by the link kernel.
struct alignas(16) LinkRec {
  double q;       // fraction of the link in the fluid
  double cu6;     // 6 w_j (c_j . u_w) at unit velocity scale
  double uw[2];   // wall velocity at unit scale
  double rho;     // pressure links: boundary density
  int32_t behind; // fluid node one step away from the wall, -1 if none
  uint8_t dir;    // direction j from the node into the boundary
  uint8_t flags;  // bit0 pressure link, bit1 radiating, bits2-3 normal_x+1, bits4-5 normal_y+1
  uint8_t vgroup;
  int8_t fgroup;  // -1: no force bookkeeping
};
static_assert(sizeof(LinkRec) == 48, "LinkRec layout");

struct CompiledDomain {
  size_t nx = 0, ny = 0, n = 0;
  bool periodic_x = false, periodic_y = false;
  int collision = COLL_TRT;
  double op = 1.0, om = 1.0;
  double accel[2] = {0.0, 0.0};
  std::vector<uint8_t> flag;        // 0 interior fluid, 1 boundary fluid, 2 not fluid
  std::vector<int32_t> bnode_idx;   // boundary nodes in y-major, x order
  std::vector<int32_t> bnode_first; // CSR offsets into links (size nb + 1)
  std::vector<LinkRec> links;       // y-major, x, direction 1..8 order
  std::vector<int32_t> pnode_idx;   // non-radiating pressure-boundary nodes (deduplicated)
  std::vector<int8_t> pnode_nx, pnode_ny;
  size_t fluid_nodes = 0;
  int ngroups = 0;
};

// Compiles the painted domain (src/sim.rs:219-354). Returns false with `err` set on a contract
// violation (tau <= 1/2, fluid on a non-periodic edge, vgroup out of range, too many groups).
bool compile_domain(const DomainSpec& spec, CompiledDomain& out, std::string& err);

// ------------------------------------------------------------------ channel plan
// Host decisions of Channel::new / Channel::step (src/cases/channel.rs:71-130).
struct ChannelPlan {
  CompiledDomain dom;
  double u_ref = 0.0;
  bool init_profile = false;        // ramp_steps == 0: start from the inflow profile
  WallVelocity profile;
  uint64_t sched_len = 0;           // steps with a non-constant control
  std::vector<double> sched;        // per step: inlet ramp, body kick
};

// ------------------------------------------------------------------ signal (src/signal.rs)
void fft_inplace(double* re, double* im, size_t n);
double series_mean(const double* x, size_t n);
double series_rms(const double* x, size_t n);
void dominant_frequency(const double* x, size_t n, double dt, double& freq, double& amp);
size_t find_peaks(const double* x, size_t n, double* pos, double* val, size_t cap);
bool crossing_frequency(const double* x, size_t n, double dt, double& out);
double sample_at(const double* x, size_t n, double pos);

}  // namespace vl
