/*
 * vortexlab-b200 — C ABI of the B200-native D2Q9 lattice-Boltzmann time step.
 *
 * The reference (vortexlab, Rust) has no FFI: its boundary is the Rust `Builder` / `Sim` /
 * `Channel` API that its cases and tests call. Every entry point below replaces one item of that
 * API; the comment gives the reference item it replaces (file:line in the reference project).
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, doubles. Host arrays are row-major with x fastest
 *    (cell index idx = y * nx + x), as in the reference (src/sim.rs:251).
 *  - Population arrays exchanged with the host use the reference layout: population i of cell idx
 *    at i * n + idx, n = nx * ny (src/sim.rs:335-336). The device layout pads each population
 *    plane to a 64-element boundary; that padding never crosses this ABI.
 *  - Every function that can fail returns an int status: VL_OK (0) or a negative VL_E* code,
 *    with a message from vl_last_error() (thread-local). Where the reference panics on a contract
 *    violation (src/sim.rs:85, :101, :222, :261, :303) this ABI returns VL_EINVAL instead; it
 *    never aborts the process. Constructors return NULL on failure.
 *  - One vl_sim is driven from one host thread; it owns one CUDA stream on the device that was
 *    current when it was built. There is no CPU fallback: without a CUDA device every vl_sim
 *    constructor fails with VL_ECUDA.
 */
#ifndef VORTEXLAB_H
#define VORTEXLAB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VL_ABI_VERSION 2

/* ---- status codes */
#define VL_OK 0
#define VL_EINVAL (-1)       /* contract violation (the reference panics)                      */
#define VL_ECUDA (-2)        /* CUDA runtime error or no CUDA device                           */
#define VL_EDIVERGED (-3)    /* non-finite force: src/cases/cylinder.rs:179-186, tunnel.rs:78-84.
                              * The step functions, like Sim::step, do not fail on divergence: they
                              * record it on the device (vl_sim_status, vl_batch_status), and the
                              * case drivers raise this code, as the reference's cases return Err. */
#define VL_ENOMEM (-4)       /* device or host allocation failed                               */
#define VL_EUNSUPPORTED (-5) /* valid request that this build does not implement               */

/* ---- enums */
enum { VL_BGK = 0, VL_TRT = 1 };                              /* src/lattice.rs:28-35 */
/* population storage: FP64; FP32; IEEE FP16 of f_i - w_i; 16-bit f_i - w_i with a sign, a 3-bit
 * exponent and a 12-bit mantissa (2^(e-9) (1 + m/4096), evenly spaced by 2^-20 below 2^-8,
 * saturating at 0.49994); 16-bit fixed point of f_i - w_i (steps 2^-19 for the rest population
 * and the diagonals, 2^-18 for the axis directions, saturating at +-0.0625 / +-0.125). The
 * narrow formats collide in FP32 and sum forces in FP64; the saturating ones report a density
 * leaving 1 +- 1/2 as divergence. */
enum { VL_F64 = 0, VL_F32 = 1, VL_F16S = 2, VL_F16C = 3, VL_F16X = 4 };
enum { VL_VEL_NONE = 0, VL_VEL_CONST = 1, VL_VEL_PARABOLIC = 2, VL_VEL_ROTATION = 3 };
enum { VL_CORNER_SHARP = 0, VL_CORNER_CHAMFERED = 1, VL_CORNER_ROUNDED = 2,
       VL_CORNER_RECESSED = 3, VL_CORNER_DOUBLE_RECESSED = 4 }; /* src/geometry.rs:188-201 */
enum { VL_INFLOW_PARABOLIC = 0, VL_INFLOW_UNIFORM = 1, VL_INFLOW_UNIFORM_OPEN = 2 }; /* channel.rs:22-33 */

#define VL_VGROUPS 4   /* src/sim.rs:67 */
#define VL_MAX_FGROUPS 4  /* force groups per sim (the reference has no limit; see vl_builder_add_wall) */

typedef struct vl_shape vl_shape;
typedef struct vl_builder vl_builder;
typedef struct vl_sim vl_sim;
typedef struct vl_channel vl_channel;

/* Wall velocity as tagged data; replaces the closure `VelocityFn` (src/sim.rs:34), which C
 * cannot carry. The forms are exactly the closures the reference's cases build:
 *   VL_VEL_CONST      p = {ux, uy}              -> [ux, uy]
 *   VL_VEL_PARABOLIC  p = {u_mean, h}           -> [6 u_mean s (h - s) / h^2, 0], s = clamp(y - 1/2, 0, h)
 *                                                  (src/cases/channel.rs:77-86)
 *   VL_VEL_ROTATION   p = {cx, cy}              -> [-(y - cy), x - cx] (src/cases/channel.rs:104) */
typedef struct {
  int kind;
  double p[4];
} vl_velocity;

/* src/sim.rs:38-49 (`Wall`). fgroup < 0 means no force bookkeeping. `shape` (may be NULL) is
 * owned by the builder after vl_builder_add_wall returns, whether or not the call succeeds. */
typedef struct {
  vl_velocity velocity;
  int vgroup;
  int fgroup;
  vl_shape* shape;
} vl_wall;

const char* vl_last_error(void);
/* Status code of the last failure on this thread (for constructors, which return NULL). */
int vl_last_status(void);
int vl_abi_version(void);
/* Number of CUDA devices visible (0 on a machine without GPU). */
int vl_device_count(void);
/* Makes `device` current for this host thread; sims built afterwards live on it. */
int vl_set_device(int device);
/* Page-locked host buffers (for fast, asynchronous host<->device copies); NULL on failure. */
void* vl_pinned_alloc(size_t bytes);
void vl_pinned_free(void* p);

/* ================================================================ shapes: src/geometry.rs */
vl_shape* vl_shape_circle(double cx, double cy, double r);                 /* :16-27  */
vl_shape* vl_shape_polygon(const double* xy, size_t npts);                 /* :30-49, xy = x0,y0,x1,y1,... */
vl_shape* vl_shape_rounded_square(double cx, double cy, double half, double r); /* :52-66 */
vl_shape* vl_shape_rotated(vl_shape* inner, double cx, double cy, double angle); /* :69-82, takes inner */
vl_shape* vl_shape_translated(vl_shape* inner, double dx, double dy);      /* :85-95, takes inner */
vl_shape* vl_shape_section(int corner, double b, double cx, double cy, double d, double angle); /* :251-261 */
vl_shape* vl_shape_bitmap(size_t w, size_t h, const float* level, double x0, double y0, double scale); /* :120-185 */
vl_shape* vl_shape_outside_band(double y0, double y1);                     /* src/cases/poiseuille.rs:12-21 */
/* New body classes for the batched tunnels (no reference counterpart). */
vl_shape* vl_shape_ellipse(double cx, double cy, double a, double b);
vl_shape* vl_shape_star(double cx, double cy, const double* radii, size_t nvert, double phase);
/* Union of disks given as (cx, cy, r) triples: inside if any disk contains the point (the disk
 * test of Circle, src/geometry.rs:22-27). Used for the seeded obstacle field of the periodic box. */
vl_shape* vl_shape_disks(const double* cxcyr, size_t ndisks);
void vl_shape_free(vl_shape* s);
int vl_shape_inside(const vl_shape* s, double x, double y);                /* Shape::inside :12-14 */
double vl_cut_fraction(const vl_shape* s, double x, double y, double dx, double dy); /* :268-279 */
/* out = {x_min, x_max, y_min, y_max}; returns 1 if found, 0 if nothing inside (:99-115). */
int vl_bounding_box(const vl_shape* s, double reach, double step, double* out);

/* ================================================================ builder: src/sim.rs:70-137 */
vl_builder* vl_builder_new(size_t nx, size_t ny);                          /* Builder::new :84-97 */
void vl_builder_free(vl_builder* b);
int vl_builder_set_periodic(vl_builder* b, int periodic_x, int periodic_y); /* pub fields :73-74 */
int vl_builder_set_tau(vl_builder* b, double tau);                         /* :75 */
int vl_builder_set_collision(vl_builder* b, int collision, double magic);  /* :76 */
int vl_builder_set_accel(vl_builder* b, double gx, double gy);             /* :78 */
/* Builder::add(Kind::Wall) :100-104. Returns the kind id (1..254) or a negative status. */
int vl_builder_add_wall(vl_builder* b, const vl_wall* wall);
int vl_builder_add_static_wall(vl_builder* b);                             /* :107-109 */
int vl_builder_add_pressure(vl_builder* b, double rho);                    /* Kind::Pressure :56 */
int vl_builder_add_radiating(vl_builder* b, double rho);                   /* Kind::Radiating :62 */
int vl_builder_fill_rect(vl_builder* b, size_t x0, size_t x1, size_t y0, size_t y1, int kind); /* :112-118 */
int vl_builder_fill_shape(vl_builder* b, int kind);                        /* :121-132 */
/* Host-side view of the link tables Sim::from_builder would build (src/sim.rs:243-328), without
 * touching a GPU. Call with NULL arrays to get the counts, then with arrays of n (flags), nbnodes
 * (bnode_idx), nbnodes + 1 (bnode_first), 5 * nlinks (link_f64 = q, cu6, uw_x, uw_y, rho) and
 * 7 * nlinks (link_i32 = dir, pressure, radiating, vgroup, fgroup, behind, normal code
 * 1 + (nx + 1) + 3 * ny) values. For testing the host compiler against the oracle. */
int vl_builder_link_table(vl_builder* b, size_t* nlinks, size_t* nbnodes, size_t* npnodes, uint8_t* flags,
                          int32_t* bnode_idx, int32_t* bnode_first, double* link_f64, int32_t* link_i32);
/* Host-side view of how the staged step (VL_SCHEDULE_STAGED) splits its work, without touching a
 * GPU: links per block of its link kernel, link blocks, the blocks run before the first bulk part
 * (0 = the step is not split) and the rows of that first bulk part. No reference counterpart (the
 * reference's link pass is serial); for testing the split rule on the tables it is applied to. */
int vl_builder_stage_split(vl_builder* b, int* links_per_block, int* link_blocks, int* split_blocks,
                           int* split_rows);
/* Builder::build + Sim::from_builder (:134-136, :219-354): classifies the cells, builds the
 * boundary-node and link lists once on the host, uploads them and allocates the population
 * buffers in the given storage precision. Consumes `b` (freed on success and on failure). */
vl_sim* vl_builder_build(vl_builder* b, int precision);

/* ================================================================ sim: src/sim.rs:180-673 */
void vl_sim_free(vl_sim* s);
int vl_sim_info(const vl_sim* s, size_t* nx, size_t* ny, size_t* fluid_nodes, size_t* link_count,
                size_t* bnode_count, int* ngroups, int* precision);        /* fluid_nodes :377, link_count :386 */
/* Sim::init :357-371 with the field given as three host arrays of n values (x fastest).
 * NULL arrays mean the uniform values (rho0, ux0, uy0). Solid cells get (1, 0, 0). Resets t. */
int vl_sim_init(vl_sim* s, const double* rho, const double* ux, const double* uy,
                double rho0, double ux0, double uy0);
/* Sim::step :391-420, `steps` times, queued on the sim's stream (returns before completion). */
int vl_sim_step(vl_sim* s, uint64_t steps);
int vl_sim_synchronize(vl_sim* s);
int vl_sim_set_vscale(vl_sim* s, int group, double value);                 /* pub vscale :196 */
int vl_sim_get_vscale(const vl_sim* s, double* out4);
int vl_sim_set_outflow_target(vl_sim* s, int enabled, double target);      /* pub outflow_target :208 */
int vl_sim_outlet_density_offset(vl_sim* s, double* out);                 /* pub outlet_density_offset :210 */
int vl_sim_t(vl_sim* s, uint64_t* t);                                      /* pub t :214 */
/* Divergence check: nonfinite = 1 once a step produced a non-finite force, with the step index
 * (t before that step). The reference's cases test `!cd.is_finite()` after every step
 * (src/cases/cylinder.rs:179-186, src/cases/tunnel.rs:78-84); here the device records it. */
int vl_sim_status(vl_sim* s, int* nonfinite, uint64_t* first_t);
/* pub force :198 — force[g] = (fx, fy) of the last step; out holds 2 * ngroups doubles. */
int vl_sim_force(vl_sim* s, double* out);
/* All populations (FP64, reference layout, 9 * n values) of the current state (`a`). */
int vl_sim_download(vl_sim* s, double* out);
/* Replaces the current populations (FP64, reference layout). */
int vl_sim_upload(vl_sim* s, const double* in);
int vl_sim_flags(vl_sim* s, uint8_t* out);                                 /* flag :187-188: 0 interior, 1 boundary, 2 solid */
int vl_sim_macros_field(vl_sim* s, double* rho, double* ux, double* uy);   /* Sim::macros :527-534 over all cells */
int vl_sim_macros(vl_sim* s, size_t x, size_t y, double* out3);            /* Sim::macros :527-534 */
int vl_sim_total_mass(vl_sim* s, double* out);                             /* :538-548, on the device in FP64 */
int vl_sim_total_momentum(vl_sim* s, double* out2);                        /* :551-563, on the device in FP64 */
int vl_sim_max_speed(vl_sim* s, double* out);                              /* :566-579 (NaN on blow-up) */
int vl_sim_vorticity(vl_sim* s, float* out);                               /* :582-620 */
int vl_sim_probe_density(vl_sim* s, double x, double y, double* out);      /* :624-644 */
int vl_sim_probe_density_at_wall(vl_sim* s, double x, double y, double nx, double ny, double* out); /* :648-651 */
int vl_sim_state_hash(vl_sim* s, uint64_t* out);                           /* :654-668 */

/* ---- per-step recording (the device writes, the host downloads in bulk)
 * While enabled, every step appends one record of VL_REC doubles to a device history:
 *   [0 .. 2*VL_MAX_FGROUPS)  force[g] = (fx, fy) for g < ngroups (zeros above)
 *   [8]  outlet density offset used in that step
 *   [9]  pressure-drop probe value after that step (see vl_sim_set_dp_probe), else 0
 * Replaces the per-step host reads of Channel::coefficients (src/cases/channel.rs:133-136) and
 * Rig::pressure_drop (src/cases/cylinder.rs:54-59). */
#define VL_REC 10
int vl_sim_record(vl_sim* s, uint64_t capacity);   /* 0 disables; (re)starts at the next step */
int vl_sim_history(vl_sim* s, double* out, uint64_t* count);  /* out: count * VL_REC doubles */
/* Pressure drop CS2 (p_front - p_back) / u_ref^2 between the wall points (xc - r, yc) and
 * (xc + r, yc), each from Sim::probe_density_at_wall, evaluated on the device after every step. */
int vl_sim_set_dp_probe(vl_sim* s, double xc, double yc, double r, double u_ref);
/* Device time of the last vl_sim_step batch in milliseconds (CUDA events on the sim's stream). */
int vl_sim_last_step_ms(vl_sim* s, float* ms);
/* Runs `steps` steps launched one at a time with CUDA events around every kernel on the sim's
 * stream; returns the summed device milliseconds of the link kernels, of the bulk kernels and of
 * the whole batch (any pointer may be NULL). Used to measure each kernel's share of a step. */
int vl_sim_step_profiled(vl_sim* s, uint64_t steps, double* link_ms, double* bulk_ms, double* total_ms);
/* How each step is launched. VL_SCHEDULE_CONCURRENT: the link kernel (boundary nodes) on a second
 * stream, forked from and joined to the sim's stream, beside the bulk kernel (interior nodes);
 * VL_SCHEDULE_LINKS_FIRST / VL_SCHEDULE_BULK_FIRST: the same two kernels in order on one stream;
 * VL_SCHEDULE_STAGED: a kernel that applies the link rules only (the population each link returns
 * into the fluid), then a bulk kernel that updates every fluid cell, boundary cells included, in
 * coalesced row tiles. All four give bit-identical results; only the speed differs. The batch
 * engine (vl_batch_set_schedule) takes the first three. */
enum { VL_SCHEDULE_CONCURRENT = 0, VL_SCHEDULE_LINKS_FIRST = 1, VL_SCHEDULE_BULK_FIRST = 2, VL_SCHEDULE_STAGED = 3,
       VL_SCHEDULE_COUNT = 4 };
int vl_sim_set_schedule(vl_sim* s, int schedule);
int vl_sim_get_schedule(const vl_sim* s);
/* FP32 and 16-bit storage: the most neighbouring cells of a row one thread of the bulk kernel
 * updates (1, 2 or 4; default 2 for FP32, 4 for the 16-bit formats). With 2 or 4 every population plane moves as one vector per
 * thread and the collision runs on packed FP32 pairs; the kernel uses the largest of 4, 2, 1 that
 * is allowed and divides the row length (one cell per thread with a body force). Results are
 * bit-identical whatever the setting. No reference counterpart (the reference updates one cell
 * per loop iteration, src/sim.rs:700-735). */
int vl_sim_set_cells_per_thread(vl_sim* s, int cells);
/* FP32 and 16-bit storage: 1 (the default) = the bulk kernel streams the populations it reads into
 * shared memory with asynchronous bulk copies (a ring of stages filled by one producer thread per
 * block), where every row and plane is a whole number of 16-byte units and the multi-cell form
 * applies; 0 = it loads them directly. Results are bit-identical either way. No reference
 * counterpart. */
int vl_sim_set_bulk_copies(vl_sim* s, int on);
/* Each block of the bulk kernel asks the L2 to fetch (bulk prefetch) the rows its tile will read
 * `rows` output rows later (0: none), so that the blocks then running find them in the L2.
 * Default: none for FP64; for the narrow formats about two waves of blocks ahead (2 x SMs blocks).
 * Results are unchanged. No reference counterpart. */
int vl_sim_set_prefetch_rows(vl_sim* s, int rows);
/* Times each schedule for `steps_each` steps on the current state without advancing it (t, the
 * force, the history and the populations of the current state are unchanged) and keeps the
 * fastest. ms (may be NULL) receives the milliseconds per step of the VL_SCHEDULE_COUNT
 * schedules, in VL_SCHEDULE_* order. */
int vl_sim_autotune(vl_sim* s, int steps_each, double* ms);
/* Number of kernel launches issued by this sim so far (steps launch one or two kernels each). */
int vl_sim_launch_count(vl_sim* s, uint64_t* out);

/* ---- allocation-free reduction
 * No counterpart in the reference. Total mass, total momentum and largest speed (the quantities
 * of vl_sim_total_mass / vl_sim_total_momentum / vl_sim_max_speed) of a population array that the
 * caller owns, for callers that cannot allocate device memory: a host framework that hands out
 * every device byte from its own pool, a plugin that may only touch the buffers it is given, code
 * running where cudaMalloc is not allowed. The call allocates nothing: its per-block partial sums
 * live in a fixed array inside this library (112 KB held on every GPU that loads it, until the
 * process exits).
 *   populations  device pointer, FP64, population i of cell idx at i * plane_stride + idx
 *   flag         device pointer, one byte per cell (2 = not fluid, skipped), as vl_sim_flags
 *   n            cells, at most VL_REDUCE_STATIC_MAX_CELLS (larger n: VL_EINVAL)
 *   gx, gy       body acceleration (the speed is that of Sim::macros)
 *   out4         device pointer to 4 doubles: mass, momentum x, momentum y, largest speed
 *   stream       cudaStream_t to run on (NULL: the default stream); returns before completion
 * The first call on a device looks up the array's device address (once per device, with that
 * device current) and keeps it for the life of the process; make that first call before any
 * stream capture. A cudaDeviceReset (or any other teardown of the device's primary context)
 * invalidates that address: do not call this function on that device again in the same process. Every call reuses the same
 * array and overwrites each slot it reads, so nothing needs clearing, but calls whose kernels
 * overlap on the GPU (other streams, other host threads) race on it. */
#define VL_REDUCE_STATIC_MAX_CELLS 33554432
int vl_reduce_f64_static(const double* populations, size_t plane_stride, const uint8_t* flag, size_t n,
                         double gx, double gy, double* out4, void* stream);

/* ================================================================ channel: src/cases/channel.rs */
/* Spec :47-58 plus Kick :37-45. `body` is owned by the channel after the call. */
typedef struct {
  size_t nx, ny;
  int inflow;       /* VL_INFLOW_* */
  double u;         /* u_mean (parabolic) or u (uniform) */
  double nu;
  int collision;
  double magic;
  vl_shape* body;
  uint64_t ramp_steps;
  int has_kick;
  double kick_cx, kick_cy, kick_omega;
  uint64_t kick_start, kick_duration;
} vl_channel_spec;

vl_channel* vl_channel_new(const vl_channel_spec* spec, int precision);  /* Channel::new :71-116 */
void vl_channel_free(vl_channel* c);
vl_sim* vl_channel_sim(vl_channel* c);                                     /* pub sim :61 */
int vl_channel_set_absorbing(vl_channel* c, int on);                       /* pub absorbing_outlet :67 */
/* Channel::step :118-130, `steps` times. The per-step controls (inlet ramp, outlet target, body
 * kick) come from a schedule uploaded once, so a batch of steps needs no host round trip. */
int vl_channel_step(vl_channel* c, uint64_t steps);
int vl_channel_coefficients(vl_channel* c, double d, double* cd, double* cl); /* :133-136 */
double vl_channel_u_ref(const vl_channel* c);

/* ================================================================ batched tunnels
 * No single reference counterpart: the reference runs one Channel at a time
 * (src/cases/tunnel.rs:52-92). A batch advances many channels of uneven sizes, shapes and Reynolds
 * numbers together on one device, each for its own number of steps; every tunnel follows
 * Channel::step exactly (in FP64 a tunnel in a batch is bit-identical to the same tunnel run alone;
 * in FP32 / FP16 it agrees to rounding: multiply-add contraction may differ between the kernels). */
typedef struct vl_batch vl_batch;
vl_batch* vl_batch_new(int precision);
void vl_batch_free(vl_batch* b);
/* Adds a channel (takes spec->body) to be run for `steps` steps; returns its index. */
int vl_batch_add_channel(vl_batch* b, const vl_channel_spec* spec, uint64_t steps);
/* Packs every tunnel into one device arena and starts them (t = 0). */
int vl_batch_build(vl_batch* b);
int vl_batch_size(const vl_batch* b);
int vl_batch_tunnel_info(const vl_batch* b, int k, size_t* nx, size_t* ny, size_t* fluid_nodes, uint64_t* steps);
/* Bulk tile shape: 2^log2_tx cells x ty rows = 256 cells (32 <= 2^log2_tx <= 256), times the
 * bulk cells per thread; or (5, 0): the packed layout, 8 consecutive warp segments (32 cells times
 * the cells per thread, of one row each) of a tunnel's rows laid end to end, so that only the last
 * segment of each row runs past the row end. */
int vl_batch_set_tile(vl_batch* b, int log2_tx, int ty);
/* FP32 and 16-bit storage: 2 (the default where every tunnel's row length is even) bulk cells of a
 * row per thread, as vl_sim_set_cells_per_thread, or 1. Results are bit-identical either way. */
int vl_batch_set_cells_per_thread(vl_batch* b, int cells);
/* Each bulk block asks the L2 to fetch the rows of the tile `tiles` places later in the tile list
 * (0: none; default 3 x SMs for the narrow formats, none for FP64), as vl_sim_set_prefetch_rows. */
int vl_batch_set_prefetch_tiles(vl_batch* b, int tiles);
int vl_batch_get_tile(const vl_batch* b, int* log2_tx, int* ty);
int vl_batch_set_schedule(vl_batch* b, int schedule);  /* VL_SCHEDULE_* */
/* Times the tile shapes 256x1, 128x2, 64x4, 32x8 and the packed layout on the current state
 * without advancing it and keeps the fastest; ms4 (may be NULL) receives milliseconds per step for
 * the four row shapes. */
int vl_batch_autotune(vl_batch* b, int steps_each, double* ms4);
/* The same; ms (may be NULL) receives up to n of the five times (row shapes, then packed). */
int vl_batch_autotune_layouts(vl_batch* b, int steps_each, double* ms, int n);
/* Runs every unfinished tunnel until it has done its steps (max_steps = 0), or at most max_steps
 * global steps. Synchronous. */
int vl_batch_run(vl_batch* b, uint64_t max_steps);
/* The same steps enqueued on the batch's stream without waiting for them; vl_batch_wait (or any
 * call that reads the batch's state) waits. While they run, the host may read the force records
 * of steps complete at the previous wait (vl_batch_history_copy) and end tunnels
 * (vl_batch_set_steps with a step at or after the enqueued run's end). */
int vl_batch_run_async(vl_batch* b, uint64_t max_steps);
int vl_batch_wait(vl_batch* b);
/* Force records (fx, fy per step) of n ranges, concatenated into out (2 * sum(counts) doubles):
 * steps [firsts[i], firsts[i] + counts[i]) of tunnel ks[i]. Every range must lie within the
 * tunnel's history and before the tunnel's steps complete at the last wait (records a tunnel has
 * not written, after it ended, are not defined). Read on a stream of its own, so it does not wait
 * for a run in flight. No reference counterpart (the on-line stopping rule's input). */
int vl_batch_history_copy(vl_batch* b, int n, const int* ks, const uint64_t* firsts, const uint64_t* counts,
                          double* out);
int vl_batch_last_run_ms(vl_batch* b, float* ms);
int vl_batch_global_step(const vl_batch* b, uint64_t* s);
int vl_batch_launch_count(const vl_batch* b, uint64_t* out);
/* Steps done, divergence flag and the last force (fx, fy) of tunnel k. */
int vl_batch_status(vl_batch* b, int k, uint64_t* t, int* nonfinite, double* force2);
/* Force (fx, fy) of tunnel k after each of its steps so far: 2 * count doubles. */
int vl_batch_force_history(vl_batch* b, int k, double* out, uint64_t* count);
/* The records of steps [first, first + max) of tunnel k that exist so far (count receives how
 * many; 2 doubles each): the increments an on-line stopping rule reads between runs. */
int vl_batch_force_history_range(vl_batch* b, int k, uint64_t first, uint64_t max, double* out, uint64_t* count);
/* FP64 populations of tunnel k (reference layout, 9 * nx * ny values), its flags, its state hash. */
int vl_batch_download(vl_batch* b, int k, double* out);
/* Ends tunnel k after `steps` steps instead of the count it was added with (which stays the upper
 * bound and sizes its force history); allowed while the tunnel has not run past `steps`, counting
 * the steps of a run in flight, which the change follows on the stream. Lets a caller stop each
 * tunnel at a moment it picks from the tunnel's own force history. */
int vl_batch_set_steps(vl_batch* b, int k, uint64_t steps);
/* Holds tunnel k at its start state (before the batch's first step): it takes no steps until
 * vl_batch_start. vl_batch_start starts a held tunnel: its step 0 is the batch's next global step
 * after the steps already enqueued (start receives that global step; may be NULL). A tunnel's
 * steps, history and vl_batch_set_steps count from its own step 0. A caller keeps a uniform-start
 * twin of a warm-started tunnel held in the same batch and starts it only if the warm start fails
 * (the fallback of the learned warm start). No reference counterpart. */
int vl_batch_hold(vl_batch* b, int k);
int vl_batch_start(vl_batch* b, int k, uint64_t* start);
/* Density and velocity of every cell of tunnel k at its current step (solids (1, 0, 0)), FP64,
 * row-major n = nx * ny values each: Sim::macros (src/sim.rs:527-536) over the whole grid. */
int vl_batch_macros_field(vl_batch* b, int k, double* rho, double* ux, double* uy);
/* Sim::init (src/sim.rs:357-371) for tunnel k of a built batch before its first step: the
 * equilibria of the FP64 fields rho, ux, uy (n = nx * ny values each, row-major) into both
 * population buffers, solids at rest. The warm-start hook of the batched engine. */
int vl_batch_init(vl_batch* b, int k, const double* rho, const double* ux, const double* uy);
/* The same from a coarse cell-centred grid of normalised fields in device memory (FP32
 * [gh][gw][gc], gc >= 3): lattice cell (x, y) samples it bilinearly at column (x - x0) / dx - 1/2
 * and row (y - y0) / dy - 1/2, clamped at the grid's edges, and decodes channels 0-2 to
 * u_x = u (1 + v0), u_y = u v1, rho = 1 + 1.5 u^2 v2 (the warm-start network's output), all on the
 * device. */
int vl_batch_init_grid(vl_batch* b, int k, const float* grid, int gh, int gw, int gc, double x0, double dx, double y0,
                       double dy, double u);
int vl_batch_flags(vl_batch* b, int k, uint8_t* out);
int vl_batch_state_hash(vl_batch* b, int k, uint64_t* out);

/* ================================================================ learned warm start: kernels
 * No reference counterpart. Device-pointer kernels of the warm-start network (a convolutional
 * network trained on solver-generated wakes); the caller owns every buffer.
 * vl_nn_gemm_bf16: out[m, n] = epilogue(sum_k a[m, k] * b[n, k]) on the tcgen05 tensor cores,
 * BF16 inputs (leading dimensions lda / ldb multiples of 8), FP32 accumulation. By default a is
 * stored [M][K] and b [N][K] (K contiguous); with VL_GEMM_A_MN a is stored [K][M] and with
 * VL_GEMM_B_MN b is stored [K][N] (M or N contiguous; then bn >= 64). flags also select the
 * epilogue: 1 accumulate into FP32 out, 2 add bias[n], 4 ReLU, 8 store BF16. bn: tile width 32,
 * 64, 128 or 256. err (device int, may be NULL) becomes nonzero if a tile timed out waiting for
 * its data (every wait of the kernel is bounded; the tile is then skipped and its tensor memory
 * freed). VL_GEMM_TEST_TIMEOUT exercises that path: the first operand load of every tile is never
 * issued and the waits give up after a short limit; out is not written, err is set. Asynchronous
 * on `stream`. */
enum { VL_GEMM_ACCUM = 1, VL_GEMM_BIAS = 2, VL_GEMM_RELU = 4, VL_GEMM_BF16 = 8, VL_GEMM_A_MN = 16, VL_GEMM_B_MN = 32,
       VL_GEMM_TEST_TIMEOUT = 64 };
int vl_nn_gemm_bf16(const void* a, int lda, const void* b, int ldb, int M, int N, int K, void* out, int ldc,
                    const float* bias, int flags, int bn, int* err, void* stream);
/* Gathers and elementwise kernels around the GEMM. Activations are NHWC BF16 (row = pixel,
 * channels contiguous); a 3x3 convolution (padding 1, stride 1 or 2) is im2col + GEMM, with the
 * im2col row in (ky, kx, c) order zero-padded to kp (a multiple of 64) columns. */
int vl_nn_im2col(const void* x, int B, int H, int W, int C, int stride, int kp, void* cols, void* stream);
int vl_nn_col2im(const float* dcols, int B, int H, int W, int C, int stride, int kp, float* dx, int accumulate,
                 void* stream);
/* dz = dy * (y > 0) (relu) or dy, as BF16 [R, C] and (dzt, may be NULL) transposed [C, R]; colsum (may be NULL)
 * receives per 32-row tile column sums [C][ceil(R / 32)] that vl_nn_bias_grad reduces to db. */
int vl_nn_act_bwd(const float* dy, const void* y, int R, int C, int relu, void* dz, void* dzt, float* colsum,
                  void* stream);
int vl_nn_bias_grad(const float* colsum, int R, int C, float* db, void* stream);
/* BF16 transpose [R, C] -> [C, R], R and C even. */
int vl_nn_transpose_bf16(const void* a, int R, int C, void* at, void* stream);
/* Weights wf [cin, kpf] of the input-gradient convolution of a stride-1 3x3 layer with weights
 * w [cout, kp]: wf[c, (ky, kx, co)] = w[co, (2 - ky, 2 - kx, c)], so dX = conv3x3(dZ, wf). */
int vl_nn_flip_weights(const void* w, int cout, int cin, int kp, int kpf, void* wf, void* stream);
/* Nearest 2x upsampling into channels [coff, coff + C) of a ctot-channel output, and its adjoint. */
int vl_nn_up2(const void* x, int B, int H, int W, int C, void* y, int ctot, int coff, void* stream);
int vl_nn_up2_bwd(const float* dy, int B, int H, int W, int C, int ctot, int coff, float* dx, int accumulate,
                  void* stream);
int vl_nn_copy_channels(const void* x, long long R, int C, void* y, int ctot, int coff, void* stream);
int vl_nn_slice_channels(const float* y, long long R, int ctot, int coff, int C, float* x, int accumulate, void* stream);
/* Weighted mean-squared error of out [R, C] against tgt [R, cuse] on the first cuse channels (w
 * per row): per-block FP64 partial sums of sum(w (out - tgt)^2) * inv_count and the gradient
 * 2 w (out - tgt) * inv_count (zero on channels cuse..C-1). */
int vl_nn_mse(const float* out, const float* tgt, const float* w, long long R, int C, int cuse, double inv_count,
              float* dout, double* partial, int blocks, void* stream);
/* Adam step `step` (1-based) on FP32 weights; wb (may be NULL) receives a BF16 copy. */
int vl_nn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
               int step, void* wb, void* stream);
int vl_nn_f32_to_bf16(const float* a, long long n, void* b, void* stream);

/* ================================================================ signal: src/signal.rs */
int vl_fft(double* re, double* im, size_t n);                              /* :6-44 */
double vl_mean(const double* x, size_t n);                                 /* :61-63 */
double vl_rms(const double* x, size_t n);                                  /* :66-69 */
int vl_dominant_frequency(const double* x, size_t n, double dt, double* freq, double* amp); /* :92-107 */
size_t vl_peaks(const double* x, size_t n, double* pos, double* val, size_t cap);           /* :111-123 */
int vl_crossing_frequency(const double* x, size_t n, double dt, double* out);                /* :127-140 */
double vl_sample_at(const double* x, size_t n, double pos);                /* :143-147 */
double vl_ramp(uint64_t t, uint64_t steps);                                /* src/cases/mod.rs:11-18 */
double vl_tau_for(double nu);                                              /* src/lattice.rs:53-55 */

#ifdef __cplusplus
}
#endif
#endif /* VORTEXLAB_H */
