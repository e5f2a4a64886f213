// C ABI of vortexlab-b200 (include/vortexlab.h): shapes, builder, device-resident sims, the
// channel case and signal analysis. Host code; the kernels live in vl_step_*.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/vortexlab.h"
#include "vl_device.cuh"
#include "vl_host.hpp"
#include "vl_internal.hpp"
#include "vl_launch.hpp"

struct vl_builder {
  vl::DomainSpec spec;
};

namespace {

thread_local std::string g_err;
thread_local int g_code = VL_OK;

int fail(int code, const std::string& msg) {
  g_err = msg;
  g_code = code;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? VL_ENOMEM : VL_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VL_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

vl_shape* wrap_shape(std::unique_ptr<vl::Shape> s) {
  auto w = new vl_shape();
  w->s = std::move(s);
  return w;
}

constexpr int kGraphSteps = 32;  // steps per captured CUDA graph (even: buffer parity returns)
constexpr int kReduceBlocks = 296;

}  // namespace

int vl::set_error(int code, const char* msg) { return fail(code, msg); }

// ==================================================================== device-resident sim
struct vl_sim {
  int device = 0;
  int prec = VL_F64;
  const vl::Launchers* L = nullptr;
  vl::CompiledDomain dom;
  size_t n = 0;
  unsigned ns = 0;
  void* buf[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t* d_flag = nullptr;
  int32_t* d_bidx = nullptr;
  int32_t* d_bfirst = nullptr;
  vl::LinkRecDev* d_links = nullptr;
  int32_t* d_pidx = nullptr;
  int8_t* d_pn = nullptr;
  vl::Ctl* d_ctl = nullptr;
  double* d_partials = nullptr;
  double* d_hist = nullptr;
  double* d_sched = nullptr;
  double* d_red = nullptr;
  int32_t* d_cells = nullptr;
  double* d_gather = nullptr;
  int2* d_bdesc = nullptr;         // staged step: per boundary node {first link, link-direction mask}
  int32_t* d_wbfirst = nullptr;    // staged step: boundary nodes before each 32-cell warp slot
  int32_t* d_lnode = nullptr;      // staged step: boundary node of each link
  void* d_lb = nullptr;            // staged step: returning population per link
  void* d_ownc = nullptr;          // staged step: boundary nodes' own populations (CSR order)
  bool own_ok = false;             // d_ownc holds the boundary nodes of the current state
  int split_links = 0, split_rows = 0;  // staged step in two parts (0: one part)
  cudaStream_t stream = nullptr;   // the sim's stream: bulk kernel, copies, everything else
  cudaStream_t aux = nullptr;      // the link kernel of each step, forked from and joined to `stream`
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  vl::StepParams P{};
  int ck = 1;
  cudaGraphExec_t gexec = nullptr;
  uint64_t launches = 0;
  int kernels_per_step = 1;  // kernel launches of one step (twice that for the staged step in two parts)
  uint64_t step_launches() const { return (uint64_t)kernels_per_step * (schedule == 3 && split_links > 0 ? 2 : 1); }
  // How a step is launched: 0 concurrent (fork/join over two streams), 1 link kernel then bulk
  // kernel on one stream, 2 bulk then link, 3 staged (link values, then the bulk kernel that also
  // updates boundary cells; one stream).
  int schedule = 0;
  uint64_t t_host = 0;
  uint64_t rec_start = 0, rec_cap = 0;
  bool timed = false;
  // host mirror of the control block
  vl::Ctl hctl{};

  ~vl_sim() {
    if (device >= 0) cudaSetDevice(device);
    if (gexec) cudaGraphExecDestroy(gexec);
    void* ptrs[] = {buf[0], buf[1], d_flag, d_bidx, d_bfirst, d_links, d_pidx, d_pn, d_ctl,
                    d_partials, d_hist, d_sched, d_red, d_cells, d_gather, d_bdesc, d_wbfirst, d_lb, d_ownc, d_lnode};
    for (void* p : ptrs)
      if (p) cudaFree(p);
    for (cudaEvent_t e : pev) cudaEventDestroy(e);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
  }

  const void* a() const { return buf[cur]; }
  void* b() const { return buf[cur ^ 1]; }

  int push_ctl() {
    VL_CUDA(cudaMemcpyAsync(d_ctl, &hctl, sizeof(vl::Ctl), cudaMemcpyHostToDevice, stream));
    return VL_OK;
  }
  // Reads the device control block into the host mirror (synchronises the stream).
  int pull_ctl() {
    VL_CUDA(cudaMemcpyAsync(&hctl, d_ctl, sizeof(vl::Ctl), cudaMemcpyDeviceToHost, stream));
    VL_CUDA(cudaStreamSynchronize(stream));
    return VL_OK;
  }

  // One step: the link kernel on `aux` and the bulk kernel on `stream`, concurrently. They read
  // only `a` and write disjoint cells of `b`; the join makes the next step wait for both. Optional
  // timing events bracket each kernel on its own stream.
  cudaError_t enqueue_step(cudaEvent_t lk0 = nullptr, cudaEvent_t lk1 = nullptr, cudaEvent_t bk0 = nullptr,
                           cudaEvent_t bk1 = nullptr) {
    cudaError_t e;
    cudaStream_t ls = schedule == 0 ? aux : stream;
    const int staged = schedule == 3 ? 0x400 : 0;
    auto links = [&]() -> cudaError_t {
      cudaError_t r;
      if (lk0 && (r = cudaEventRecord(lk0, ls)) != cudaSuccess) return r;
      if ((r = L->step(P, ck | 0x100 | staged, a(), b(), ls)) != cudaSuccess) return r;
      if (lk1 && (r = cudaEventRecord(lk1, ls)) != cudaSuccess) return r;
      return cudaSuccess;
    };
    auto bulk = [&]() -> cudaError_t {
      cudaError_t r;
      if (bk0 && (r = cudaEventRecord(bk0, stream)) != cudaSuccess) return r;
      if ((r = L->step(P, ck | 0x200 | staged, a(), b(), stream)) != cudaSuccess) return r;
      if (bk1 && (r = cudaEventRecord(bk1, stream)) != cudaSuccess) return r;
      return cudaSuccess;
    };
    if (schedule == 3 && split_links > 0) return enqueue_staged_split(lk0, lk1, bk0, bk1);
    if (schedule == 1 || schedule == 3) {
      if ((e = links()) != cudaSuccess) return e;
      return bulk();
    }
    if (schedule == 2) {
      if ((e = bulk()) != cudaSuccess) return e;
      return links();
    }
    if ((e = cudaEventRecord(ev_fork, stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(aux, ev_fork, 0)) != cudaSuccess) return e;
    if ((e = links()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev_join, aux)) != cudaSuccess) return e;
    if ((e = bulk()) != cudaSuccess) return e;
    return cudaStreamWaitEvent(stream, ev_join, 0);
  }

  // The staged step in two parts. The first `split_links` link blocks run first; then the bulk
  // tiles of the rows whose boundary nodes they hold (`split_rows` rows), while the remaining link
  // blocks run beside them on `aux`; then the remaining tiles, after both. Only the first part of
  // the link kernel is exposed. The events bracket the exposed link part and the two bulk parts.
  cudaError_t enqueue_staged_split(cudaEvent_t lk0, cudaEvent_t lk1, cudaEvent_t bk0, cudaEvent_t bk1) {
    cudaError_t e;
    vl::StepParams pa = P, pb = P;
    pa.link_b0 = 0;
    pa.link_n = split_links;
    pa.bulk_b0 = 0;
    pa.bulk_n = split_rows;
    pb.link_b0 = split_links;
    pb.link_n = P.nlinkblk - split_links;
    pb.bulk_b0 = split_rows;
    pb.bulk_n = P.ny - split_rows;
    const int lk = ck | 0x100 | 0x400, bk = ck | 0x200 | 0x400;
    if ((e = cudaEventRecord(ev_fork, stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(aux, ev_fork, 0)) != cudaSuccess) return e;
    if (lk0 && (e = cudaEventRecord(lk0, stream)) != cudaSuccess) return e;
    if ((e = L->step(pa, lk, a(), b(), stream)) != cudaSuccess) return e;
    if (lk1 && (e = cudaEventRecord(lk1, stream)) != cudaSuccess) return e;
    if ((e = L->step(pb, lk, a(), b(), aux)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev_join, aux)) != cudaSuccess) return e;
    if (bk0 && (e = cudaEventRecord(bk0, stream)) != cudaSuccess) return e;
    if ((e = L->step(pa, bk, a(), b(), stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(stream, ev_join, 0)) != cudaSuccess) return e;
    if ((e = L->step(pb, bk, a(), b(), stream)) != cudaSuccess) return e;
    if (bk1 && (e = cudaEventRecord(bk1, stream)) != cudaSuccess) return e;
    return cudaSuccess;
  }

  int set_cells_per_thread(int c) {
    if (c != 1 && c != 2 && c != 4) return fail(VL_EINVAL, "cells per thread must be 1, 2 or 4");
    if (c != P.pairs && gexec) {
      VL_CUDA(cudaStreamSynchronize(stream));
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    P.pairs = c;
    return VL_OK;
  }

  int set_prefetch_rows(int rows) {
    if (rows < 0 || rows > 4096) return fail(VL_EINVAL, "prefetch rows must be in 0..4096");
    if (rows != P.prefetch_rows && gexec) {
      VL_CUDA(cudaStreamSynchronize(stream));
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    P.prefetch_rows = rows;
    return VL_OK;
  }

  int set_bulk_copies(int on) {
    if ((on != 0) != (P.stream != 0) && gexec) {
      VL_CUDA(cudaStreamSynchronize(stream));
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    P.stream = on ? 1 : 0;
    return VL_OK;
  }

  int set_schedule(int sc) {
    if (sc < 0 || sc >= VL_SCHEDULE_COUNT) return fail(VL_EINVAL, "schedule must be 0, 1, 2 or 3");
    if (sc != schedule && gexec) {
      VL_CUDA(cudaStreamSynchronize(stream));
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    schedule = sc;
    return VL_OK;
  }

  // Times every schedule on the current state without advancing it: the control block is put in
  // dry mode (the epilogue commits nothing) and each timed step recomputes `b` from the same `a`.
  int autotune(int steps_each, double* ms_out) {
    VL_CUDA(cudaSetDevice(device));
    int rc = pull_ctl();
    if (rc) return rc;
    hctl.dry = 1;
    if ((rc = push_ctl())) return rc;
    double best = 1e300;
    int best_sc = schedule;
    for (int sc = 0; sc < VL_SCHEDULE_COUNT; ++sc) {
      schedule = sc;
      own_ok = false;
      if ((rc = prepare_steps())) return rc;
      for (int k = 0; k < 2; ++k) {
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) return cuda_fail(e, "autotune");
      }
      VL_CUDA(cudaEventRecord(ev0, stream));
      for (int k = 0; k < steps_each; ++k) {
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) return cuda_fail(e, "autotune");
      }
      VL_CUDA(cudaEventRecord(ev1, stream));
      VL_CUDA(cudaEventSynchronize(ev1));
      float ms = 0.f;
      VL_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
      if (ms_out) ms_out[sc] = ms / steps_each;
      if (ms < best) { best = ms; best_sc = sc; }
    }
    // the dry staged steps left the copy of `b`, not of `a`
    own_ok = false;
    if ((rc = pull_ctl())) return rc;
    hctl.dry = 0;
    if ((rc = push_ctl())) return rc;
    schedule = -1;
    return set_schedule(best_sc);
  }

  // The pressure probe of step t is evaluated during step t + 1; the last step of a batch gets
  // it from this one-block kernel.
  int flush_probe() {
    if (!hctl.dp_on) return VL_OK;
    cudaError_t e = L->probe(P, a(), stream);
    if (e != cudaSuccess) return cuda_fail(e, "probe launch");
    launches += 1;
    return VL_OK;
  }

  // The staged step reads the boundary nodes' own populations from d_ownc, which each staged bulk
  // kernel refreshes for the next step; after anything else set the state it is gathered from `a`.
  int prepare_steps() {
    if (schedule != 3 || own_ok) return VL_OK;
    cudaError_t e = L->gather_own(P, a(), stream);
    if (e != cudaSuccess) return cuda_fail(e, "gather own populations");
    launches += 1;
    own_ok = true;
    return VL_OK;
  }

  int launch_one() {
    cudaError_t e = enqueue_step();
    if (e != cudaSuccess) return cuda_fail(e, "step launch");
    cur ^= 1;
    launches += step_launches();
    return VL_OK;
  }

  int ensure_graph() {
    if (gexec) return VL_OK;
    cudaGraph_t g = nullptr;
    VL_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int saved = cur;
    cur = 0;
    for (int k = 0; k < kGraphSteps; ++k) {
      cudaError_t e = enqueue_step();
      cur ^= 1;
      if (e != cudaSuccess) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        cur = saved;
        return cuda_fail(e, "graph capture");
      }
    }
    cur = saved;
    VL_CUDA(cudaStreamEndCapture(stream, &g));
    cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
    return VL_OK;
  }

  int step(uint64_t steps) {
    VL_CUDA(cudaSetDevice(device));
    if (int rc = prepare_steps()) return rc;
    VL_CUDA(cudaEventRecord(ev0, stream));
    uint64_t left = steps;
    while (left > 0) {
      if (left >= (uint64_t)kGraphSteps && cur == 0) {
        int rc = ensure_graph();
        if (rc) return rc;
        VL_CUDA(cudaGraphLaunch(gexec, stream));
        launches += (uint64_t)kGraphSteps * step_launches();
        left -= kGraphSteps;
      } else {
        int rc = launch_one();
        if (rc) return rc;
        left -= 1;
      }
    }
    VL_CUDA(cudaEventRecord(ev1, stream));
    timed = true;
    t_host += steps;
    if (steps) own_ok = schedule == 3;
    return flush_probe();
  }

  // Steps launched one by one with CUDA events around each kernel on the sim's stream; returns
  // the summed device time of the link kernels, of the bulk kernels and of the whole batch.
  std::vector<cudaEvent_t> pev;
  int step_profiled(uint64_t steps, double* link_ms, double* bulk_ms, double* total_ms) {
    VL_CUDA(cudaSetDevice(device));
    const size_t need = 4 * (size_t)steps + 2;
    while (pev.size() < need) {
      cudaEvent_t e;
      VL_CUDA(cudaEventCreate(&e));
      pev.push_back(e);
    }
    if (int rc = prepare_steps()) return rc;
    VL_CUDA(cudaEventRecord(pev[0], stream));
    for (uint64_t k = 0; k < steps; ++k) {
      cudaEvent_t* e4 = &pev[2 + 4 * k];
      cudaError_t e = enqueue_step(e4[0], e4[1], e4[2], e4[3]);
      if (e != cudaSuccess) return cuda_fail(e, "profiled step");
      cur ^= 1;
      launches += step_launches();
    }
    own_ok = schedule == 3;
    VL_CUDA(cudaEventRecord(pev[1], stream));
    VL_CUDA(cudaEventSynchronize(pev[1]));
    double lk = 0.0, bk = 0.0;
    for (uint64_t k = 0; k < steps; ++k) {
      const cudaEvent_t* e4 = &pev[2 + 4 * k];
      float m = 0.f;
      VL_CUDA(cudaEventElapsedTime(&m, e4[0], e4[1]));
      lk += m;
      VL_CUDA(cudaEventElapsedTime(&m, e4[2], e4[3]));
      bk += m;
    }
    float tot = 0.f;
    VL_CUDA(cudaEventElapsedTime(&tot, pev[0], pev[1]));
    if (link_ms) *link_ms = lk;
    if (bulk_ms) *bulk_ms = bk;
    if (total_ms) *total_ms = tot;
    t_host += steps;
    return flush_probe();
  }

  // 9 FP64 populations of each listed cell (reference order).
  int gather(const std::vector<int32_t>& cells, std::vector<double>& out) {
    out.assign(cells.size() * 9, 0.0);
    if (cells.empty()) return VL_OK;
    if (cells.size() > 64) return fail(VL_EINVAL, "gather: too many cells");
    VL_CUDA(cudaMemcpyAsync(d_cells, cells.data(), cells.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
    cudaError_t e = L->gather((int)cells.size(), ns, d_cells, a(), d_gather, stream);
    if (e != cudaSuccess) return cuda_fail(e, "gather");
    VL_CUDA(cudaMemcpyAsync(out.data(), d_gather, out.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VL_CUDA(cudaStreamSynchronize(stream));
    return VL_OK;
  }
};

namespace {

// Bilinear probe weights of Sim::probe_density (src/sim.rs:624-644) for the point (x, y): up to
// four (cell, weight) pairs, in the reference's corner order, for fluid cells with weight > 0.
void probe_corners(const vl_sim& s, double x, double y, int32_t* idx, double* w) {
  const double i = std::floor(x), j = std::floor(y);
  const double fx = x - i, fy = y - j;
  const long di[4] = {0, 1, 0, 1}, dj[4] = {0, 0, 1, 1};
  const double wk[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
  for (int k = 0; k < 4; ++k) {
    idx[k] = -1;
    w[k] = 0.0;
    const long xi = (long)i + di[k], yj = (long)j + dj[k];
    if (xi < 0 || yj < 0 || xi >= (long)s.dom.nx || yj >= (long)s.dom.ny) continue;
    const size_t c = (size_t)yj * s.dom.nx + (size_t)xi;
    if (s.dom.flag[c] != 2 && wk[k] > 0.0) {
      idx[k] = (int32_t)c;
      w[k] = wk[k];
    }
  }
}

void moments_host(const double* f, double& rho, double& jx, double& jy) { vl::moments(f, rho, jx, jy); }

int sim_probe_density(vl_sim* s, double x, double y, double* out) {
  int32_t idx[4];
  double w[4];
  probe_corners(*s, x, y, idx, w);
  std::vector<int32_t> cells;
  for (int k = 0; k < 4; ++k)
    if (idx[k] >= 0) cells.push_back(idx[k]);
  std::vector<double> f;
  int rc = s->gather(cells, f);
  if (rc) return rc;
  double sum = 0.0, wsum = 0.0;
  size_t m = 0;
  for (int k = 0; k < 4; ++k) {
    if (idx[k] < 0) continue;
    double rho, jx, jy;
    moments_host(&f[9 * m], rho, jx, jy);
    ++m;
    sum += w[k] * rho;
    wsum += w[k];
  }
  *out = wsum > 0.0 ? sum / wsum : std::nan("");
  return VL_OK;
}

int alloc_copy(void** dst, const void* src, size_t bytes) {
  if (bytes == 0) bytes = 16;
  VL_CUDA(cudaMalloc(dst, bytes));
  if (src) VL_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return VL_OK;
}

// Tables of the staged step. bdesc[k] = {first link of boundary node k, bit j set for each of its
// link directions j}; the node's links must be stored by ascending direction, so that the link of
// direction j is first + popc(mask below j). wbfirst[w] = boundary nodes (CSR order = cell order)
// before the first cell of warp slot w of the bulk grid (block = row tile, 32 cells per warp).
bool staged_tables(const vl::CompiledDomain& d, int tiles_per_row, std::vector<int2>& bdesc,
                   std::vector<int32_t>& wbfirst, std::string& err) {
  const size_t nb = d.bnode_idx.size();
  bdesc.assign(nb ? nb : 1, int2{0, 0});
  for (size_t k = 0; k < nb; ++k) {
    const int first = d.bnode_first[k], last = d.bnode_first[k + 1];
    int mask = 0, prev = 0;
    for (int l = first; l < last; ++l) {
      const int j = d.links[(size_t)l].dir;
      if (j <= prev || j > 8) { err = "staged step: links of a node must have ascending directions 1..8"; return false; }
      prev = j;
      mask |= 1 << j;
    }
    bdesc[k] = int2{first, mask};
  }
  const int wpt = vl::kBlock / 32;
  wbfirst.assign((size_t)tiles_per_row * d.ny * wpt, 0);
  size_t k = 0;  // boundary nodes before the current cell
  for (size_t y = 0; y < d.ny; ++y) {
    for (int t = 0; t < tiles_per_row; ++t) {
      for (int w = 0; w < wpt; ++w) {
        const size_t x0 = (size_t)t * vl::kBlock + (size_t)w * 32;
        const size_t start = y * d.nx + std::min(x0, d.nx);
        while (k < nb && (size_t)d.bnode_idx[k] < start) ++k;
        wbfirst[(y * tiles_per_row + t) * wpt + w] = (int32_t)k;
      }
    }
  }
  return true;
}

#ifndef VL_STAGE_SPLIT
#define VL_STAGE_SPLIT 4
#endif

// Creates the device-resident sim for a compiled domain.
// Split point of the staged step: a fraction 1 / VL_STAGE_SPLIT of the link blocks, and the row
// tiles before the row of the node of the first link they leave to the second part (every
// boundary node of the earlier rows has all its links in the first part). 0, 0: one part.
void staged_split(const vl::CompiledDomain& d, const std::vector<int32_t>& lnode, int& split_links, int& split_rows) {
  split_links = split_rows = 0;
  const int per = vl::kBlock * vl::kStagePer;
  const int nlinkblk = std::max(1, ((int)d.links.size() + per - 1) / per);
  if (nlinkblk >= VL_STAGE_SPLIT) {
    const int la = nlinkblk / VL_STAGE_SPLIT;
    const int row = d.bnode_idx[(size_t)lnode[(size_t)la * per]] / (int)d.nx;
    if (row > 0) {
      split_links = la;
      split_rows = row;
    }
  }
}

vl_sim* make_sim(vl::CompiledDomain&& dom, int precision) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    fail(VL_ECUDA, "no CUDA device: vortexlab-b200 has no CPU fallback");
    return nullptr;
  }
  auto s = std::make_unique<vl_sim>();
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    fail(VL_ECUDA, "cudaGetDevice failed");
    return nullptr;
  }
  s->prec = precision;
  switch (precision) {
    case VL_F64: s->L = &vl::launchers_f64(); break;
    case VL_F32: s->L = &vl::launchers_f32(); break;
    case VL_F16S: s->L = &vl::launchers_f16s(); break;
    case VL_F16C: s->L = &vl::launchers_f16c(); break;
    case VL_F16X: s->L = &vl::launchers_f16x(); break;
    default: fail(VL_EINVAL, "unknown precision"); return nullptr;
  }
  s->dom = std::move(dom);
  vl::CompiledDomain& d = s->dom;
  s->n = d.n;
  s->ns = (unsigned)((d.n + 63) / 64 * 64);
  if ((unsigned long long)s->ns * 9ull > 0xFFFFFFFFull) {
    fail(VL_EINVAL, "grid too large: 9 population planes must fit 32-bit offsets");
    return nullptr;
  }
  auto chk = [&](int rc) { return rc == VL_OK; };
  const size_t pop_bytes = (size_t)s->ns * 9 * s->L->elem;
  if (!chk(alloc_copy(&s->buf[0], nullptr, pop_bytes)) || !chk(alloc_copy(&s->buf[1], nullptr, pop_bytes)))
    return nullptr;
  if (cudaMemset(s->buf[0], 0, pop_bytes) != cudaSuccess || cudaMemset(s->buf[1], 0, pop_bytes) != cudaSuccess) {
    fail(VL_ECUDA, "memset");
    return nullptr;
  }
  std::vector<vl::LinkRecDev> links(d.links.size());
  for (size_t k = 0; k < d.links.size(); ++k) {
    const vl::LinkRec& h = d.links[k];
    vl::LinkRecDev& g = links[k];
    g.q = h.q; g.cu6 = h.cu6; g.uw0 = h.uw[0]; g.uw1 = h.uw[1]; g.rho = h.rho;
    g.behind = h.behind; g.dir = h.dir; g.flags = h.flags; g.vgroup = h.vgroup; g.fgroup = h.fgroup;
  }
  std::vector<int8_t> pn(2 * d.pnode_idx.size());
  for (size_t k = 0; k < d.pnode_idx.size(); ++k) { pn[2 * k] = d.pnode_nx[k]; pn[2 * k + 1] = d.pnode_ny[k]; }
  if (!chk(alloc_copy((void**)&s->d_flag, d.flag.data(), d.n)) ||
      !chk(alloc_copy((void**)&s->d_bidx, d.bnode_idx.data(), d.bnode_idx.size() * 4)) ||
      !chk(alloc_copy((void**)&s->d_bfirst, d.bnode_first.data(), d.bnode_first.size() * 4)) ||
      !chk(alloc_copy((void**)&s->d_links, links.data(), links.size() * sizeof(vl::LinkRecDev))) ||
      !chk(alloc_copy((void**)&s->d_pidx, d.pnode_idx.data(), d.pnode_idx.size() * 4)) ||
      !chk(alloc_copy((void**)&s->d_pn, pn.data(), pn.size())) ||
      !chk(alloc_copy((void**)&s->d_ctl, nullptr, sizeof(vl::Ctl))) ||
      !chk(alloc_copy((void**)&s->d_red, nullptr, kReduceBlocks * 7 * sizeof(double))) ||
      !chk(alloc_copy((void**)&s->d_cells, nullptr, 64 * sizeof(int32_t))) ||
      !chk(alloc_copy((void**)&s->d_gather, nullptr, 64 * 9 * sizeof(double))))
    return nullptr;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
    fail(VL_ECUDA, "stream/event creation");
    return nullptr;
  }
  // Launch geometry: one bulk block per row tile of kBlock cells; one link thread per boundary
  // node, and at least one link block (it runs the end-of-step epilogue).
  const bool forced = d.accel[0] != 0.0 || d.accel[1] != 0.0;
  s->ck = forced ? 2 : (d.collision == vl::COLL_BGK ? 0 : 1);
  vl::StepParams& P = s->P;
  P.nx = (int)d.nx;
  P.ny = (int)d.ny;
  P.ns = s->ns;
  P.tiles_per_row = (int)((d.nx + vl::kBlock - 1) / vl::kBlock);
  P.ntiles = P.tiles_per_row * (int)d.ny;
  P.nbulk = P.ntiles;
  const int nb = (int)d.bnode_idx.size();
  P.nlink = std::max(1, (nb + vl::kBlock - 1) / vl::kBlock);
  s->kernels_per_step = 2;
  P.coll = d.collision;
  P.forced = forced ? 1 : 0;
  P.op = d.op;
  P.om = d.om;
  P.gx = d.accel[0];
  P.gy = d.accel[1];
  P.sqrt_cs2 = std::sqrt(1.0 / 3.0);
  P.flag = s->d_flag;
  P.bnode_idx = s->d_bidx;
  P.bnode_first = s->d_bfirst;
  P.nb = nb;
  P.links = s->d_links;
  P.pnode_idx = s->d_pidx;
  P.pnode_n = s->d_pn;
  P.np = (int)d.pnode_idx.size();
  P.ctl = s->d_ctl;
  P.ngroups = d.ngroups;
  P.nlinks = (int)d.links.size();
  P.nlinkblk = std::max(1, (P.nlinks + vl::kBlock * vl::kStagePer - 1) / (vl::kBlock * vl::kStagePer));
  if (!chk(alloc_copy((void**)&s->d_partials, nullptr,
                      (size_t)std::max(P.nlink, P.nlinkblk) * 2 * vl::kMaxGroups * sizeof(double))))
    return nullptr;
  P.partials = s->d_partials;
  // Staged step: node descriptors, per-warp boundary ranks and the per-link output.
  std::vector<int2> bdesc;
  std::vector<int32_t> wbfirst;
  std::string serr;
  if (!staged_tables(d, P.tiles_per_row, bdesc, wbfirst, serr)) {
    fail(VL_EINVAL, serr.c_str());
    return nullptr;
  }
  const size_t r_elem = precision == VL_F64 ? sizeof(double) : sizeof(float);
  if (!chk(alloc_copy((void**)&s->d_bdesc, bdesc.data(), bdesc.size() * sizeof(int2))) ||
      !chk(alloc_copy((void**)&s->d_wbfirst, wbfirst.data(), wbfirst.size() * sizeof(int32_t))) ||
      !chk(alloc_copy(&s->d_lb, nullptr, d.links.size() * r_elem)))
    return nullptr;
  P.nbs = (unsigned)((nb + 63) / 64 * 64);
  if (!chk(alloc_copy(&s->d_ownc, nullptr, (size_t)P.nbs * 9 * s->L->elem))) return nullptr;
  std::vector<int32_t> lnode(d.links.size());
  for (int k = 0; k < nb; ++k)
    for (int l = d.bnode_first[k]; l < d.bnode_first[k + 1]; ++l) lnode[(size_t)l] = k;
  if (!chk(alloc_copy((void**)&s->d_lnode, lnode.data(), lnode.size() * sizeof(int32_t)))) return nullptr;
  P.lnode = s->d_lnode;
  P.link_b0 = 0;
  P.link_n = P.nlinkblk;
  P.bulk_b0 = 0;
  P.bulk_n = P.ny;
  // cells per thread of the narrow bulk kernel: 2 for FP32 (its 4-cell form needs twice the
  // registers and ran slower on the box), 4 for the 16-bit formats
  P.pairs = precision == VL_F32 ? 2 : 4;
  P.stream = 0;
  // Narrow formats: each bulk-kernel block prefetches into the L2 the tile about two waves of
  // blocks ahead (2 x SMs blocks, in rows of the multi-cell tiling); measured +4.5 % (FP32) and
  // +9.5 % (IEEE half) on the 8192 x 4096 box. FP64, whose one-cell kernel keeps 64 warps of loads
  // in flight per SM, ran slower with it and does not prefetch.
  P.prefetch_rows = 0;
  if (precision != VL_F64) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int v = d.nx % 4 == 0 && P.pairs >= 4 ? 4 : (d.nx % 2 == 0 && P.pairs >= 2 ? 2 : 1);
    const int tiles = (int)((d.nx + v * vl::kBlock - 1) / (v * vl::kBlock));
    P.prefetch_rows = std::min((int)d.ny - 1, std::max(1, (2 * sms + tiles - 1) / tiles));
  }
  staged_split(d, lnode, s->split_links, s->split_rows);
  P.bdesc = s->d_bdesc;
  P.warp_bfirst = s->d_wbfirst;
  P.lb = s->d_lb;
  P.ownc = s->d_ownc;
  // Control block: vscale = 1, no outflow target (src/sim.rs:344-347).
  std::memset(&s->hctl, 0, sizeof(vl::Ctl));
  for (int g = 0; g < 4; ++g) s->hctl.vscale[g] = 1.0;
  for (int k = 0; k < vl::kProbeCorners; ++k) s->hctl.probe_idx[k] = -1;
  if (s->push_ctl() != VL_OK) return nullptr;
  // Sim::from_builder ends with init to (1, 0, 0) (src/sim.rs:352).
  if (vl_sim_init(s.get(), nullptr, nullptr, nullptr, 1.0, 0.0, 0.0) != VL_OK) return nullptr;
  return s.release();
}

}  // namespace

// ==================================================================== C ABI
extern "C" {

const char* vl_last_error(void) { return g_err.c_str(); }
int vl_last_status(void) { return g_code; }
int vl_abi_version(void) { return VL_ABI_VERSION; }
int vl_set_device(int device) {
  VL_CUDA(cudaSetDevice(device));
  return VL_OK;
}
void* vl_pinned_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
    cudaGetLastError();
    fail(VL_ENOMEM, "cudaMallocHost failed");
    return nullptr;
  }
  return p;
}
void vl_pinned_free(void* p) {
  if (p) cudaFreeHost(p);
}
int vl_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// ---------------------------------------------------------------- shapes
vl_shape* vl_shape_circle(double cx, double cy, double r) { return wrap_shape(std::make_unique<vl::CircleShape>(cx, cy, r)); }
vl_shape* vl_shape_polygon(const double* xy, size_t npts) {
  if (!xy || npts < 3) { fail(VL_EINVAL, "polygon needs at least 3 points"); return nullptr; }
  auto p = std::make_unique<vl::PolygonShape>();
  for (size_t k = 0; k < npts; ++k) { p->vx.push_back(xy[2 * k]); p->vy.push_back(xy[2 * k + 1]); }
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_rounded_square(double cx, double cy, double half, double r) {
  auto p = std::make_unique<vl::RoundedSquareShape>();
  p->cx = cx; p->cy = cy; p->half = half; p->r = r;
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_rotated(vl_shape* inner, double cx, double cy, double angle) {
  if (!inner) { fail(VL_EINVAL, "null inner shape"); return nullptr; }
  auto p = std::make_unique<vl::RotatedShape>();
  p->inner = std::move(inner->s); delete inner;
  p->cx = cx; p->cy = cy; p->angle = angle;
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_translated(vl_shape* inner, double dx, double dy) {
  if (!inner) { fail(VL_EINVAL, "null inner shape"); return nullptr; }
  auto p = std::make_unique<vl::TranslatedShape>();
  p->inner = std::move(inner->s); delete inner;
  p->dx = dx; p->dy = dy;
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_section(int corner, double b, double cx, double cy, double d, double angle) {
  if (corner < 0 || corner > 4) { fail(VL_EINVAL, "unknown corner kind"); return nullptr; }
  return wrap_shape(vl::make_section(corner, b, cx, cy, d, angle));
}
vl_shape* vl_shape_bitmap(size_t w, size_t h, const float* level, double x0, double y0, double scale) {
  if (!level || w == 0 || h == 0) { fail(VL_EINVAL, "empty bitmap"); return nullptr; }
  auto p = std::make_unique<vl::BitmapShape>();
  p->w = w; p->h = h; p->level.assign(level, level + w * h);
  p->x0 = x0; p->y0 = y0; p->scale = scale;
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_outside_band(double y0, double y1) {
  auto p = std::make_unique<vl::OutsideBandShape>();
  p->y0 = y0; p->y1 = y1;
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_ellipse(double cx, double cy, double a, double b) {
  if (!(a > 0.0 && b > 0.0)) { fail(VL_EINVAL, "ellipse semi-axes must be positive"); return nullptr; }
  auto p = std::make_unique<vl::EllipseShape>();
  p->cx = cx; p->cy = cy; p->a = a; p->b = b;
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_disks(const double* cxcyr, size_t ndisks) {
  if (!cxcyr || ndisks == 0) { fail(VL_EINVAL, "disk union needs at least one disk"); return nullptr; }
  auto p = std::make_unique<vl::DiskUnionShape>();
  for (size_t k = 0; k < ndisks; ++k) {
    p->cx.push_back(cxcyr[3 * k]);
    p->cy.push_back(cxcyr[3 * k + 1]);
    p->r.push_back(cxcyr[3 * k + 2]);
  }
  p->index();
  return wrap_shape(std::move(p));
}
vl_shape* vl_shape_star(double cx, double cy, const double* radii, size_t nvert, double phase) {
  if (!radii || nvert < 3) { fail(VL_EINVAL, "star polygon needs at least 3 vertices"); return nullptr; }
  return wrap_shape(vl::make_star(cx, cy, radii, nvert, phase));
}
void vl_shape_free(vl_shape* s) { delete s; }
int vl_shape_inside(const vl_shape* s, double x, double y) { return s && s->s->inside(x, y) ? 1 : 0; }
double vl_cut_fraction(const vl_shape* s, double x, double y, double dx, double dy) {
  return s ? vl::cut_fraction(*s->s, x, y, dx, dy) : std::nan("");
}
int vl_bounding_box(const vl_shape* s, double reach, double step, double* out) {
  if (!s || !out || !(step > 0.0)) return fail(VL_EINVAL, "bounding_box: bad arguments");
  return vl::bounding_box(*s->s, reach, step, out) ? 1 : 0;
}

// ---------------------------------------------------------------- builder
vl_builder* vl_builder_new(size_t nx, size_t ny) {
  if (nx < 3 || ny < 3) { fail(VL_EINVAL, "grid must be at least 3 x 3"); return nullptr; }
  auto b = new vl_builder();
  b->spec.nx = nx;
  b->spec.ny = ny;
  b->spec.kinds.emplace_back();
  b->spec.paint.assign(nx * ny, 0);
  return b;
}
void vl_builder_free(vl_builder* b) { delete b; }
int vl_builder_set_periodic(vl_builder* b, int px, int py) {
  if (!b) return fail(VL_EINVAL, "null builder");
  b->spec.periodic_x = px != 0;
  b->spec.periodic_y = py != 0;
  return VL_OK;
}
int vl_builder_set_tau(vl_builder* b, double tau) {
  if (!b) return fail(VL_EINVAL, "null builder");
  b->spec.tau = tau;
  return VL_OK;
}
int vl_builder_set_collision(vl_builder* b, int collision, double magic) {
  if (!b || (collision != VL_BGK && collision != VL_TRT)) return fail(VL_EINVAL, "bad collision model");
  b->spec.collision = collision;
  b->spec.magic = magic;
  return VL_OK;
}
int vl_builder_set_accel(vl_builder* b, double gx, double gy) {
  if (!b) return fail(VL_EINVAL, "null builder");
  b->spec.accel[0] = gx;
  b->spec.accel[1] = gy;
  return VL_OK;
}
static int add_kind(vl_builder* b, vl::CellKind&& k) {
  if (b->spec.kinds.size() >= 255) return fail(VL_EINVAL, "at most 254 cell kinds (src/sim.rs:101)");
  b->spec.kinds.push_back(std::move(k));
  return (int)b->spec.kinds.size() - 1;
}
int vl_builder_add_wall(vl_builder* b, const vl_wall* w) {
  std::unique_ptr<vl::Shape> shape;
  if (w && w->shape) { shape = std::move(w->shape->s); delete w->shape; }
  if (!b || !w) return fail(VL_EINVAL, "null builder or wall");
  if (w->vgroup < 0 || w->vgroup >= VL_VGROUPS) return fail(VL_EINVAL, "vgroup must be below 4 (src/sim.rs:303)");
  if (w->fgroup >= VL_MAX_FGROUPS) return fail(VL_EINVAL, "force group must be below VL_MAX_FGROUPS (4)");
  if (w->velocity.kind < VL_VEL_NONE || w->velocity.kind > VL_VEL_ROTATION) return fail(VL_EINVAL, "unknown velocity kind");
  vl::CellKind k;
  k.tag = vl::KIND_WALL;
  k.velocity.kind = w->velocity.kind;
  for (int i = 0; i < 4; ++i) k.velocity.p[i] = w->velocity.p[i];
  k.vgroup = w->vgroup;
  k.fgroup = w->fgroup < 0 ? -1 : w->fgroup;
  k.shape = std::move(shape);
  return add_kind(b, std::move(k));
}
int vl_builder_add_static_wall(vl_builder* b) {
  if (!b) return fail(VL_EINVAL, "null builder");
  vl::CellKind k;
  k.tag = vl::KIND_WALL;
  return add_kind(b, std::move(k));
}
int vl_builder_add_pressure(vl_builder* b, double rho) {
  if (!b) return fail(VL_EINVAL, "null builder");
  vl::CellKind k;
  k.tag = vl::KIND_PRESSURE;
  k.rho = rho;
  return add_kind(b, std::move(k));
}
int vl_builder_add_radiating(vl_builder* b, double rho) {
  if (!b) return fail(VL_EINVAL, "null builder");
  vl::CellKind k;
  k.tag = vl::KIND_RADIATING;
  k.rho = rho;
  return add_kind(b, std::move(k));
}
int vl_builder_fill_rect(vl_builder* b, size_t x0, size_t x1, size_t y0, size_t y1, int kind) {
  if (!b) return fail(VL_EINVAL, "null builder");
  if (kind < 0 || (size_t)kind >= b->spec.kinds.size()) return fail(VL_EINVAL, "unknown kind");
  if (x1 >= b->spec.nx || y1 >= b->spec.ny) return fail(VL_EINVAL, "rectangle outside the grid");
  for (size_t y = y0; y <= y1; ++y)
    for (size_t x = x0; x <= x1; ++x) b->spec.paint[y * b->spec.nx + x] = (uint8_t)kind;
  return VL_OK;
}
int vl_builder_fill_shape(vl_builder* b, int kind) {
  if (!b) return fail(VL_EINVAL, "null builder");
  if (kind < 0 || (size_t)kind >= b->spec.kinds.size()) return fail(VL_EINVAL, "unknown kind");
  const vl::CellKind& k = b->spec.kinds[kind];
  if (k.tag != vl::KIND_WALL || !k.shape) return fail(VL_EINVAL, "fill_shape needs a wall kind with an outline");
  for (size_t y = 0; y < b->spec.ny; ++y)
    for (size_t x = 0; x < b->spec.nx; ++x)
      if (k.shape->inside((double)x, (double)y)) b->spec.paint[y * b->spec.nx + x] = (uint8_t)kind;
  return VL_OK;
}
int vl_builder_link_table(vl_builder* b, size_t* nlinks, size_t* nbnodes, size_t* npnodes, uint8_t* flags,
                          int32_t* bnode_idx, int32_t* bnode_first, double* link_f64, int32_t* link_i32) {
  if (!b || !nlinks || !nbnodes || !npnodes) return fail(VL_EINVAL, "null argument");
  vl::CompiledDomain dom;
  std::string err;
  if (!vl::compile_domain(b->spec, dom, err)) return fail(VL_EINVAL, err);
  *nlinks = dom.links.size();
  *nbnodes = dom.bnode_idx.size();
  *npnodes = dom.pnode_idx.size();
  if (flags) std::memcpy(flags, dom.flag.data(), dom.n);
  if (bnode_idx) std::memcpy(bnode_idx, dom.bnode_idx.data(), dom.bnode_idx.size() * 4);
  if (bnode_first) std::memcpy(bnode_first, dom.bnode_first.data(), dom.bnode_first.size() * 4);
  for (size_t k = 0; k < dom.links.size(); ++k) {
    const vl::LinkRec& L = dom.links[k];
    if (link_f64) {
      double* o = link_f64 + 5 * k;
      o[0] = L.q; o[1] = L.cu6; o[2] = L.uw[0]; o[3] = L.uw[1]; o[4] = L.rho;
    }
    if (link_i32) {
      int32_t* o = link_i32 + 7 * k;
      o[0] = L.dir; o[1] = L.flags & 1; o[2] = (L.flags >> 1) & 1; o[3] = L.vgroup; o[4] = L.fgroup;
      o[5] = L.behind; o[6] = ((L.flags >> 2) & 3) - 1 + 3 * (((L.flags >> 4) & 3) - 1 + 1) + 1;
    }
  }
  return VL_OK;
}

int vl_builder_stage_split(vl_builder* b, int* links_per_block, int* link_blocks, int* split_blocks,
                           int* split_rows) {
  if (!b) return fail(VL_EINVAL, "null builder");
  vl::CompiledDomain dom;
  std::string err;
  if (!vl::compile_domain(b->spec, dom, err)) return fail(VL_EINVAL, err);
  std::vector<int32_t> lnode(dom.links.size());
  for (size_t k = 0; k + 1 < dom.bnode_first.size(); ++k)
    for (int l = dom.bnode_first[k]; l < dom.bnode_first[k + 1]; ++l) lnode[(size_t)l] = (int32_t)k;
  const int per = vl::kBlock * vl::kStagePer;
  int sl = 0, sr = 0;
  staged_split(dom, lnode, sl, sr);
  if (links_per_block) *links_per_block = per;
  if (link_blocks) *link_blocks = std::max(1, ((int)dom.links.size() + per - 1) / per);
  if (split_blocks) *split_blocks = sl;
  if (split_rows) *split_rows = sr;
  return VL_OK;
}

vl_sim* vl_builder_build(vl_builder* b, int precision) {
  if (!b) { fail(VL_EINVAL, "null builder"); return nullptr; }
  std::unique_ptr<vl_builder> own(b);
  vl::CompiledDomain dom;
  std::string err;
  if (!vl::compile_domain(b->spec, dom, err)) { fail(VL_EINVAL, err); return nullptr; }
  return make_sim(std::move(dom), precision);
}

// ---------------------------------------------------------------- sim
void vl_sim_free(vl_sim* s) { delete s; }

int vl_sim_info(const vl_sim* s, size_t* nx, size_t* ny, size_t* fluid, size_t* nlinks, size_t* nbn, int* ngroups,
                int* prec) {
  if (!s) return fail(VL_EINVAL, "null sim");
  if (nx) *nx = s->dom.nx;
  if (ny) *ny = s->dom.ny;
  if (fluid) *fluid = s->dom.fluid_nodes;
  if (nlinks) *nlinks = s->dom.links.size();
  if (nbn) *nbn = s->dom.bnode_idx.size();
  if (ngroups) *ngroups = s->dom.ngroups;
  if (prec) *prec = s->prec;
  return VL_OK;
}

int vl_sim_init(vl_sim* s, const double* rho, const double* ux, const double* uy, double rho0, double ux0, double uy0) {
  if (!s) return fail(VL_EINVAL, "null sim");
  if ((rho || ux || uy) && !(rho && ux && uy)) return fail(VL_EINVAL, "init: give all three field arrays or none");
  VL_CUDA(cudaSetDevice(s->device));
  double* d_field = nullptr;
  const size_t n = s->n;
  if (rho) {
    VL_CUDA(cudaMalloc(&d_field, 3 * n * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(d_field, rho, n * 8, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_field + n, ux, n * 8, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_field + 2 * n, uy, n * 8, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) { cudaFree(d_field); return cuda_fail(e, "init upload"); }
  }
  cudaError_t e = s->L->init((int)n, s->ns, s->d_flag, d_field, d_field ? d_field + n : nullptr,
                             d_field ? d_field + 2 * n : nullptr, rho0, ux0, uy0, s->buf[0], s->buf[1], s->stream);
  if (d_field) {
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    cudaFree(d_field);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) return cuda_fail(e, "init");
  s->own_ok = false;
  // t = 0 (src/sim.rs:370); the force and the outlet offset restart from zero.
  int rc = s->pull_ctl();
  if (rc) return rc;
  s->hctl.t = 0;
  s->hctl.arrive = 0;
  s->hctl.nonfinite = 0;
  s->hctl.nonfinite_t = 0;
  s->hctl.drho = 0.0;
  for (int k = 0; k < 2 * vl::kMaxGroups; ++k) s->hctl.force[k] = 0.0;
  s->t_host = 0;
  if (s->rec_cap) s->hctl.rec_start = 0;
  s->rec_start = 0;
  return s->push_ctl();
}

int vl_sim_step(vl_sim* s, uint64_t steps) {
  if (!s) return fail(VL_EINVAL, "null sim");
  return s->step(steps);
}

int vl_sim_synchronize(vl_sim* s) {
  if (!s) return fail(VL_EINVAL, "null sim");
  VL_CUDA(cudaStreamSynchronize(s->stream));
  return VL_OK;
}

int vl_sim_set_vscale(vl_sim* s, int g, double v) {
  if (!s || g < 0 || g >= VL_VGROUPS) return fail(VL_EINVAL, "vscale group out of range");
  int rc = s->pull_ctl();
  if (rc) return rc;
  s->hctl.vscale[g] = v;
  return s->push_ctl();
}

int vl_sim_get_vscale(const vl_sim* cs, double* out4) {
  vl_sim* s = const_cast<vl_sim*>(cs);
  if (!s || !out4) return fail(VL_EINVAL, "null argument");
  int rc = s->pull_ctl();
  if (rc) return rc;
  for (int g = 0; g < 4; ++g) out4[g] = s->hctl.vscale[g];
  return VL_OK;
}

int vl_sim_set_outflow_target(vl_sim* s, int enabled, double target) {
  if (!s) return fail(VL_EINVAL, "null sim");
  int rc = s->pull_ctl();
  if (rc) return rc;
  s->hctl.has_target = enabled ? 1 : 0;
  s->hctl.target = target;
  return s->push_ctl();
}

int vl_sim_outlet_density_offset(vl_sim* s, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  int rc = s->pull_ctl();
  if (rc) return rc;
  *out = s->hctl.drho;
  return VL_OK;
}

int vl_sim_t(vl_sim* s, uint64_t* t) {
  if (!s || !t) return fail(VL_EINVAL, "null argument");
  int rc = s->pull_ctl();
  if (rc) return rc;
  *t = s->hctl.t;
  return VL_OK;
}

int vl_sim_force(vl_sim* s, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  int rc = s->pull_ctl();
  if (rc) return rc;
  for (int k = 0; k < 2 * s->dom.ngroups; ++k) out[k] = s->hctl.force[k];
  return VL_OK;
}

int vl_sim_status(vl_sim* s, int* nonfinite, uint64_t* first_t) {
  if (!s) return fail(VL_EINVAL, "null sim");
  int rc = s->pull_ctl();
  if (rc) return rc;
  if (nonfinite) *nonfinite = s->hctl.nonfinite;
  if (first_t) *first_t = s->hctl.nonfinite_t;
  return VL_OK;
}

int vl_sim_download(vl_sim* s, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  VL_CUDA(cudaSetDevice(s->device));
  const size_t n = s->n;
  if (s->prec == VL_F64) {
    VL_CUDA(cudaMemcpy2DAsync(out, n * 8, s->a(), (size_t)s->ns * 8, n * 8, 9, cudaMemcpyDeviceToHost, s->stream));
  } else {
    double* tmp = nullptr;
    VL_CUDA(cudaMalloc(&tmp, 9 * n * sizeof(double)));
    cudaError_t e = s->L->to_f64((int)n, s->ns, s->a(), tmp, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, 9 * n * 8, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "download");
  }
  VL_CUDA(cudaStreamSynchronize(s->stream));
  return VL_OK;
}

int vl_sim_upload(vl_sim* s, const double* in) {
  if (!s || !in) return fail(VL_EINVAL, "null argument");
  VL_CUDA(cudaSetDevice(s->device));
  s->own_ok = false;
  const size_t n = s->n;
  if (s->prec == VL_F64) {
    VL_CUDA(cudaMemcpy2DAsync(s->buf[s->cur], (size_t)s->ns * 8, in, n * 8, n * 8, 9, cudaMemcpyHostToDevice, s->stream));
  } else {
    double* tmp = nullptr;
    VL_CUDA(cudaMalloc(&tmp, 9 * n * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(tmp, in, 9 * n * 8, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = s->L->from_f64((int)n, s->ns, tmp, s->buf[s->cur], s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "upload");
  }
  VL_CUDA(cudaStreamSynchronize(s->stream));
  return VL_OK;
}

int vl_sim_flags(vl_sim* s, uint8_t* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  std::memcpy(out, s->dom.flag.data(), s->n);
  return VL_OK;
}

int vl_sim_macros_field(vl_sim* s, double* rho, double* ux, double* uy) {
  if (!s || !rho || !ux || !uy) return fail(VL_EINVAL, "null argument");
  VL_CUDA(cudaSetDevice(s->device));
  const size_t n = s->n;
  double* tmp = nullptr;
  VL_CUDA(cudaMalloc(&tmp, 3 * n * sizeof(double)));
  cudaError_t e = s->L->macros((int)n, s->ns, s->d_flag, s->dom.accel[0], s->dom.accel[1], s->a(), tmp, tmp + n,
                               tmp + 2 * n, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rho, tmp, n * 8, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ux, tmp + n, n * 8, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(uy, tmp + 2 * n, n * 8, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(e, "macros_field");
  return VL_OK;
}

int vl_sim_macros(vl_sim* s, size_t x, size_t y, double* out3) {
  if (!s || !out3 || x >= s->dom.nx || y >= s->dom.ny) return fail(VL_EINVAL, "macros: bad arguments");
  const size_t idx = y * s->dom.nx + x;
  if (s->dom.flag[idx] == 2) { out3[0] = 1.0; out3[1] = 0.0; out3[2] = 0.0; return VL_OK; }
  std::vector<double> f;
  int rc = s->gather({(int32_t)idx}, f);
  if (rc) return rc;
  double rho, jx, jy;
  moments_host(f.data(), rho, jx, jy);
  out3[0] = rho;
  out3[1] = jx / rho - 0.5 * s->dom.accel[0];
  out3[2] = jy / rho - 0.5 * s->dom.accel[1];
  return VL_OK;
}

static int sim_reduce(vl_sim* s, double* mass, double* mom, double* vmax) {
  VL_CUDA(cudaSetDevice(s->device));
  cudaError_t e = s->L->reduce((int)s->n, s->ns, s->d_flag, s->dom.accel[0], s->dom.accel[1], s->a(), s->d_red,
                               kReduceBlocks, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "reduce");
  std::vector<double> r(kReduceBlocks * 7);
  VL_CUDA(cudaMemcpyAsync(r.data(), s->d_red, r.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  VL_CUDA(cudaStreamSynchronize(s->stream));
  // Fixed-order combination of the per-block compensated sums.
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double vm = 0.0;
  bool nan = false;
  for (int b = 0; b < kReduceBlocks; ++b) {
    const double* o = &r[7 * b];
    for (int k = 0; k < 3; ++k) {
      double& sum = acc[2 * k];
      double& comp = acc[2 * k + 1];
      const double x = o[2 * k];
      const double t = sum + x;
      comp += std::fabs(sum) >= std::fabs(x) ? (sum - t) + x : (x - t) + sum;
      sum = t;
      comp += o[2 * k + 1];
    }
    if (std::isnan(o[6])) nan = true; else vm = std::fmax(vm, o[6]);
  }
  if (mass) *mass = acc[0] + acc[1];
  if (mom) { mom[0] = acc[2] + acc[3]; mom[1] = acc[4] + acc[5]; }
  if (vmax) *vmax = nan ? std::nan("") : vm;
  return VL_OK;
}

int vl_sim_total_mass(vl_sim* s, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  return sim_reduce(s, out, nullptr, nullptr);
}
int vl_sim_total_momentum(vl_sim* s, double* out2) {
  if (!s || !out2) return fail(VL_EINVAL, "null argument");
  return sim_reduce(s, nullptr, out2, nullptr);
}
int vl_sim_max_speed(vl_sim* s, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  return sim_reduce(s, nullptr, nullptr, out);
}

// Sim::vorticity (src/sim.rs:582-620): central differences, one-sided next to solids.
int vl_sim_vorticity(vl_sim* s, float* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  const size_t nx = s->dom.nx, ny = s->dom.ny, n = s->n;
  std::vector<double> rho(n), ux(n), uy(n);
  int rc = vl_sim_macros_field(s, rho.data(), ux.data(), uy.data());
  if (rc) return rc;
  for (size_t k = 0; k < n; ++k) {
    out[k] = 0.0f;
    if (s->dom.flag[k] == 2) { ux[k] = 0.0; uy[k] = 0.0; }
  }
  auto fluid = [&](long x, long y) {
    return x >= 0 && y >= 0 && x < (long)nx && y < (long)ny && s->dom.flag[(size_t)y * nx + (size_t)x] != 2;
  };
  auto get = [&](long x, long y, int comp) {
    const size_t k = (size_t)y * nx + (size_t)x;
    return comp == 0 ? ux[k] : uy[k];
  };
  for (long y = 0; y < (long)ny; ++y) {
    for (long x = 0; x < (long)nx; ++x) {
      if (!fluid(x, y)) continue;
      auto diff = [&](long dx, long dy, int comp) -> double {
        const bool p = fluid(x + dx, y + dy), m = fluid(x - dx, y - dy);
        if (p && m) return 0.5 * (get(x + dx, y + dy, comp) - get(x - dx, y - dy, comp));
        if (p) return get(x + dx, y + dy, comp) - get(x, y, comp);
        if (m) return get(x, y, comp) - get(x - dx, y - dy, comp);
        return 0.0;
      };
      out[(size_t)y * nx + (size_t)x] = (float)(diff(1, 0, 1) - diff(0, 1, 0));
    }
  }
  return VL_OK;
}

int vl_sim_probe_density(vl_sim* s, double x, double y, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  return sim_probe_density(s, x, y, out);
}

int vl_sim_probe_density_at_wall(vl_sim* s, double x, double y, double nx, double ny, double* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  double p[3];
  for (int d = 1; d <= 3; ++d) {
    int rc = sim_probe_density(s, x + (double)d * nx, y + (double)d * ny, &p[d - 1]);
    if (rc) return rc;
  }
  *out = 3.0 * p[0] - 3.0 * p[1] + p[2];
  return VL_OK;
}

// FNV-1a over the little-endian bytes of every fluid population, cell-major (src/sim.rs:654-668).
int vl_sim_state_hash(vl_sim* s, uint64_t* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  const size_t n = s->n;
  std::vector<double> f(9 * n);
  int rc = vl_sim_download(s, f.data());
  if (rc) return rc;
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t idx = 0; idx < n; ++idx) {
    if (s->dom.flag[idx] == 2) continue;
    for (int i = 0; i < 9; ++i) {
      uint64_t bits;
      std::memcpy(&bits, &f[(size_t)i * n + idx], 8);
      for (int k = 0; k < 8; ++k) {
        h ^= (bits >> (8 * k)) & 0xffu;
        h *= 0x100000001b3ull;
      }
    }
  }
  *out = h;
  return VL_OK;
}

int vl_sim_record(vl_sim* s, uint64_t capacity) {
  if (!s) return fail(VL_EINVAL, "null sim");
  VL_CUDA(cudaSetDevice(s->device));
  int rc = s->pull_ctl();
  if (rc) return rc;
  if (capacity > s->rec_cap || capacity == 0) {
    if (s->d_hist) { cudaFree(s->d_hist); s->d_hist = nullptr; }
    if (capacity) VL_CUDA(cudaMalloc(&s->d_hist, capacity * vl::kRec * sizeof(double)));
  }
  s->rec_cap = capacity;
  s->rec_start = s->hctl.t;
  s->hctl.hist = s->d_hist;
  s->hctl.rec_cap = capacity;
  s->hctl.rec_start = s->hctl.t;
  return s->push_ctl();
}

int vl_sim_history(vl_sim* s, double* out, uint64_t* count) {
  if (!s || !count) return fail(VL_EINVAL, "null argument");
  int rc = s->pull_ctl();
  if (rc) return rc;
  uint64_t have = s->hctl.t >= s->hctl.rec_start ? s->hctl.t - s->hctl.rec_start : 0;
  have = std::min(have, s->rec_cap);
  if (out && have) {
    VL_CUDA(cudaMemcpyAsync(out, s->d_hist, have * vl::kRec * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    VL_CUDA(cudaStreamSynchronize(s->stream));
  }
  *count = have;
  return VL_OK;
}

int vl_sim_set_dp_probe(vl_sim* s, double xc, double yc, double r, double u_ref) {
  if (!s) return fail(VL_EINVAL, "null sim");
  int rc = s->pull_ctl();
  if (rc) return rc;
  // Front wall point (xc - r, yc) with outward normal (-1, 0), back (xc + r, yc) with (1, 0);
  // samples at distances 1, 2, 3 (src/sim.rs:648-651, src/cases/cylinder.rs:54-59).
  const double wx[2] = {xc - r, xc + r}, nxv[2] = {-1.0, 1.0};
  for (int side = 0; side < 2; ++side)
    for (int d = 0; d < 3; ++d) {
      const int base = (side * 3 + d) * 4;
      probe_corners(*s, wx[side] + (double)(d + 1) * nxv[side], yc + (double)(d + 1) * 0.0, &s->hctl.probe_idx[base],
                    &s->hctl.probe_w[base]);
    }
  s->hctl.dp_on = 1;
  s->hctl.u_ref = u_ref;
  return s->push_ctl();
}

int vl_sim_last_step_ms(vl_sim* s, float* ms) {
  if (!s || !ms) return fail(VL_EINVAL, "null argument");
  if (!s->timed) return fail(VL_EINVAL, "no step batch timed yet");
  VL_CUDA(cudaEventSynchronize(s->ev1));
  VL_CUDA(cudaEventElapsedTime(ms, s->ev0, s->ev1));
  return VL_OK;
}

int vl_sim_set_schedule(vl_sim* s, int schedule) {
  if (!s) return fail(VL_EINVAL, "null sim");
  return s->set_schedule(schedule);
}

int vl_sim_get_schedule(const vl_sim* s) { return s ? s->schedule : VL_EINVAL; }

int vl_sim_set_prefetch_rows(vl_sim* s, int rows) {
  if (!s) return fail(VL_EINVAL, "null sim");
  return s->set_prefetch_rows(rows);
}

int vl_sim_set_bulk_copies(vl_sim* s, int on) {
  if (!s) return fail(VL_EINVAL, "null sim");
  return s->set_bulk_copies(on);
}

int vl_sim_set_cells_per_thread(vl_sim* s, int cells) {
  if (!s) return fail(VL_EINVAL, "null sim");
  return s->set_cells_per_thread(cells);
}

int vl_sim_autotune(vl_sim* s, int steps_each, double* ms3) {
  if (!s || steps_each < 1) return fail(VL_EINVAL, "autotune: bad arguments");
  return s->autotune(steps_each, ms3);
}

int vl_sim_step_profiled(vl_sim* s, uint64_t steps, double* link_ms, double* bulk_ms, double* total_ms) {
  if (!s || steps == 0) return fail(VL_EINVAL, "step_profiled: bad arguments");
  return s->step_profiled(steps, link_ms, bulk_ms, total_ms);
}

int vl_sim_launch_count(vl_sim* s, uint64_t* out) {
  if (!s || !out) return fail(VL_EINVAL, "null argument");
  *out = s->launches;
  return VL_OK;
}

// ---------------------------------------------------------------- channel (src/cases/channel.rs)
}  // extern "C"

struct vl_channel {
  vl_sim* sim = nullptr;
  double u_ref = 0.0;
  uint64_t ramp_steps = 0;
  ~vl_channel() { delete sim; }
};

// Everything Channel::new and Channel::step decide on the host (src/cases/channel.rs:71-130): the
// compiled domain, whether to start from the inflow profile, and the per-step control schedule
// (inlet ramp, body kick) up to the step after which both are constant.
int vl::plan_channel(const vl_channel_spec* sp, std::unique_ptr<vl::Shape> body, ChannelPlan& out) {
  if (!body) return fail(VL_EINVAL, "channel needs a body shape");
  const size_t nx = sp->nx, ny = sp->ny;
  if (nx < 3 || ny < 3) return fail(VL_EINVAL, "grid must be at least 3 x 3");
  if (sp->inflow < 0 || sp->inflow > 2) return fail(VL_EINVAL, "unknown inflow");
  // Inlet (moving wall, vgroup 1) at x = 0, outlet (pressure 1) at x = nx-1, side walls, body
  // (vgroup 2, force group 0).
  const double h = (double)(ny - 2);
  vl::DomainSpec spec;
  spec.nx = nx;
  spec.ny = ny;
  spec.tau = vl_tau_for(sp->nu);
  spec.collision = sp->collision;
  spec.magic = sp->magic;
  spec.kinds.emplace_back();
  spec.paint.assign(nx * ny, 0);
  vl::WallVelocity profile;
  if (sp->inflow == VL_INFLOW_PARABOLIC) { profile.kind = vl::VEL_PARABOLIC; profile.p[0] = sp->u; profile.p[1] = h; }
  else { profile.kind = vl::VEL_CONST; profile.p[0] = sp->u; }
  auto add = [&](vl::CellKind&& k) {
    spec.kinds.push_back(std::move(k));
    return (uint8_t)(spec.kinds.size() - 1);
  };
  auto fill = [&](size_t x0, size_t x1, size_t y0, size_t y1, uint8_t k) {
    for (size_t y = y0; y <= y1; ++y)
      for (size_t x = x0; x <= x1; ++x) spec.paint[y * nx + x] = k;
  };
  vl::CellKind inlet;
  inlet.tag = vl::KIND_WALL;
  inlet.velocity = profile;
  inlet.vgroup = 1;
  const uint8_t k_in = add(std::move(inlet));
  vl::CellKind outlet;
  outlet.tag = vl::KIND_PRESSURE;
  outlet.rho = 1.0;
  const uint8_t k_out = add(std::move(outlet));
  vl::CellKind walls;
  if (sp->inflow == VL_INFLOW_PARABOLIC) walls.tag = vl::KIND_WALL;
  else if (sp->inflow == VL_INFLOW_UNIFORM) {
    walls.tag = vl::KIND_WALL;
    walls.velocity.kind = vl::VEL_CONST;
    walls.velocity.p[0] = sp->u;
    walls.vgroup = 1;
  } else {
    walls.tag = vl::KIND_RADIATING;
    walls.rho = 1.0;
  }
  const uint8_t k_w = add(std::move(walls));
  fill(0, 0, 0, ny - 1, k_in);
  fill(nx - 1, nx - 1, 0, ny - 1, k_out);
  fill(1, nx - 2, 0, 0, k_w);
  fill(1, nx - 2, ny - 1, ny - 1, k_w);
  if (sp->inflow != VL_INFLOW_UNIFORM_OPEN) {
    fill(0, nx - 1, 0, 0, k_w);
    fill(0, nx - 1, ny - 1, ny - 1, k_w);
  }
  vl::CellKind bk;
  bk.tag = vl::KIND_WALL;
  bk.vgroup = 2;
  bk.fgroup = 0;
  if (sp->has_kick) { bk.velocity.kind = vl::VEL_ROTATION; bk.velocity.p[0] = sp->kick_cx; bk.velocity.p[1] = sp->kick_cy; }
  bk.shape = std::move(body);
  const uint8_t k_b = add(std::move(bk));
  {
    const vl::Shape& shape = *spec.kinds[k_b].shape;
    for (size_t y = 0; y < ny; ++y)
      for (size_t x = 0; x < nx; ++x)
        if (shape.inside((double)x, (double)y)) spec.paint[y * nx + x] = k_b;
  }
  std::string err;
  if (!vl::compile_domain(spec, out.dom, err)) return fail(VL_EINVAL, err);
  out.u_ref = sp->u;
  out.init_profile = sp->ramp_steps == 0;
  out.profile = profile;
  uint64_t len = sp->ramp_steps;
  if (sp->has_kick) len = std::max<uint64_t>(len, sp->kick_start + sp->kick_duration);
  out.sched_len = len;
  out.sched.assign(2 * std::max<uint64_t>(len, 1), 0.0);
  for (uint64_t t = 0; t < len; ++t) {
    out.sched[2 * t] = vl_ramp(t, sp->ramp_steps);
    double v2 = 0.0;
    if (sp->has_kick && t >= sp->kick_start && t < sp->kick_start + sp->kick_duration) {
      const double s = (double)(t - sp->kick_start) / (double)sp->kick_duration;
      const double a = std::sin(M_PI * s);
      v2 = sp->kick_omega * (a * a) * std::copysign(1.0, std::sin(2.0 * M_PI * s));
    }
    out.sched[2 * t + 1] = v2;
  }
  return VL_OK;
}

// The inflow profile as (rho, ux, uy) arrays for a start from the developed inflow
// (src/cases/channel.rs:108-110).
void vl::profile_field(const ChannelPlan& plan, std::vector<double>& rho, std::vector<double>& ux,
                       std::vector<double>& uy) {
  const size_t nx = plan.dom.nx, ny = plan.dom.ny;
  rho.assign(nx * ny, 1.0);
  ux.assign(nx * ny, 0.0);
  uy.assign(nx * ny, 0.0);
  for (size_t y = 0; y < ny; ++y) {
    double u, v;
    plan.profile.at(0.0, (double)y, u, v);
    for (size_t x = 0; x < nx; ++x) ux[y * nx + x] = u;
  }
}

extern "C" {

vl_channel* vl_channel_new(const vl_channel_spec* sp, int precision) {
  if (!sp) { fail(VL_EINVAL, "null spec"); return nullptr; }
  std::unique_ptr<vl::Shape> body;
  if (sp->body) { body = std::move(sp->body->s); delete sp->body; }
  vl::ChannelPlan plan;
  if (vl::plan_channel(sp, std::move(body), plan) != VL_OK) return nullptr;
  const vl::ChannelPlan& pl = plan;
  std::vector<double> rho, ux, uy;
  if (pl.init_profile) vl::profile_field(pl, rho, ux, uy);
  const std::vector<double> sched = pl.sched;
  const uint64_t len = pl.sched_len;
  vl_sim* sim = make_sim(std::move(plan.dom), precision);
  if (!sim) return nullptr;
  auto ch = std::make_unique<vl_channel>();
  ch->sim = sim;
  ch->u_ref = sp->u;
  ch->ramp_steps = sp->ramp_steps;
  if (!rho.empty() && vl_sim_init(sim, rho.data(), ux.data(), uy.data(), 1.0, 0.0, 0.0) != VL_OK) return nullptr;
  if (cudaMalloc(&sim->d_sched, sched.size() * sizeof(double)) != cudaSuccess ||
      cudaMemcpy(sim->d_sched, sched.data(), sched.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    fail(VL_ECUDA, "schedule upload");
    return nullptr;
  }
  if (sim->pull_ctl() != VL_OK) return nullptr;
  sim->hctl.sched_on = 1;
  sim->hctl.sched = sim->d_sched;
  sim->hctl.sched_len = len;
  sim->hctl.u_ref = sp->u;
  sim->hctl.absorbing = 1;
  if (sim->push_ctl() != VL_OK) return nullptr;
  return ch.release();
}

void vl_channel_free(vl_channel* c) { delete c; }
vl_sim* vl_channel_sim(vl_channel* c) { return c ? c->sim : nullptr; }
double vl_channel_u_ref(const vl_channel* c) { return c ? c->u_ref : std::nan(""); }

int vl_channel_set_absorbing(vl_channel* c, int on) {
  if (!c) return fail(VL_EINVAL, "null channel");
  int rc = c->sim->pull_ctl();
  if (rc) return rc;
  c->sim->hctl.absorbing = on ? 1 : 0;
  return c->sim->push_ctl();
}

int vl_channel_step(vl_channel* c, uint64_t steps) {
  if (!c) return fail(VL_EINVAL, "null channel");
  return c->sim->step(steps);
}

int vl_channel_coefficients(vl_channel* c, double d, double* cd, double* cl) {
  if (!c || !cd || !cl) return fail(VL_EINVAL, "null argument");
  double f[2 * VL_MAX_FGROUPS] = {0};
  int rc = vl_sim_force(c->sim, f);
  if (rc) return rc;
  const double k = 2.0 / (c->u_ref * c->u_ref * d);
  *cd = k * f[0];
  *cl = k * f[1];
  return VL_OK;
}

// ---------------------------------------------------------------- signal / small helpers
int vl_fft(double* re, double* im, size_t n) {
  if (!re || !im || n == 0 || (n & (n - 1))) return fail(VL_EINVAL, "FFT length must be a power of two");
  vl::fft_inplace(re, im, n);
  return VL_OK;
}
double vl_mean(const double* x, size_t n) { return vl::series_mean(x, n); }
double vl_rms(const double* x, size_t n) { return vl::series_rms(x, n); }
int vl_dominant_frequency(const double* x, size_t n, double dt, double* freq, double* amp) {
  if (!x || n < 2 || !freq || !amp) return fail(VL_EINVAL, "dominant_frequency: bad arguments");
  vl::dominant_frequency(x, n, dt, *freq, *amp);
  return VL_OK;
}
size_t vl_peaks(const double* x, size_t n, double* pos, double* val, size_t cap) {
  return x ? vl::find_peaks(x, n, pos, val, cap) : 0;
}
int vl_crossing_frequency(const double* x, size_t n, double dt, double* out) {
  if (!x || !out) return fail(VL_EINVAL, "null argument");
  return vl::crossing_frequency(x, n, dt, *out) ? 1 : 0;
}
double vl_sample_at(const double* x, size_t n, double pos) { return (x && n >= 2) ? vl::sample_at(x, n, pos) : std::nan(""); }
double vl_ramp(uint64_t t, uint64_t steps) {
  if (steps == 0 || t >= steps) return 1.0;
  const double s = (double)t / (double)steps;
  return s * s * (3.0 - 2.0 * s);
}
double vl_tau_for(double nu) { return nu / (1.0 / 3.0) + 0.5; }

}  // extern "C"
