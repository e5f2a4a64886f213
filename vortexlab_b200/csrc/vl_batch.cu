// Batched tunnels (C ABI vl_batch_*): many channels of uneven sizes, shapes and Reynolds numbers
// advanced together on one device, each for its own number of steps.
//
// Global step s advances every tunnel that still has steps to run. Between the steps at which some
// tunnel finishes, the set of active tunnels is fixed: that stretch ("segment") uses one tile list
// and one link-chunk list and is replayed from a captured CUDA graph of 32 steps. Each step is the
// batched link kernel and the batched bulk kernel, scheduled as for a single sim (concurrent on a
// forked stream, either order on one stream, or the staged pair).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/vortexlab.h"
#include "vl_batch.cuh"
#include "vl_internal.hpp"
#include "vl_launch.hpp"

namespace {

int fail(int code, const std::string& m) { return vl::set_error(code, m.c_str()); }

bool precision_is_f64(int prec) { return prec == VL_F64; }

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? VL_ENOMEM : VL_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VB_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

constexpr int kGraphSteps = 32;

// A tunnel's new end, set on the stream behind the steps already enqueued (the value travels as
// a launch argument, so the host does not wait for those steps as a pageable copy would).
__global__ void k_set_steps(vl::BatchTunnel* tun, int k, unsigned long long steps) { tun[k].steps = steps; }

template <class T>
int upload(T** dst, const std::vector<T>& v) {
  const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
  VB_CUDA(cudaMalloc((void**)dst, bytes));
  if (!v.empty()) VB_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return VL_OK;
}

}  // namespace

struct vl_batch {
  int device = 0;
  int prec = VL_F32;
  bool pairs_ok = false;   // narrow storage and every tunnel's row length even
  const vl::Launchers* L = nullptr;
  std::vector<vl::ChannelPlan> plans;
  std::vector<uint64_t> steps;
  bool built = false;
  std::vector<vl::BatchTunnel> tun;
  // Global step at which each tunnel takes its step 0 (kHeld: not started yet). A tunnel is active
  // at global step s while start <= s < start + its steps; the device counts in tunnel steps.
  static constexpr uint64_t kHeld = ~0ull;
  std::vector<uint64_t> start;
  std::vector<int4> chunks_all;          // every chunk, tunnel-major
  std::vector<int> chunk_first;          // first chunk of each tunnel in chunks_all
  void* buf[2] = {nullptr, nullptr};
  uint8_t* d_flag = nullptr;
  int32_t* d_bidx = nullptr;
  int32_t* d_bfirst = nullptr;
  vl::LinkRecDev* d_links = nullptr;
  int32_t* d_pidx = nullptr;
  int8_t* d_pn = nullptr;
  double* d_sched = nullptr;
  vl::BatchTunnel* d_tun = nullptr;
  vl::BatchState* d_st = nullptr;
  int4* d_tiles = nullptr;
  size_t tiles_cap = 0;
  int4* d_chunks = nullptr;
  int* d_outl = nullptr;                 // active tunnels with an absorbing outlet
  double* d_partials = nullptr;
  double* d_hist = nullptr;
  int2* d_bdesc = nullptr;               // staged step: per boundary node {first link, direction mask}
  int32_t* d_segb = nullptr;             // staged step: boundary nodes before each 32-cell row segment
  void* d_lb = nullptr;                  // staged step: returning population per link
  void* d_ownc = nullptr;                // staged step: boundary nodes' own populations
  bool own_ok = false;                   // d_ownc holds the active tunnels' current boundary nodes
  cudaStream_t stream = nullptr, aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev0 = nullptr, ev1 = nullptr;
  vl::BatchParams P{};
  int ntiles = 0, nchunks = 0;
  int schedule = 0;
  int log2_tx = 8, ty = 1;
  uint64_t s = 0;
  uint64_t launches = 0;
  cudaGraphExec_t gexec = nullptr;
  std::vector<int4> tiles_h, chunks_h;   // host copies of the current work lists
  std::vector<int> outl_h;
  std::vector<char> listed;              // which tunnels the current work lists hold
  int listed_tx = -1, listed_ty = -1, listed_pairs = -1;
  bool timed = false;
  bool in_flight = false;                // a run was enqueued and not yet waited for
  uint64_t s_done = 0;                   // global steps complete on the device at the last wait
  cudaStream_t copy = nullptr;           // history reads beside a run in flight
  std::vector<cudaGraphExec_t> retired;  // graphs replaced while a run may still execute them
  double* h_stage = nullptr;             // pinned staging of those reads
  size_t h_stage_cap = 0;                // doubles

  ~vl_batch() {
    cudaSetDevice(device);
    if (gexec) cudaGraphExecDestroy(gexec);
    for (cudaGraphExec_t g : retired) cudaGraphExecDestroy(g);
    void* ptrs[] = {buf[0], buf[1], d_flag, d_bidx, d_bfirst, d_links, d_pidx, d_pn, d_sched,
                    d_tun, d_st, d_tiles, d_chunks, d_outl, d_partials, d_hist, d_bdesc, d_segb, d_lb, d_ownc};
    for (void* p : ptrs)
      if (p) cudaFree(p);
    cudaEvent_t evs[] = {ev_fork, ev_join, ev0, ev1};
    for (cudaEvent_t e : evs)
      if (e) cudaEventDestroy(e);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
    if (copy) cudaStreamDestroy(copy);
    if (h_stage) cudaFreeHost(h_stage);
  }

  const void* a() const { return buf[s & 1]; }
  void* b() const { return buf[(s & 1) ^ 1]; }
  void* tunnel_ptr(void* base, int k) const { return (char*)base + tun[k].pop_off * L->elem; }
  // The buffer that holds tunnel k's state after t of its own steps (its step 0 took the global
  // step start; a held tunnel's start state is in both buffers).
  int parity(size_t k, uint64_t t) const { return (int)(((start[k] == kHeld ? 0 : start[k]) + t) & 1); }
  // Global step after the last step of tunnel k (0 while it is held).
  uint64_t end_of(size_t k) const { return start[k] == kHeld ? 0 : start[k] + tun[k].steps; }
  // Steps tunnel k has done (or has enqueued) by global step g.
  uint64_t done_by(size_t k, uint64_t g) const {
    return start[k] == kHeld || g <= start[k] ? 0 : std::min<uint64_t>(g - start[k], tun[k].steps);
  }

  // Drops the captured graph (its steps no longer fit the work lists or the tunnels' ends). A run
  // in flight may still be executing it, and destroying it then waits for that run, so it is
  // destroyed at the next wait instead.
  void drop_graph() {
    if (!gexec) return;
    if (in_flight)
      retired.push_back(gexec);
    else
      cudaGraphExecDestroy(gexec);
    gexec = nullptr;
  }

  // Work lists of the tunnels active at global step s (the ones with steps left).
  int build_lists(bool all) {
    tiles_h.clear();
    chunks_h.clear();
    outl_h.clear();
    const int tx = (1 << log2_tx) << (P.pairs ? 1 : 0);   // cells per tile row
    const int seg = 32 << (P.pairs ? 1 : 0);               // packed layout: cells per warp segment
    const int wpb = vl::kBlock / 32;                       // warp segments per packed tile
    for (size_t k = 0; k < tun.size(); ++k) {
      if (!all && s >= end_of(k)) continue;
      const vl::BatchTunnel& T = tun[k];
      if (ty == 0) {
        const int total = T.ny * ((T.nx + seg - 1) / seg);
        for (int g0 = 0; g0 < total; g0 += wpb) tiles_h.push_back(make_int4((int)k, g0, 0, 0));
      } else {
        for (int y0 = 0; y0 < T.ny; y0 += ty)
          for (int x0 = 0; x0 < T.nx; x0 += tx) tiles_h.push_back(make_int4((int)k, y0, x0, 0));
      }
      for (int c = 0; c < T.nchunks; ++c) chunks_h.push_back(chunks_all[chunk_first[k] + c]);
      if (T.absorbing && T.np > 0 && T.nchunks > 0) outl_h.push_back((int)k);
    }
    if (tiles_h.size() > tiles_cap) {
      if (d_tiles) cudaFree(d_tiles);
      d_tiles = nullptr;
      tiles_cap = tiles_h.size();
      VB_CUDA(cudaMalloc(&d_tiles, tiles_cap * sizeof(int4)));
    }
    VB_CUDA(cudaMemcpyAsync(d_tiles, tiles_h.data(), tiles_h.size() * sizeof(int4), cudaMemcpyHostToDevice, stream));
    // Pageable host to device: the host vectors are staged before the calls return, and the
    // copies are ordered after any run still in flight on the stream, which reads the old lists.
    VB_CUDA(cudaMemcpyAsync(d_chunks, chunks_h.data(), chunks_h.size() * sizeof(int4), cudaMemcpyHostToDevice, stream));
    if (!outl_h.empty())
      VB_CUDA(cudaMemcpyAsync(d_outl, outl_h.data(), outl_h.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    listed.assign(tun.size(), 0);
    for (size_t k = 0; k < tun.size(); ++k) listed[k] = all || s < end_of(k);
    listed_tx = log2_tx;
    listed_ty = ty;
    listed_pairs = P.pairs;
    ntiles = (int)tiles_h.size();
    nchunks = (int)chunks_h.size();
    P.ntiles = ntiles;
    P.tiles = d_tiles;
    P.chunks = d_chunks;
    P.outl = d_outl;
    P.noutl = (int)outl_h.size();
    P.log2_tx = log2_tx;
    P.ty = ty;
    P.packed = ty == 0;
    drop_graph();
    return VL_OK;
  }

  // Kernels a step launches: bulk and links, and the outlet offsets where a tunnel has an outlet.
  int per_step() const { return (ntiles > 0) + (nchunks > 0) + (nchunks > 0 && P.noutl > 0); }

  // Whether the work lists already hold exactly the tunnels active at step s.
  bool lists_current() const {
    if (listed.size() != tun.size() || listed_tx != log2_tx || listed_ty != ty || listed_pairs != P.pairs) return false;
    for (size_t k = 0; k < tun.size(); ++k)
      if ((bool)listed[k] != (s < end_of(k))) return false;
    return true;
  }

  // The staged step reads the boundary nodes' own populations from d_ownc; after anything other
  // than a staged step set the state they are gathered from `a` for the active tunnels.
  int prepare_steps() {
    if (schedule != 3 || own_ok) return VL_OK;
    cudaError_t e = L->batch_gather_own(P, nchunks, a(), stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch gather own populations");
    launches += 1;
    own_ok = true;
    return VL_OK;
  }

  cudaError_t enqueue_step() {
    cudaError_t e;
    if (schedule == 3) {
      if ((e = L->batch_step(P, ntiles, nchunks, 1 | 4, a(), b(), stream)) != cudaSuccess) return e;
      return L->batch_step(P, ntiles, nchunks, 2 | 4, a(), b(), stream);
    }
    cudaStream_t ls = schedule == 0 ? aux : stream;
    if (schedule == 0) {
      if ((e = cudaEventRecord(ev_fork, stream)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(aux, ev_fork, 0)) != cudaSuccess) return e;
    }
    if (schedule == 2) {
      if ((e = L->batch_step(P, ntiles, nchunks, 2, a(), b(), stream)) != cudaSuccess) return e;
      return L->batch_step(P, ntiles, nchunks, 1, a(), b(), stream);
    }
    if ((e = L->batch_step(P, ntiles, nchunks, 1, a(), b(), ls)) != cudaSuccess) return e;
    if (schedule == 0 && (e = cudaEventRecord(ev_join, aux)) != cudaSuccess) return e;
    if ((e = L->batch_step(P, ntiles, nchunks, 2, a(), b(), stream)) != cudaSuccess) return e;
    if (schedule == 0) return cudaStreamWaitEvent(stream, ev_join, 0);
    return cudaSuccess;
  }

  int ensure_graph() {
    if (gexec) return VL_OK;
    cudaGraph_t g = nullptr;
    const uint64_t saved = s;
    VB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kGraphSteps; ++k) {
      cudaError_t e = enqueue_step();
      ++s;
      if (e != cudaSuccess) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        s = saved;
        return cuda_fail(e, "batch graph capture");
      }
    }
    s = saved;
    VB_CUDA(cudaStreamEndCapture(stream, &g));
    cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
    return VL_OK;
  }

  // Enqueues the steps of a run on the stream without waiting for them.
  int enqueue_run(uint64_t max_steps) {
    VB_CUDA(cudaSetDevice(device));
    uint64_t end_all = 0;
    for (size_t k = 0; k < tun.size(); ++k) end_all = std::max<uint64_t>(end_all, end_of(k));
    const uint64_t stop = max_steps ? std::min<uint64_t>(end_all, s + max_steps) : end_all;
    VB_CUDA(cudaEventRecord(ev0, stream));
    in_flight = true;   // from here on a graph launched below may be executing
    while (s < stop) {
      uint64_t seg_end = stop;
      for (size_t k = 0; k < tun.size(); ++k)
        if (end_of(k) > s) seg_end = std::min<uint64_t>(seg_end, end_of(k));
      int rc = lists_current() ? VL_OK : build_lists(false);
      if (rc) return rc;
      if ((rc = prepare_steps())) return rc;
      while (s < seg_end) {
        if (seg_end - s >= (uint64_t)kGraphSteps && (s & 1) == 0) {
          rc = ensure_graph();
          if (rc) return rc;
          VB_CUDA(cudaGraphLaunch(gexec, stream));
          s += kGraphSteps;
          launches += (uint64_t)per_step() * kGraphSteps;
        } else {
          cudaError_t e = enqueue_step();
          if (e != cudaSuccess) return cuda_fail(e, "batch step");
          ++s;
          launches += per_step();
        }
      }
      own_ok = schedule == 3;
    }
    VB_CUDA(cudaEventRecord(ev1, stream));
    in_flight = true;
    timed = false;
    return VL_OK;
  }

  int wait() {
    VB_CUDA(cudaSetDevice(device));
    VB_CUDA(cudaStreamSynchronize(stream));
    if (in_flight) timed = true;
    in_flight = false;
    s_done = s;
    for (cudaGraphExec_t g : retired) cudaGraphExecDestroy(g);
    retired.clear();
    return VL_OK;
  }

  int run(uint64_t max_steps) {
    int rc = enqueue_run(max_steps);
    return rc ? rc : wait();
  }

  // Times the candidate tile shapes on the current state without advancing it and keeps the
  // fastest. Shapes: 256 x 1, 128 x 2, 64 x 4, 32 x 8 cells.
  // Layouts: rows of 256 x 1, 128 x 2, 64 x 4, 32 x 8 cells (times the cells per thread), and the
  // packed layout (log2_tx 5, ty 0). ms (may be NULL) receives up to n of the five times.
  int autotune(int steps_each, double* ms, int n) {
    VB_CUDA(cudaSetDevice(device));
    const int shapes[5][2] = {{8, 1}, {7, 2}, {6, 4}, {5, 8}, {5, 0}};
    double best = 1e300;
    int bi = 0;
    P.dry = 1;
    for (int c = 0; c < 5; ++c) {
      log2_tx = shapes[c][0];
      ty = shapes[c][1];
      int rc = build_lists(false);
      if (rc) { P.dry = 0; return rc; }
      if ((rc = prepare_steps())) { P.dry = 0; return rc; }
      for (int k = 0; k < steps_each + 2; ++k) {
        if (k == 2) VB_CUDA(cudaEventRecord(ev0, stream));
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) { P.dry = 0; return cuda_fail(e, "batch autotune"); }
      }
      VB_CUDA(cudaEventRecord(ev1, stream));
      VB_CUDA(cudaEventSynchronize(ev1));
      float t = 0.f;
      VB_CUDA(cudaEventElapsedTime(&t, ev0, ev1));
      if (ms && c < n) ms[c] = t / steps_each;
      if (t < best) { best = t; bi = c; }
    }
    P.dry = 0;
    own_ok = false;  // the dry staged steps left the copy of `b`, not of `a`
    log2_tx = shapes[bi][0];
    ty = shapes[bi][1];
    timed = false;
    return build_lists(false);
  }
};

extern "C" {

vl_batch* vl_batch_new(int precision) {
  const vl::Launchers* L = nullptr;
  switch (precision) {
    case VL_F64: L = &vl::launchers_f64(); break;
    case VL_F32: L = &vl::launchers_f32(); break;
    case VL_F16S: L = &vl::launchers_f16s(); break;
    case VL_F16C: L = &vl::launchers_f16c(); break;
    case VL_F16X: L = &vl::launchers_f16x(); break;
    default: fail(VL_EINVAL, "unknown precision"); return nullptr;
  }
  auto b = new vl_batch();
  b->prec = precision;
  b->L = L;
  return b;
}

void vl_batch_free(vl_batch* b) { delete b; }

int vl_batch_add_channel(vl_batch* b, const vl_channel_spec* sp, uint64_t steps) {
  std::unique_ptr<vl::Shape> body;
  if (sp && sp->body) { body = std::move(sp->body->s); delete sp->body; }
  if (!b || !sp) return fail(VL_EINVAL, "null batch or spec");
  if (b->built) return fail(VL_EINVAL, "batch already built");
  if (steps == 0) return fail(VL_EINVAL, "a tunnel needs at least one step");
  vl::ChannelPlan plan;
  int rc = vl::plan_channel(sp, std::move(body), plan);
  if (rc) return rc;
  if (plan.dom.ngroups != 1) return fail(VL_EINVAL, "batched tunnels need a body with force group 0");
  b->plans.push_back(std::move(plan));
  b->steps.push_back(steps);
  return (int)b->plans.size() - 1;
}

int vl_batch_build(vl_batch* b) {
  if (!b) return fail(VL_EINVAL, "null batch");
  if (b->built) return fail(VL_EINVAL, "batch already built");
  if (b->plans.empty()) return fail(VL_EINVAL, "empty batch");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(VL_ECUDA, "no CUDA device: vortexlab-b200 has no CPU fallback");
  }
  VB_CUDA(cudaGetDevice(&b->device));
  const size_t nt = b->plans.size();
  std::vector<uint8_t> flag;
  std::vector<int32_t> bidx, bfirst, pidx;
  std::vector<int8_t> pn;
  std::vector<vl::LinkRecDev> links;
  std::vector<double> sched;
  std::vector<int2> bdesc;
  std::vector<int32_t> segb;
  unsigned long long pop = 0, cells = 0, hist = 0;
  int nchunk = 0;
  b->tun.resize(nt);
  b->chunk_first.resize(nt);
  for (size_t k = 0; k < nt; ++k) {
    const vl::ChannelPlan& pl = b->plans[k];
    const vl::CompiledDomain& d = pl.dom;
    vl::BatchTunnel& T = b->tun[k];
    std::memset(&T, 0, sizeof T);
    T.nx = (int)d.nx;
    T.ny = (int)d.ny;
    T.ns = (unsigned)((d.n + 63) / 64 * 64);
    if ((unsigned long long)T.ns * 9ull > 0xFFFFFFFFull) return fail(VL_EINVAL, "tunnel too large");
    T.coll = d.collision;
    T.pop_off = pop;
    pop += 9ull * T.ns;
    T.cell_off = cells;
    cells += d.n;
    T.b_off = (int)bidx.size();
    T.nb = (int)d.bnode_idx.size();
    T.p_off = (int)pidx.size();
    T.np = (int)d.pnode_idx.size();
    T.nchunks = (T.nb + vl::kBlock - 1) / vl::kBlock;
    T.chunk_off = nchunk;
    T.op = d.op;
    T.om = d.om;
    T.u_ref = pl.u_ref;
    T.absorbing = 1;
    T.sched_off = sched.size();
    T.sched_len = pl.sched_len;
    T.steps = b->steps[k];
    T.hist_off = hist;
    hist += T.steps;
    flag.insert(flag.end(), d.flag.begin(), d.flag.end());
    const int32_t loff = (int32_t)links.size();
    for (int32_t v : d.bnode_idx) bidx.push_back(v);
    for (size_t j = 0; j + 1 < d.bnode_first.size(); ++j) bfirst.push_back(d.bnode_first[j] + loff);
    // Staged-step tables: node descriptors (links by ascending direction) and, per 32-cell row
    // segment, the global rank of the first boundary node at or after the segment's first cell.
    for (size_t j = 0; j + 1 < d.bnode_first.size(); ++j) {
      int mask = 0, prev = 0;
      for (int l = d.bnode_first[j]; l < d.bnode_first[j + 1]; ++l) {
        const int dir = d.links[(size_t)l].dir;
        if (dir <= prev || dir > 8) return fail(VL_EINVAL, "staged step: links of a node must have ascending directions");
        prev = dir;
        mask |= 1 << dir;
      }
      bdesc.push_back(int2{d.bnode_first[j] + loff, mask});
    }
    T.segs = (T.nx + 31) / 32;
    T.seg_off = (int)segb.size();
    {
      size_t kb = 0;
      for (size_t y = 0; y < d.ny; ++y)
        for (int sg = 0; sg < T.segs; ++sg) {
          const size_t start = y * d.nx + (size_t)sg * 32;
          while (kb < d.bnode_idx.size() && (size_t)d.bnode_idx[kb] < start) ++kb;
          segb.push_back(T.b_off + (int32_t)kb);
        }
    }
    for (const vl::LinkRec& h : d.links) {
      vl::LinkRecDev g;
      g.q = h.q; g.cu6 = h.cu6; g.uw0 = h.uw[0]; g.uw1 = h.uw[1]; g.rho = h.rho;
      g.behind = h.behind; g.dir = h.dir; g.flags = h.flags; g.vgroup = h.vgroup; g.fgroup = h.fgroup;
      links.push_back(g);
    }
    for (size_t j = 0; j < d.pnode_idx.size(); ++j) {
      pidx.push_back(d.pnode_idx[j]);
      pn.push_back(d.pnode_nx[j]);
      pn.push_back(d.pnode_ny[j]);
    }
    sched.insert(sched.end(), pl.sched.begin(), pl.sched.begin() + 2 * pl.sched_len);
    b->chunk_first[k] = (int)b->chunks_all.size();
    for (int c = 0; c < T.nchunks; ++c)
      b->chunks_all.push_back(make_int4((int)k, T.b_off + c * vl::kBlock, std::min(vl::kBlock, T.nb - c * vl::kBlock), nchunk + c));
    nchunk += T.nchunks;
  }
  bfirst.push_back((int32_t)links.size());
  if (links.size() > 0x7fffffffu || cells > 0xFFFFFFFFull || segb.size() > 0x7fffffffu)
    return fail(VL_EINVAL, "batch too large");
  const size_t pop_bytes = pop * b->L->elem;
  VB_CUDA(cudaMalloc(&b->buf[0], pop_bytes));
  VB_CUDA(cudaMalloc(&b->buf[1], pop_bytes));
  int rc;
  if ((rc = upload(&b->d_flag, flag)) || (rc = upload(&b->d_bidx, bidx)) || (rc = upload(&b->d_bfirst, bfirst)) ||
      (rc = upload(&b->d_links, links)) || (rc = upload(&b->d_pidx, pidx)) || (rc = upload(&b->d_pn, pn)) ||
      (rc = upload(&b->d_sched, sched)) || (rc = upload(&b->d_tun, b->tun)))
    return rc;
  std::vector<vl::BatchState> st(nt);
  std::memset(st.data(), 0, st.size() * sizeof(vl::BatchState));
  if ((rc = upload(&b->d_st, st))) return rc;
  if ((rc = upload(&b->d_bdesc, bdesc)) || (rc = upload(&b->d_segb, segb))) return rc;
  const size_t r_elem = precision_is_f64(b->prec) ? sizeof(double) : sizeof(float);
  const unsigned nbs = (unsigned)((bidx.size() + 63) / 64 * 64);
  VB_CUDA(cudaMalloc(&b->d_lb, std::max<size_t>(links.size() * r_elem, 16)));
  VB_CUDA(cudaMalloc(&b->d_ownc, std::max<size_t>((size_t)nbs * 9 * b->L->elem, 16)));
  VB_CUDA(cudaMalloc(&b->d_chunks, std::max<size_t>(b->chunks_all.size(), 1) * sizeof(int4)));
  VB_CUDA(cudaMalloc(&b->d_outl, std::max<size_t>(nt, 1) * sizeof(int)));
  VB_CUDA(cudaMalloc(&b->d_partials, std::max(nchunk, 1) * 2 * sizeof(double)));
  VB_CUDA(cudaMalloc(&b->d_hist, std::max<unsigned long long>(hist, 1) * 2 * sizeof(double)));
  VB_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
#ifdef VL_BATCH_AUX_PRIORITY
  {
    int lo = 0, hi = 0;
    VB_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    VB_CUDA(cudaStreamCreateWithPriority(&b->aux, cudaStreamNonBlocking, hi));
  }
#else
  VB_CUDA(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
#endif
  VB_CUDA(cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking));
  VB_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  VB_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
  VB_CUDA(cudaEventCreate(&b->ev0));
  VB_CUDA(cudaEventCreate(&b->ev1));
  // Start states: uniform rest, or the inflow profile when the tunnel has no ramp
  // (src/cases/channel.rs:108-110), into both buffers.
  for (size_t k = 0; k < nt; ++k) {
    const vl::ChannelPlan& pl = b->plans[k];
    const vl::BatchTunnel& T = b->tun[k];
    double* field = nullptr;
    if (pl.init_profile) {
      std::vector<double> rho, ux, uy;
      vl::profile_field(pl, rho, ux, uy);
      const size_t n = pl.dom.n;
      VB_CUDA(cudaMalloc(&field, 3 * n * sizeof(double)));
      VB_CUDA(cudaMemcpy(field, rho.data(), n * 8, cudaMemcpyHostToDevice));
      VB_CUDA(cudaMemcpy(field + n, ux.data(), n * 8, cudaMemcpyHostToDevice));
      VB_CUDA(cudaMemcpy(field + 2 * n, uy.data(), n * 8, cudaMemcpyHostToDevice));
    }
    const size_t n = pl.dom.n;
    cudaError_t e = b->L->init((int)n, T.ns, b->d_flag + T.cell_off, field, field ? field + n : nullptr,
                               field ? field + 2 * n : nullptr, 1.0, 0.0, 0.0, b->tunnel_ptr(b->buf[0], (int)k),
                               b->tunnel_ptr(b->buf[1], (int)k), b->stream);
    if (field) {
      cudaStreamSynchronize(b->stream);
      cudaFree(field);
    }
    if (e != cudaSuccess) return cuda_fail(e, "batch init");
  }
  VB_CUDA(cudaStreamSynchronize(b->stream));
  vl::BatchParams& P = b->P;
  P.tun = b->d_tun;
  P.st = b->d_st;
  P.flag = b->d_flag;
  P.bnode_idx = b->d_bidx;
  P.bnode_first = b->d_bfirst;
  P.links = b->d_links;
  P.pnode_idx = b->d_pidx;
  P.pnode_n = b->d_pn;
  P.sched = b->d_sched;
  P.partials = b->d_partials;
  P.hist = b->d_hist;
  P.sqrt_cs2 = std::sqrt(1.0 / 3.0);
  P.dry = 0;
  P.bdesc = b->d_bdesc;
  P.seg_bfirst = b->d_segb;
  P.lb = b->d_lb;
  P.ownc = b->d_ownc;
  P.nbs = nbs;
  P.pairs = 0;
  if (!precision_is_f64(b->prec)) {
    bool even = true;
    for (const auto& T : b->tun) even = even && T.nx % 2 == 0 && T.ns % 2 == 0;
    P.pairs = even ? 1 : 0;
  }
  b->pairs_ok = P.pairs != 0;
  // narrow formats: each bulk block prefetches into the L2 the tile three waves of blocks ahead
  P.prefetch_tiles = 0;
  if (!precision_is_f64(b->prec)) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    P.prefetch_tiles = 3 * sms;
  }
  b->start.assign(nt, 0);
  b->built = true;
  // The host plans (domains) are no longer needed on the host except their sizes.
  for (auto& pl : b->plans) {
    pl.dom.links.clear();
    pl.dom.links.shrink_to_fit();
  }
  return b->build_lists(false);
}

int vl_batch_size(const vl_batch* b) { return b ? (int)b->plans.size() : VL_EINVAL; }

int vl_batch_tunnel_info(const vl_batch* b, int k, size_t* nx, size_t* ny, size_t* fluid, uint64_t* steps) {
  if (!b || k < 0 || (size_t)k >= b->plans.size()) return fail(VL_EINVAL, "tunnel index out of range");
  if (nx) *nx = b->plans[k].dom.nx;
  if (ny) *ny = b->plans[k].dom.ny;
  if (fluid) *fluid = b->plans[k].dom.fluid_nodes;
  if (steps) *steps = b->built ? b->tun[k].steps : b->steps[k];
  return VL_OK;
}

int vl_batch_set_tile(vl_batch* b, int log2_tx, int ty) {
  if (!b || !b->built) return fail(VL_EINVAL, "batch not built");
  const bool packed = log2_tx == 5 && ty == 0;
  if (!packed && (log2_tx < 5 || log2_tx > 8 || ty < 1 || (ty << log2_tx) != vl::kBlock))
    return fail(VL_EINVAL, "tile must be 2^log2_tx x ty = 256 cells with 32 <= 2^log2_tx <= 256, or (5, 0) packed");
  b->log2_tx = log2_tx;
  b->ty = ty;
  return b->build_lists(false);
}

int vl_batch_set_cells_per_thread(vl_batch* b, int cells) {
  if (!b || !b->built) return fail(VL_EINVAL, "batch not built");
  if (cells != 1 && cells != 2) return fail(VL_EINVAL, "cells per thread must be 1 or 2");
  const int want = cells == 2 && b->pairs_ok ? 1 : 0;
  if (want == b->P.pairs) return VL_OK;
  b->P.pairs = want;
  return b->build_lists(false);
}

int vl_batch_set_prefetch_tiles(vl_batch* b, int tiles) {
  if (!b || !b->built || tiles < 0) return fail(VL_EINVAL, "bad arguments");
  if (tiles == b->P.prefetch_tiles) return VL_OK;
  b->P.prefetch_tiles = tiles;
  b->drop_graph();
  return VL_OK;
}

int vl_batch_get_tile(const vl_batch* b, int* log2_tx, int* ty) {
  if (!b) return fail(VL_EINVAL, "null batch");
  if (log2_tx) *log2_tx = b->log2_tx;
  if (ty) *ty = b->ty;
  return VL_OK;
}

int vl_batch_set_schedule(vl_batch* b, int schedule) {
  if (!b || schedule < 0 || schedule >= VL_SCHEDULE_COUNT) return fail(VL_EINVAL, "schedule must be 0, 1, 2 or 3");
  b->schedule = schedule;
  b->drop_graph();
  return VL_OK;
}

int vl_batch_autotune(vl_batch* b, int steps_each, double* ms4) {
  if (!b || !b->built || steps_each < 1) return fail(VL_EINVAL, "autotune: bad arguments");
  return b->autotune(steps_each, ms4, 4);
}

int vl_batch_autotune_layouts(vl_batch* b, int steps_each, double* ms, int n) {
  if (!b || !b->built || steps_each < 1 || n < 0) return fail(VL_EINVAL, "autotune: bad arguments");
  return b->autotune(steps_each, ms, n);
}

int vl_batch_run(vl_batch* b, uint64_t max_steps) {
  if (!b || !b->built) return fail(VL_EINVAL, "batch not built");
  return b->run(max_steps);
}

int vl_batch_run_async(vl_batch* b, uint64_t max_steps) {
  if (!b || !b->built) return fail(VL_EINVAL, "batch not built");
  return b->enqueue_run(max_steps);
}

int vl_batch_wait(vl_batch* b) {
  if (!b || !b->built) return fail(VL_EINVAL, "batch not built");
  return b->wait();
}

int vl_batch_history_copy(vl_batch* b, int n, const int* ks, const uint64_t* firsts, const uint64_t* counts,
                          double* out) {
  if (!b || !b->built || n < 0 || (n && (!ks || !firsts || !counts || !out))) return fail(VL_EINVAL, "bad arguments");
  for (int i = 0; i < n; ++i) {
    const int k = ks[i];
    if (k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "tunnel index out of range");
    if (firsts[i] > b->steps[k] || counts[i] > b->steps[k] - firsts[i])
      return fail(VL_EINVAL, "range past the tunnel's force history");
    if (firsts[i] + counts[i] > b->done_by(k, b->s_done))
      return fail(VL_EINVAL, "range past the steps complete at the last wait");
  }
  VB_CUDA(cudaSetDevice(b->device));
  size_t total = 0;
  for (int i = 0; i < n; ++i) total += 2 * counts[i];
  if (total > b->h_stage_cap) {
    if (b->h_stage) VB_CUDA(cudaFreeHost(b->h_stage));
    b->h_stage = nullptr;
    b->h_stage_cap = 0;
    const size_t cap = std::max<size_t>(total, 1 << 16);
    VB_CUDA(cudaHostAlloc(&b->h_stage, cap * sizeof(double), cudaHostAllocDefault));
    b->h_stage_cap = cap;
  }
  // one copy per range into pinned memory (asynchronous DMA beside the run), one wait
  size_t at = 0;
  for (int i = 0; i < n; ++i) {
    if (counts[i])
      VB_CUDA(cudaMemcpyAsync(b->h_stage + at, b->d_hist + 2 * (b->tun[ks[i]].hist_off + firsts[i]),
                              counts[i] * 2 * sizeof(double), cudaMemcpyDeviceToHost, b->copy));
    at += 2 * counts[i];
  }
  VB_CUDA(cudaStreamSynchronize(b->copy));
  if (total) std::memcpy(out, b->h_stage, total * sizeof(double));
  return VL_OK;
}

int vl_batch_last_run_ms(vl_batch* b, float* ms) {
  if (!b || !ms || !b->timed) return fail(VL_EINVAL, "no run timed yet");
  VB_CUDA(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  return VL_OK;
}

int vl_batch_global_step(const vl_batch* b, uint64_t* s) {
  if (!b || !s) return fail(VL_EINVAL, "null argument");
  *s = b->s;
  return VL_OK;
}

int vl_batch_launch_count(const vl_batch* b, uint64_t* out) {
  if (!b || !out) return fail(VL_EINVAL, "null argument");
  *out = b->launches;
  return VL_OK;
}

static int pull_state(vl_batch* b, int k, vl::BatchState* st) {
  VB_CUDA(cudaMemcpyAsync(st, b->d_st + k, sizeof *st, cudaMemcpyDeviceToHost, b->stream));
  return b->wait();
}

int vl_batch_status(vl_batch* b, int k, uint64_t* t, int* nonfinite, double* force2) {
  if (!b || !b->built || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "tunnel index out of range");
  vl::BatchState st;
  int rc = pull_state(b, k, &st);
  if (rc) return rc;
  if (t) *t = st.t;
  if (nonfinite) *nonfinite = st.nonfinite;
  if (force2) { force2[0] = st.force[0]; force2[1] = st.force[1]; }
  return VL_OK;
}

int vl_batch_force_history(vl_batch* b, int k, double* out, uint64_t* count) {
  if (!b || !b->built || !count || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "bad arguments");
  vl::BatchState st;
  int rc = pull_state(b, k, &st);
  if (rc) return rc;
  const uint64_t have = std::min<uint64_t>(st.t, b->tun[k].steps);
  if (out && have)
    VB_CUDA(cudaMemcpy(out, b->d_hist + 2 * b->tun[k].hist_off, have * 2 * sizeof(double), cudaMemcpyDeviceToHost));
  *count = have;
  return VL_OK;
}

int vl_batch_force_history_range(vl_batch* b, int k, uint64_t first, uint64_t max, double* out, uint64_t* count) {
  if (!b || !b->built || !count || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "bad arguments");
  vl::BatchState st;
  int rc = pull_state(b, k, &st);
  if (rc) return rc;
  const uint64_t have = std::min<uint64_t>(st.t, b->tun[k].steps);
  const uint64_t n = first >= have ? 0 : std::min<uint64_t>(have - first, max);
  if (out && n)
    VB_CUDA(cudaMemcpy(out, b->d_hist + 2 * (b->tun[k].hist_off + first), n * 2 * sizeof(double),
                       cudaMemcpyDeviceToHost));
  *count = n;
  return VL_OK;
}

int vl_batch_download(vl_batch* b, int k, double* out) {
  if (!b || !b->built || !out || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "bad arguments");
  vl::BatchState st;
  int rc = pull_state(b, k, &st);
  if (rc) return rc;
  const size_t n = b->plans[k].dom.n;
  const vl::BatchTunnel& T = b->tun[k];
  double* tmp = nullptr;
  VB_CUDA(cudaMalloc(&tmp, 9 * n * sizeof(double)));
  cudaError_t e = b->L->to_f64((int)n, T.ns, b->tunnel_ptr(b->buf[b->parity(k, st.t)], k), tmp, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, 9 * n * 8, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(e, "batch download");
  return VL_OK;
}

int vl_batch_hold(vl_batch* b, int k) {
  if (!b || !b->built || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "bad arguments");
  if (b->s != 0) return fail(VL_EINVAL, "a tunnel can only be held before the batch's first step");
  if (b->start[k] == vl_batch::kHeld) return VL_OK;
  b->start[k] = vl_batch::kHeld;
  b->drop_graph();
  return VL_OK;
}

int vl_batch_start(vl_batch* b, int k, uint64_t* start) {
  if (!b || !b->built || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "bad arguments");
  if (b->start[k] != vl_batch::kHeld) return fail(VL_EINVAL, "the tunnel is not held");
  b->start[k] = b->s;        // its step 0 follows the steps already enqueued
  b->own_ok = false;         // the staged step's copy of boundary populations lacks it
  b->drop_graph();
  if (start) *start = b->s;
  return VL_OK;
}

int vl_batch_set_steps(vl_batch* b, int k, uint64_t steps) {
  if (!b || !b->built || k < 0 || (size_t)k >= b->tun.size()) return fail(VL_EINVAL, "bad arguments");
  vl::BatchTunnel& T = b->tun[k];
  const uint64_t done = b->done_by(k, b->s);
  if (steps < done || (b->start[k] != vl_batch::kHeld && b->s > b->end_of(k)))
    return fail(VL_EINVAL, "the tunnel has already run past that step");
  if (steps > b->steps[k]) return fail(VL_EINVAL, "a tunnel cannot run longer than the steps it was added with");
  if (steps == T.steps) return VL_OK;
  T.steps = steps;
  // ordered after a run in flight, which still reads the old end
  VB_CUDA(cudaSetDevice(b->device));
  k_set_steps<<<1, 1, 0, b->stream>>>(b->d_tun, k, (unsigned long long)steps);
  VB_CUDA(cudaGetLastError());
  b->launches += 1;
  b->drop_graph();      // the captured steps may cover the new end: capture again
  return VL_OK;
}

int vl_batch_macros_field(vl_batch* b, int k, double* rho, double* ux, double* uy) {
  if (!b || !b->built || !rho || !ux || !uy || k < 0 || (size_t)k >= b->tun.size())
    return fail(VL_EINVAL, "bad arguments");
  vl::BatchState st;
  int rc = pull_state(b, k, &st);
  if (rc) return rc;
  const size_t n = b->plans[k].dom.n;
  const vl::BatchTunnel& T = b->tun[k];
  double* tmp = nullptr;
  VB_CUDA(cudaMalloc(&tmp, 3 * n * sizeof(double)));
  cudaError_t e = b->L->macros((int)n, T.ns, b->d_flag + T.cell_off, 0.0, 0.0, b->tunnel_ptr(b->buf[b->parity(k, st.t)], k), tmp,
                               tmp + n, tmp + 2 * n, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rho, tmp, n * 8, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ux, tmp + n, n * 8, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(uy, tmp + 2 * n, n * 8, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(e, "batch macros");
  return VL_OK;
}

int vl_batch_init(vl_batch* b, int k, const double* rho, const double* ux, const double* uy) {
  if (!b || !b->built || !rho || !ux || !uy || k < 0 || (size_t)k >= b->tun.size())
    return fail(VL_EINVAL, "bad arguments");
  if (b->s != 0) return fail(VL_EINVAL, "a tunnel can only be initialised before the batch's first step");
  b->own_ok = false;
  const size_t n = b->plans[k].dom.n;
  const vl::BatchTunnel& T = b->tun[k];
  double* field = nullptr;
  VB_CUDA(cudaMalloc(&field, 3 * n * sizeof(double)));
  cudaError_t e = cudaMemcpyAsync(field, rho, n * 8, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(field + n, ux, n * 8, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(field + 2 * n, uy, n * 8, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = b->L->init((int)n, T.ns, b->d_flag + T.cell_off, field, field + n, field + 2 * n, 1.0, 0.0, 0.0,
                   b->tunnel_ptr(b->buf[0], k), b->tunnel_ptr(b->buf[1], k), b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(field);
  if (e != cudaSuccess) return cuda_fail(e, "batch init");
  return VL_OK;
}

int vl_batch_init_grid(vl_batch* b, int k, const float* grid, int gh, int gw, int gc, double x0, double dx, double y0,
                       double dy, double u) {
  if (!b || !b->built || !grid || k < 0 || (size_t)k >= b->tun.size() || gh < 2 || gw < 2 || gc < 3 || !(dx > 0.0) ||
      !(dy > 0.0))
    return fail(VL_EINVAL, "bad arguments");
  if (b->s != 0) return fail(VL_EINVAL, "a tunnel can only be initialised before the batch's first step");
  b->own_ok = false;
  const vl::BatchTunnel& T = b->tun[k];
  const size_t n = b->plans[k].dom.n;
  cudaError_t e = b->L->init_grid(T.nx, (int)n, T.ns, b->d_flag + T.cell_off, grid, gh, gw, gc, x0, dx, y0, dy, u,
                                  b->tunnel_ptr(b->buf[0], k), b->tunnel_ptr(b->buf[1], k), b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch init from grid");
  return VL_OK;
}

int vl_batch_flags(vl_batch* b, int k, uint8_t* out) {
  if (!b || !out || k < 0 || (size_t)k >= b->plans.size()) return fail(VL_EINVAL, "bad arguments");
  std::memcpy(out, b->plans[k].dom.flag.data(), b->plans[k].dom.n);
  return VL_OK;
}

int vl_batch_state_hash(vl_batch* b, int k, uint64_t* out) {
  if (!b || !out || k < 0 || (size_t)k >= b->plans.size()) return fail(VL_EINVAL, "bad arguments");
  const size_t n = b->plans[k].dom.n;
  std::vector<double> f(9 * n);
  int rc = vl_batch_download(b, k, f.data());
  if (rc) return rc;
  const std::vector<uint8_t>& flag = b->plans[k].dom.flag;
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t idx = 0; idx < n; ++idx) {
    if (flag[idx] == 2) continue;
    for (int i = 0; i < 9; ++i) {
      uint64_t bits;
      std::memcpy(&bits, &f[(size_t)i * n + idx], 8);
      for (int q = 0; q < 8; ++q) {
        h ^= (bits >> (8 * q)) & 0xffu;
        h *= 0x100000001b3ull;
      }
    }
  }
  *out = h;
  return VL_OK;
}

}  // extern "C"
