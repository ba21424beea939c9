// esr_host.cu -- solver runtime and the C ABI (include/eulersr.h).
//
// A solver owns every case slot of every mesh it was created with. One step
// of all live slots is one launch per kernel (K1 recon, K2 flux, per stage);
// the launch grid walks a block table whose entries point into per-mesh
// segments, so meshes of different sizes (the ragged batch) share launches.
// Steps are issued in chunks captured once as CUDA graphs; stop-rule checks
// (norm reduction + bookkeeping) sit inside the chunk graph at multiples of
// check_every, so a run needs no host round trip until the host polls.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "esr_device.cuh"
#include "esr_faithful.h"
#include "esr_internal.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define ESR_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? ESR_ERR_OOM : ESR_ERR_CUDA,                \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                         \
    }                                                                                          \
  } while (0)

#define ESR_TRY(expr)            \
  do {                           \
    int r_ = (expr);             \
    if (r_ != ESR_OK) return r_; \
  } while (0)

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() { if (p) cudaFree(p); }
  int alloc(size_t count) {
    if (p) { cudaFree(p); p = nullptr; }
    n = count;
    if (count == 0) return ESR_OK;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) { p = nullptr; return fail(ESR_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e)); }
    return ESR_OK;
  }
  // at least `count` elements, keeping the buffer when it is large enough: a
  // call that runs often allocates once and frees nothing (cudaFree waits for
  // every stream of the device, including other solvers' work)
  int reserve(size_t count) {
    if (p && n >= count) return ESR_OK;
    return alloc(count);
  }
};

// page-locked host memory owned by the solver (tables of the overlapped copies)
template <typename T>
struct PinnedBuf {
  T* p = nullptr;
  size_t n = 0;
  ~PinnedBuf() { if (p) cudaFreeHost(p); }
  int reserve(size_t count) {
    if (count <= n) return ESR_OK;
    if (p) { cudaFreeHost(p); p = nullptr; n = 0; }
    cudaError_t e = cudaMallocHost(&p, count * sizeof(T));
    if (e != cudaSuccess) { p = nullptr; return fail(ESR_ERR_OOM, std::string("cudaMallocHost: ") + cudaGetErrorString(e)); }
    n = count;
    return ESR_OK;
  }
};

constexpr int kChunkMax = 64;       // steps per captured chunk (upper bound)
constexpr int kReduceThreads = 256;
constexpr int kReduceCells = 2048;  // cells per reduction block

}  // namespace

using namespace esr;

int esr::report_error(int code, const std::string& msg) { return fail(code, msg); }

// ------------------------------------------------------------------ solver
struct SolverBase {
  virtual ~SolverBase() = default;
  int64_t launches = 0;
  bool batch_busy = false;   // a submitted batch owns the slots until its results are read or it is cancelled
};

template <typename T>
struct SolverT : SolverBase {
  using V = V4<T>;
  esr_params P{};
  int device = 0;
  cudaStream_t stream = nullptr;
  int block = 128;

  struct MeshDev {
    HostMesh own;            // the solver's copy: the caller may destroy its mesh
    const HostMesh* hm = nullptr;
    DevBuf<T> geo;
    DevBuf<int4> nbr;
    DevBuf<int> wall_cell;
    DevBuf<T> wall_nx, wall_ny, wall_ds;
    DevBuf<LsqRef> lsq;  // reference-fidelity float32: per-call least-squares data
    DevBuf<int> patch;   // first cell of every patch (+ n_cells)
    DevBuf<int> inv;  // caller cell -> solver cell
    int B = 0, case0 = 0;
    long long off = 0;
  };
  std::vector<std::unique_ptr<MeshDev>> meshes;
  int n_slots = 0;
  long long total = 0;   // items (cells x slots) over all meshes
  int n_chunks = 0;      // reduction chunks per case (max over meshes)

  DevBuf<Seg<T>> d_segs;
  DevBuf<int2> d_blk;
  int n_blk = 0;
  DevBuf<int4> d_live;   // per mesh segment: live slots (A, divider of A)
  std::vector<int4> h_live_poll;   // its host copy at a batch poll
  std::vector<int4> h_live_full;   // A = B for every segment
  DevBuf<int4> d_pblk;   // K2 by patches: (mesh segment, patch, first slot) per block
  int n_pblk = 0;
  bool use_patch = false;
  // second register budget of each fast float32 kernel (autotuned)
  bool k1_alt = false, k2_alt = false, kp_alt = false;
  // K2 per cell for a batch's tail: once few cases run, a patch block's lanes
  // (one per slot of a 32-slot group) are mostly idle while the per-cell K2
  // maps its threads onto the live slots alone; both give the same bits
  bool tail_cell_k2 = false;
#ifndef ESR_TAIL_SLOTS
#define ESR_TAIL_SLOTS 24
#endif
  static constexpr int kTailSlots = ESR_TAIL_SLOTS;   // live slots per mesh at or below which the tail form runs
  DevBuf<int> d_case_seg, d_case_slot, d_ncells;

  DevBuf<V> W, Wa, Wref, FV, Wp;   // Wp: probe step output (batch solves)
  DevBuf<T> dt_local, res;
  DevBuf<T> dt, strength;
  DevBuf<V> inlet;
  DevBuf<double> cfl, tf, qref, forces;
  DevBuf<long long> max_steps, t_start, t_end;
  DevBuf<int> active, step, nmax, nmax_inf, ref_step, streak, streak_start, stopping, status, due, fill;
  DevBuf<double> last_rel, thr;
  DevBuf<int> eng_track, eng_patience, eng_streak, eng_start, eng_stop, eng_stopping;
  DevBuf<double4> eng_t;
  DevBuf<double2> partial;
  DevBuf<double> stage_rows;  // host rows staging for set/get state

  // host mirrors of per-slot case data
  std::vector<int> hcase_index;
  Consts<T> kc{};

  // graphs
  cudaGraphExec_t g_run = nullptr;   // chunk with stop-rule checks
  int g_run_len = 0;
  cudaGraphExec_t g_plain = nullptr; // chunk without checks
  int g_plain_len = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  // per-launch event pairs while profiling (kind 0 recon, 1 flux, 2 other)
  struct Tap { cudaEvent_t a, b; int kind; };
  std::vector<Tap>* taps = nullptr;
  void tap_begin(int kind) {
    if (!taps) return;
    Tap t{nullptr, nullptr, kind};
    cudaEventCreate(&t.a);
    cudaEventCreate(&t.b);
    cudaEventRecord(t.a, stream);
    taps->push_back(t);
  }
  void tap_end() {
    if (taps && !taps->empty()) cudaEventRecord(taps->back().b, stream);
  }

  ~SolverT() override {
    if (pend) {   // a batch still pending: let its work finish before its buffers go
      cudaStreamSynchronize(stream);
      pend.reset();
    }
    if (g_run) cudaGraphExecDestroy(g_run);
    if (g_plain) cudaGraphExecDestroy(g_plain);
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : {ev_in_ready, ev_in_consumed, ev_out_ready, ev_out_done})
      if (e) cudaEventDestroy(e);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (stream) cudaStreamDestroy(stream);
  }

  Cases<T> cases(bool ignore_nmax = false) {
    Cases<T> c;
    c.dt = dt.p; c.inlet = inlet.p; c.strength = strength.p; c.active = active.p; c.step = step.p;
    c.nmax = ignore_nmax ? nmax_inf.p : nmax.p;
    return c;
  }
  CaseCtl ctl() {
    CaseCtl c;
    c.active = active.p; c.step = step.p; c.nmax = nmax.p; c.ref_step = ref_step.p; c.streak = streak.p;
    c.streak_start = streak_start.p; c.stopping_step = stopping.p; c.status = status.p; c.due = due.p;
    c.last_rel = last_rel.p; c.t_start = t_start.p; c.t_end = t_end.p;
    c.eng_track = eng_track.p; c.eng_patience = eng_patience.p; c.eng_t = eng_t.p; c.eng_streak = eng_streak.p;
    c.eng_start = eng_start.p; c.eng_stop = eng_stop.p; c.eng_stopping = eng_stopping.p; c.forces = forces.p;
    c.thr = thr.p;
    return c;
  }
  CaseMap cmap() { return CaseMap{d_case_seg.p, d_case_slot.p}; }
  Seg<T> hseg0{};   // host copy of the first segment (one-mesh block map)
  BlockMap<T> bmap() { return BlockMap<T>{d_segs.p, d_blk.p, hseg0, meshes.size() == 1 ? 1 : 0}; }
  // float32 with esr_params.fidelity = ESR_FIDELITY_REFERENCE: the kernels of esr_faithful.cu
  bool faithful() const { return sizeof(T) == 4 && P.fidelity == ESR_FIDELITY_REFERENCE; }
  static constexpr bool kF = sizeof(T) == 4;   // FAST flag of the kernels this file instantiates
  // K2 by patches applies to float32 fast-fidelity HLLC + MUSCL solves
  bool patch_eligible() const {
    return sizeof(T) == 4 && !faithful() && P.flux == ESR_FLUX_HLLC && P.reconstruction == ESR_RECON_MUSCL;
  }

  int init(const esr_mesh* const* ms, const int32_t* slots, int nm, const esr_params* p) {
    P = *p;
    device = p->device;
    ESR_CUDA(cudaSetDevice(device));
    int least = 0, greatest = 0;
    ESR_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int prio = std::min(least, std::max(greatest, (int)p->stream_priority));
    ESR_CUDA(cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, prio));
    ESR_CUDA(cudaEventCreate(&ev0));
    ESR_CUDA(cudaEventCreate(&ev1));
    const double g = p->gamma;
    kc.gamma = (T)g;
    kc.gm1 = (T)(g - 1.0);
    kc.gm1_14 = (T)(1.4 - 1.0);
    kc.inv_gm1 = (T)(1.0 / (g - 1.0));
    kc.inv_gm1_14 = (T)(1.0 / (1.4 - 1.0));
    kc.half = (T)0.5;
    kc.eps_lim = sizeof(T) == 8 ? (T)1e-12 : (T)1e-7;
    kc.venk_eps = (T)1e-7;
    kc.ss_eps = (T)1e-6;
    kc.den_eps = (T)1e-12;
    // layout
    long long off = 0;
    int case0 = 0;
    int max_cells = 0;
    for (int m = 0; m < nm; ++m) {
      auto md = std::make_unique<MeshDev>();
      md->own = ms[m]->hm;
      md->hm = &md->own;
      md->B = slots[m];
      md->case0 = case0;
      md->off = off;
      off += (long long)md->hm->n_cells * md->B;
      case0 += md->B;
      max_cells = std::max(max_cells, md->hm->n_cells);
      meshes.push_back(std::move(md));
    }
    n_slots = case0;
    total = off;
    if (n_slots <= 0 || total <= 0) return fail(ESR_ERR_ARG, "solver: no case slots");
    if (total > (long long)INT_MAX * 4) return fail(ESR_ERR_ARG, "solver: too many cells x slots");
    n_chunks = (max_cells + kReduceCells - 1) / kReduceCells;
    const auto& hm0 = *meshes[0]->hm;
    kc.sub_rho = (T)hm0.inlet_subsonic[0];
    kc.sub_u = (T)hm0.inlet_subsonic[1];
    kc.sub_v = (T)hm0.inlet_subsonic[2];
    // block size: enough blocks to cover the SMs twice when possible
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    block = p->block_size > 0 ? p->block_size : 0;
    if (p->block_size == ESR_BLOCK_PATCHES) {
      block = 128;
      use_patch = patch_eligible();
    } else if (block == 0) {   // starting point; measured below
      block = 256;
      while (block > 64 && (total + block - 1) / block < 2 * sms) block /= 2;
    }
    if (block != 64 && block != 128 && block != 256)
      return fail(ESR_ERR_ARG, "solver: block_size must be 0, 64, 128, 256 or ESR_BLOCK_PATCHES");
    // upload meshes
    std::vector<Seg<T>> hsegs;
    std::vector<int> hseg_of(n_slots), hslot_of(n_slots), hnc(n_slots);
    for (int m = 0; m < nm; ++m) {
      MeshDev& md = *meshes[m];
      const HostMesh& hm = *md.hm;
      const int N = hm.n_cells;
      // geometry records: float64 rounded once (fast), or formed as the
      // reference forms them in the run's precision (reference fidelity)
      const bool ref = P.fidelity == ESR_FIDELITY_REFERENCE;
      std::vector<T> g(hm.geo.size());
      for (size_t i = 0; i < g.size(); ++i)
        g[i] = ref ? (sizeof(T) == 4 ? (T)hm.geo_ref32[i] : (T)hm.geo_ref64[i]) : (T)hm.geo[i];
      ESR_TRY(md.geo.alloc(g.size()));
      ESR_CUDA(cudaMemcpy(md.geo.p, g.data(), g.size() * sizeof(T), cudaMemcpyHostToDevice));
      if (faithful()) {
        ESR_TRY(md.lsq.alloc(N));
        ESR_CUDA(cudaMemcpy(md.lsq.p, hm.lsq_ref32.data(), (size_t)N * sizeof(LsqRef), cudaMemcpyHostToDevice));
      }
      ESR_TRY(md.nbr.alloc(N));
      ESR_CUDA(cudaMemcpy(md.nbr.p, hm.nbr.data(), (size_t)N * sizeof(int4), cudaMemcpyHostToDevice));
      const int nw = (int)hm.wall_cell.size();
      std::vector<T> wx(nw), wy(nw), wd(nw);
      for (int i = 0; i < nw; ++i) {
        if (!ref) { wx[i] = (T)hm.wall_n[2 * i]; wy[i] = (T)hm.wall_n[2 * i + 1]; wd[i] = (T)hm.wall_ds[i]; }
        else if (sizeof(T) == 4) { wx[i] = (T)hm.wall_n_ref32[2 * i]; wy[i] = (T)hm.wall_n_ref32[2 * i + 1]; wd[i] = (T)hm.wall_ds_ref32[i]; }
        else { wx[i] = (T)hm.wall_n_ref64[2 * i]; wy[i] = (T)hm.wall_n_ref64[2 * i + 1]; wd[i] = (T)hm.wall_ds_ref64[i]; }
      }
      ESR_TRY(md.wall_cell.alloc(std::max(nw, 1)));
      ESR_TRY(md.wall_nx.alloc(std::max(nw, 1)));
      ESR_TRY(md.wall_ny.alloc(std::max(nw, 1)));
      ESR_TRY(md.wall_ds.alloc(std::max(nw, 1)));
      if (nw) {
        ESR_CUDA(cudaMemcpy(md.wall_cell.p, hm.wall_cell.data(), nw * sizeof(int), cudaMemcpyHostToDevice));
        ESR_CUDA(cudaMemcpy(md.wall_nx.p, wx.data(), nw * sizeof(T), cudaMemcpyHostToDevice));
        ESR_CUDA(cudaMemcpy(md.wall_ny.p, wy.data(), nw * sizeof(T), cudaMemcpyHostToDevice));
        ESR_CUDA(cudaMemcpy(md.wall_ds.p, wd.data(), nw * sizeof(T), cudaMemcpyHostToDevice));
      }
      ESR_TRY(md.inv.alloc(N));
      ESR_CUDA(cudaMemcpy(md.inv.p, hm.inv.data(), N * sizeof(int), cudaMemcpyHostToDevice));
      ESR_TRY(md.patch.alloc(hm.patch_start.size()));
      ESR_CUDA(cudaMemcpy(md.patch.p, hm.patch_start.data(), hm.patch_start.size() * sizeof(int),
                          cudaMemcpyHostToDevice));
      Seg<T> s{};
      s.n_cells = N; s.B = md.B; s.case0 = md.case0; s.geo_stride = G_COUNT; s.off = md.off;
      s.nbr = md.nbr.p; s.geo = md.geo.p; s.wall_cell = md.wall_cell.p; s.wall_nx = md.wall_nx.p;
      s.wall_ny = md.wall_ny.p; s.wall_ds = md.wall_ds.p; s.n_wall = nw;
      s.lsq = md.lsq.p;
      s.patch_start = md.patch.p;
      s.n_patches = (int)hm.patch_start.size() - 1;
      ESR_TRY(set_divider(s));
      h_live_full.push_back(make_int4(s.B, (int)s.b_magic, s.b_shift, 0));
      hsegs.push_back(s);
      for (int b = 0; b < md.B; ++b) { hseg_of[md.case0 + b] = m; hslot_of[md.case0 + b] = b; hnc[md.case0 + b] = N; }
    }
    ESR_TRY(d_live.alloc(hsegs.size()));
    ESR_CUDA(cudaMemcpy(d_live.p, h_live_full.data(), hsegs.size() * sizeof(int4), cudaMemcpyHostToDevice));
    for (size_t m = 0; m < hsegs.size(); ++m) hsegs[m].live = hsegs[m].B > 1 ? d_live.p + m : nullptr;
    ESR_TRY(d_segs.alloc(hsegs.size()));
    ESR_CUDA(cudaMemcpy(d_segs.p, hsegs.data(), hsegs.size() * sizeof(Seg<T>), cudaMemcpyHostToDevice));
    hseg0 = hsegs[0];
    ESR_TRY(build_blocks(block));
    ESR_TRY(build_patch_blocks());
    ESR_TRY(d_case_seg.alloc(n_slots));
    ESR_TRY(d_case_slot.alloc(n_slots));
    ESR_TRY(d_ncells.alloc(n_slots));
    ESR_CUDA(cudaMemcpy(d_case_seg.p, hseg_of.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice));
    ESR_CUDA(cudaMemcpy(d_case_slot.p, hslot_of.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice));
    ESR_CUDA(cudaMemcpy(d_ncells.p, hnc.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice));
    // state
    ESR_TRY(W.alloc(total));
    ESR_TRY(Wa.alloc(total));
    ESR_TRY(Wref.alloc(total));
    if (P.reconstruction == ESR_RECON_MUSCL) ESR_TRY(FV.alloc(3 * total));
    if (P.dt_mode == ESR_DT_LOCAL) ESR_TRY(dt_local.alloc(total));
    if (P.stop_rule == ESR_STOP_DENSITY_L2) ESR_TRY(res.alloc(total));
    ESR_CUDA(cudaMemsetAsync(W.p, 0, total * sizeof(V), stream));
    ESR_CUDA(cudaMemsetAsync(Wa.p, 0, total * sizeof(V), stream));
    ESR_CUDA(cudaMemsetAsync(Wref.p, 0, total * sizeof(V), stream));
    // per-slot arrays
    ESR_TRY(dt.alloc(n_slots)); ESR_TRY(strength.alloc(n_slots)); ESR_TRY(inlet.alloc(n_slots));
    ESR_TRY(cfl.alloc(n_slots)); ESR_TRY(tf.alloc(n_slots)); ESR_TRY(qref.alloc(n_slots));
    ESR_TRY(forces.alloc(2 * n_slots)); ESR_TRY(max_steps.alloc(n_slots));
    ESR_TRY(t_start.alloc(n_slots)); ESR_TRY(t_end.alloc(n_slots));
    for (DevBuf<int>* b : {&active, &step, &nmax, &nmax_inf, &ref_step, &streak, &streak_start, &stopping, &status, &due, &fill})
      ESR_TRY(b->alloc(n_slots));
    ESR_TRY(last_rel.alloc(n_slots));
    ESR_TRY(thr.alloc(n_slots));
    ESR_CUDA(cudaMemsetAsync(thr.p, 0, n_slots * sizeof(double), stream));
    for (DevBuf<int>* b : {&eng_track, &eng_patience, &eng_streak, &eng_start, &eng_stop, &eng_stopping}) {
      ESR_TRY(b->alloc(n_slots));
      ESR_CUDA(cudaMemsetAsync(b->p, 0, n_slots * sizeof(int), stream));
    }
    ESR_TRY(eng_t.alloc(n_slots));
    ESR_CUDA(cudaMemsetAsync(eng_t.p, 0, n_slots * sizeof(double4), stream));
    ESR_CUDA(cudaMemsetAsync(forces.p, 0, 2 * n_slots * sizeof(double), stream));
    ESR_TRY(partial.alloc((size_t)n_slots * n_chunks));
    for (DevBuf<int>* b : {&active, &step, &nmax, &ref_step, &streak, &streak_start, &stopping, &status, &due, &fill})
      ESR_CUDA(cudaMemsetAsync(b->p, 0, n_slots * sizeof(int), stream));
    std::vector<int> inf(n_slots, INT_MAX);
    ESR_CUDA(cudaMemcpy(nmax_inf.p, inf.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice));
    ESR_CUDA(cudaMemsetAsync(dt.p, 0, n_slots * sizeof(T), stream));
    ESR_CUDA(cudaMemsetAsync(strength.p, 0, n_slots * sizeof(T), stream));
    ESR_CUDA(cudaMemsetAsync(inlet.p, 0, n_slots * sizeof(V), stream));
    hcase_index.assign(n_slots, -1);
    ESR_CUDA(cudaStreamSynchronize(stream));
    if (p->block_size == 0) ESR_TRY(autotune());
    return ESR_OK;
  }

  // item -> cell without a divide: q = (umulhi(n, m) + n) >> l with
  // l = ceil(log2 B), m = floor(2^32 (2^l - B) / B) + 1 (exact for n < 2^31)
  static int set_divider(Seg<T>& s) {
    const uint32_t d = (uint32_t)s.B;
    const Divider v = make_divider(d);
    s.b_magic = v.magic;
    s.b_shift = v.shift;
    const uint64_t items = (uint64_t)s.n_cells * d;
    if (items >= (1ull << 31)) return fail(ESR_ERR_ARG, "solver: cells x slots of one mesh must stay below 2^31");
    for (uint64_t n : {uint64_t(0), uint64_t(d - 1), uint64_t(d), items - 1, items / 2 + 1}) {
      if (n < items && divide((uint32_t)n, v) != n / d) return fail(ESR_ERR_STATE, "solver: item divider check failed");
    }
    return ESR_OK;
  }

  // block table: one entry (mesh, first item) per block of `blk` items
  int build_blocks(int blk) {
    std::vector<int2> hblk;
    for (int m = 0; m < (int)meshes.size(); ++m) {
      const long long items = (long long)meshes[m]->hm->n_cells * meshes[m]->B;
      for (long long b0 = 0; b0 < items; b0 += blk) hblk.push_back(make_int2(m, (int)b0));
    }
    ESR_TRY(d_blk.alloc(hblk.size()));
    ESR_CUDA(cudaMemcpy(d_blk.p, hblk.data(), hblk.size() * sizeof(int2), cudaMemcpyHostToDevice));
    n_blk = (int)hblk.size();
    block = blk;
    return ESR_OK;
  }

  // block table of K2 by patches: every patch of every mesh x groups of 32 slots
  int build_patch_blocks() {
    std::vector<int4> h;
    for (int m = 0; m < (int)meshes.size(); ++m) {
      const std::vector<int>& ps = meshes[m]->hm->patch_start;
      const int np = (int)ps.size() - 1;
      // the kernel's shared arrays hold kPatchCells cells
      for (int p = 0; p < np; ++p)
        if (ps[p + 1] - ps[p] < 1 || ps[p + 1] - ps[p] > kPatchCells)
          return fail(ESR_ERR_STATE, "patch table: a patch has " + std::to_string(ps[p + 1] - ps[p]) + " cells");
      for (int p = 0; p < np; ++p)
        for (int b0 = 0; b0 < meshes[m]->B; b0 += 32) h.push_back(make_int4(m, p, b0, 0));
    }
    ESR_TRY(d_pblk.alloc(h.size()));
    if (!h.empty()) ESR_CUDA(cudaMemcpy(d_pblk.p, h.data(), h.size() * sizeof(int4), cudaMemcpyHostToDevice));
    n_pblk = (int)h.size();
    return ESR_OK;
  }

  // Autotuner: time one full step of every slot (the solver's own meshes,
  // scheme and slot counts; a uniform finite state, all slots live) for each
  // launch shape and keep the fastest. Shapes: the cell kernels at 64, 128
  // and 256 threads per block; at the best of those, K2's second register
  // budget, K2 by patches at both budgets, then K1's second budget with the
  // best K2. Results do not depend on the choice: every item is computed the
  // same way whatever block and kernel form it falls in. The choice is kept
  // per process for each solver shape (device, precision, scheme, meshes'
  // cells and slots), so a second solver of the same shape skips the timing.
  struct TuneChoice {
    int block = 256;
    bool patches = false, k1 = false, k2 = false, kp = false;
  };
  struct TuneEntry {
    TuneChoice choice;
    esr_tuning record;
  };
  static std::mutex& tune_mutex() { static std::mutex m; return m; }
  static std::map<std::string, TuneEntry>& tune_cache() { static std::map<std::string, TuneEntry> c; return c; }
  std::string tune_key() const {
    std::string k = std::to_string(device) + "/" + std::to_string(sizeof(T)) + "/" + std::to_string(P.fidelity) + "/" +
                    std::to_string(P.flux) + "/" + std::to_string(P.reconstruction) + "/" +
                    std::to_string(P.time_scheme) + "/" + std::to_string(P.dt_mode);
    for (const auto& m : meshes) k += "/" + std::to_string(m->hm->n_cells) + "x" + std::to_string(m->B);
    return k;
  }
  bool fast_float() const { return sizeof(T) == 4 && !faithful(); }
  int k1_minb_of(const TuneChoice& c) const {
    if (!fast_float() || P.reconstruction != ESR_RECON_MUSCL) return 0;
    return c.k1 ? ESR_K1_MINB_ALT : ESR_K1_MINB;
  }
  int k2_minb_of(const TuneChoice& c) const {
    if (!fast_float()) return 0;
    if (c.patches) return c.kp ? ESR_PATCH_MINB_ALT : ESR_PATCH_MINB;
    return c.k2 ? ESR_K2_MINB_ALT : ESR_K2_MINB;
  }
  int apply_choice(const TuneChoice& c) {
    ESR_TRY(build_blocks(c.block));
    use_patch = c.patches && patch_eligible();
    k1_alt = c.k1;
    k2_alt = c.k2;
    kp_alt = c.kp;
    return ESR_OK;
  }
  int time_choice(const TuneChoice& c, const Cases<T>& cs, double& ms) {
    ESR_TRY(apply_choice(c));
    step_kernels(cs, 0);   // warm-up
    ESR_CUDA(cudaEventRecord(ev0, stream));
    for (int r = 0; r < 3; ++r) step_kernels(cs, 0);
    ESR_CUDA(cudaEventRecord(ev1, stream));
    ESR_CUDA(cudaEventSynchronize(ev1));
    float t = 0.f;
    ESR_CUDA(cudaEventElapsedTime(&t, ev0, ev1));
    ms = t / 3.0;
    if (tuning.n_variants < ESR_TUNING_MAX_VARIANTS) {
      esr_tuning_variant& v = tuning.variants[tuning.n_variants++];
      v.block_size = c.block;
      v.k2_patches = c.patches ? 1 : 0;
      v.k1_minb = k1_minb_of(c);
      v.k2_minb = k2_minb_of(c);
      v.step_ms = ms;
    }
    return ESR_OK;
  }
  esr_tuning tuning{};
  TuneChoice chosen;
  int autotune() {
    const std::string key = tune_key();
    {
      std::lock_guard<std::mutex> lock(tune_mutex());
      auto it = tune_cache().find(key);
      if (it != tune_cache().end()) {
        chosen = it->second.choice;
        tuning = it->second.record;
        tuning.cached = 1;
        return apply_choice(chosen);
      }
    }
    const V w0 = mk4<T>(T(1), T(0.5), T(0.1), T(2.5));
    const int tb = 256;
    k_fill_uniform<T><<<(int)std::min<long long>((total + tb - 1) / tb, 65535), tb, 0, stream>>>(W.p, total, w0);
    std::vector<V> in(n_slots, w0);
    std::vector<T> dts(n_slots, T(1e-4));
    std::vector<int> on(n_slots, 1);
    ESR_CUDA(cudaMemcpyAsync(inlet.p, in.data(), n_slots * sizeof(V), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(dt.p, dts.data(), n_slots * sizeof(T), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(active.p, on.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    const Cases<T> cs = cases(true);
    const int64_t before = launches;
    tuning = esr_tuning{};
    double best = 1e300, ms = 0.0;
    TuneChoice best_c;
    auto consider = [&](const TuneChoice& c) -> int {
      ESR_TRY(time_choice(c, cs, ms));
      if (ms < best) { best = ms; best_c = c; }
      return ESR_OK;
    };
    const int cand[3] = {64, 128, 256};
    tuning.n_candidates = 3;
    for (int i = 0; i < 3; ++i) {
      TuneChoice c;
      c.block = cand[i];
      ESR_TRY(consider(c));
      tuning.candidates[i] = cand[i];
      tuning.step_ms[i] = ms;
    }
    const int best_blk = best_c.block;
    const bool muscl = P.reconstruction == ESR_RECON_MUSCL;
    if (fast_float() && muscl && P.flux == ESR_FLUX_HLLC) {   // K2 per cell, second budget
      TuneChoice c;
      c.block = best_blk;
      c.k2 = true;
      ESR_TRY(consider(c));
    }
    if (patch_eligible()) {   // K2 by patches, K1 at the best block size
      TuneChoice c;
      c.block = best_blk;
      c.patches = true;
      ESR_TRY(consider(c));
      tuning.candidates[3] = ESR_BLOCK_PATCHES;
      tuning.step_ms[3] = ms;
      tuning.n_candidates = 4;
      c.kp = true;
      ESR_TRY(consider(c));
    }
    if (fast_float() && muscl) {   // K1, second budget, with the best K2
      TuneChoice c = best_c;
      c.k1 = true;
      ESR_TRY(consider(c));
    }
    launches = before;
    chosen = best_c;
    ESR_TRY(apply_choice(chosen));
    tuning.block_size = chosen.block;
    tuning.k2_patches = use_patch ? 1 : 0;
    tuning.k1_minb = k1_minb_of(chosen);
    tuning.k2_minb = k2_minb_of(chosen);
    tuning.cached = 0;
    ESR_CUDA(cudaMemsetAsync(W.p, 0, total * sizeof(V), stream));
    ESR_CUDA(cudaMemsetAsync(Wa.p, 0, total * sizeof(V), stream));
    ESR_CUDA(cudaMemsetAsync(active.p, 0, n_slots * sizeof(int), stream));
    ESR_CUDA(cudaMemsetAsync(dt.p, 0, n_slots * sizeof(T), stream));
    ESR_CUDA(cudaMemsetAsync(inlet.p, 0, n_slots * sizeof(V), stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    ESR_CUDA(cudaGetLastError());
    std::lock_guard<std::mutex> lock(tune_mutex());
    tune_cache()[key] = TuneEntry{chosen, tuning};
    return ESR_OK;
  }
  // a launch shape given by the caller (one recorded by an earlier
  // autotuning, say); the chunk graphs are captured again at the next step
  int set_shape(const esr_tuning_variant* v) {
    if (v->block_size != 64 && v->block_size != 128 && v->block_size != 256)
      return fail(ESR_ERR_ARG, "set_shape: block_size must be 64, 128 or 256");
    if (v->k2_patches != 0 && v->k2_patches != 1) return fail(ESR_ERR_ARG, "set_shape: k2_patches must be 0 or 1");
    if (v->k2_patches && !patch_eligible())
      return fail(ESR_ERR_ARG, "set_shape: K2 by patches needs a float32 fast-fidelity HLLC + MUSCL solver");
    TuneChoice c;
    c.block = v->block_size;
    c.patches = v->k2_patches == 1;
    const bool muscl = P.reconstruction == ESR_RECON_MUSCL;
    if (v->k1_minb != 0) {
      if (!fast_float() || !muscl || (v->k1_minb != ESR_K1_MINB && v->k1_minb != ESR_K1_MINB_ALT))
        return fail(ESR_ERR_ARG, "set_shape: k1_minb must be 0 or one of K1's two register budgets (" +
                                     std::to_string(ESR_K1_MINB) + ", " + std::to_string(ESR_K1_MINB_ALT) +
                                     ") of a float32 fast-fidelity MUSCL solver");
      c.k1 = v->k1_minb == ESR_K1_MINB_ALT;
    }
    if (v->k2_minb != 0) {
      const int def = c.patches ? ESR_PATCH_MINB : ESR_K2_MINB, alt = c.patches ? ESR_PATCH_MINB_ALT : ESR_K2_MINB_ALT;
      const bool ok = fast_float() && (c.patches || (muscl && P.flux == ESR_FLUX_HLLC)) &&
                      (v->k2_minb == def || v->k2_minb == alt);
      if (!ok)
        return fail(ESR_ERR_ARG, "set_shape: k2_minb must be 0 or one of the K2 form's two register budgets (" +
                                     std::to_string(def) + ", " + std::to_string(alt) +
                                     ") of a float32 fast-fidelity HLLC + MUSCL solver");
      (c.patches ? c.kp : c.k2) = v->k2_minb == alt;
    }
    ESR_TRY(apply_choice(c));
    chosen = c;
    if (g_run) cudaGraphExecDestroy(g_run);
    if (g_plain) cudaGraphExecDestroy(g_plain);
    g_run = g_plain = nullptr;
    g_run_len = g_plain_len = 0;
    tuning.block_size = c.block;
    tuning.k2_patches = use_patch ? 1 : 0;
    tuning.k1_minb = k1_minb_of(c);
    tuning.k2_minb = k2_minb_of(c);
    return ESR_OK;
  }
  int get_tuning(esr_tuning* out) {
    *out = tuning;
    if (out->block_size == 0) out->block_size = block;   // given, not measured
    out->k2_patches = use_patch ? 1 : 0;
    TuneChoice now = chosen;
    now.patches = use_patch;
    out->k1_minb = k1_minb_of(now);
    out->k2_minb = k2_minb_of(now);
    return ESR_OK;
  }

  int mesh_of_slot(int slot, int& m, int& b) {
    if (slot < 0 || slot >= n_slots) return fail(ESR_ERR_ARG, "slot out of range");
    for (m = 0; m < (int)meshes.size(); ++m) {
      if (slot < meshes[m]->case0 + meshes[m]->B) { b = slot - meshes[m]->case0; return ESR_OK; }
    }
    return fail(ESR_ERR_ARG, "slot out of range");
  }

  // ---------------------------------------------------------------- kernels
  template <int FLUX, bool MUSCL, int STAGE, bool LOCALDT>
  void launch_flux(const V* win, const V* wbase, V* wout, const Cases<T>& cs, int pos) {
    tap_begin(1);
    bool done = false;
    if constexpr (sizeof(T) == 4 && FLUX == 0 && MUSCL) {
      if (k2_alt) {
        k_flux<T, kF, FLUX, MUSCL, STAGE, LOCALDT, ESR_K2_MINB_ALT><<<n_blk, block, 0, stream>>>(
            bmap(), win, wbase, wout, FV.p, total, cs, kc, pos, dt_local.p, res.p);
        done = true;
      }
    }
    if (!done)
      k_flux<T, kF, FLUX, MUSCL, STAGE, LOCALDT><<<n_blk, block, 0, stream>>>(bmap(), win, wbase, wout, FV.p,
                                                                              total, cs, kc, pos, dt_local.p, res.p);
    tap_end();
    ++launches;
  }
  template <int STAGE, bool LOCALDT>
  void launch_patch(const V* win, const V* wbase, V* wout, const Cases<T>& cs, int pos) {
    if constexpr (sizeof(T) == 4) {
      if (kp_alt)
        k_flux_patch<STAGE, LOCALDT, ESR_PATCH_MINB_ALT><<<n_pblk, 32 * kPatchWarps, 0, stream>>>(
            d_segs.p, d_pblk.p, win, wbase, wout, FV.p, total, cs, kc, pos, dt_local.p, res.p);
      else
        k_flux_patch<STAGE, LOCALDT><<<n_pblk, 32 * kPatchWarps, 0, stream>>>(d_segs.p, d_pblk.p, win, wbase, wout,
                                                                              FV.p, total, cs, kc, pos, dt_local.p,
                                                                              res.p);
    }
  }
  template <int STAGE>
  void flux_dispatch(const V* win, const V* wbase, V* wout, const Cases<T>& cs, int pos) {
    const bool muscl = P.reconstruction == ESR_RECON_MUSCL;
    const bool local = P.dt_mode == ESR_DT_LOCAL;
    const bool rus = P.flux == ESR_FLUX_RUSANOV;
    if constexpr (sizeof(T) == 4) {
      if (faithful()) {
        tap_begin(1);
        faithful_flux(STAGE, bmap(), win, wbase, wout, FV.p, total, cs, kc, pos, dt_local.p, res.p, rus, muscl, local,
                      n_blk, block, stream);
        tap_end();
        ++launches;
        return;
      }
      if (use_patch && !tail_cell_k2 && n_pblk > 0) {   // eligible by construction: HLLC + MUSCL, fast fidelity
        tap_begin(1);
        if (local) launch_patch<STAGE, true>(win, wbase, wout, cs, pos);
        else launch_patch<STAGE, false>(win, wbase, wout, cs, pos);
        tap_end();
        ++launches;
        return;
      }
    }
#define ESR_FLUX_CASE(F, M, L) if (rus == (F == 1) && muscl == M && local == L) { launch_flux<F, M, STAGE, L>(win, wbase, wout, cs, pos); return; }
    ESR_FLUX_CASE(0, true, false) ESR_FLUX_CASE(0, true, true) ESR_FLUX_CASE(0, false, false) ESR_FLUX_CASE(0, false, true)
    ESR_FLUX_CASE(1, true, false) ESR_FLUX_CASE(1, true, true) ESR_FLUX_CASE(1, false, false) ESR_FLUX_CASE(1, false, true)
#undef ESR_FLUX_CASE
  }
  void recon(const V* w, const Cases<T>& cs, int pos, bool write_dt) {
    const bool muscl = P.reconstruction == ESR_RECON_MUSCL;
    if (!muscl && !write_dt) return;   // constant reconstruction needs K1 only for the local dt
    if constexpr (sizeof(T) == 4) {
      if (faithful()) {
        tap_begin(0);
        faithful_recon(bmap(), w, FV.p, total, cs, kc, pos, dt_local.p, muscl, write_dt, n_blk, block, stream);
        tap_end();
        ++launches;
        return;
      }
    }
    if (!muscl) {
      k_recon<T, kF, false, true><<<n_blk, block, 0, stream>>>(bmap(), w, nullptr, 0, cs, kc, pos, dt_local.p);
      ++launches;
      return;
    }
    tap_begin(0);
    if (write_dt) {   // the local-dt K1 keeps its one budget
      k_recon<T, kF, true, true><<<n_blk, block, 0, stream>>>(bmap(), w, FV.p, total, cs, kc, pos, dt_local.p);
    } else if (sizeof(T) == 4 && k1_alt) {
      k_recon<T, kF, true, false, (sizeof(T) == 4 ? ESR_K1_MINB_ALT : 0)><<<n_blk, block, 0, stream>>>(
          bmap(), w, FV.p, total, cs, kc, pos, dt_local.p);
    } else {
      k_recon<T, kF, true, false><<<n_blk, block, 0, stream>>>(bmap(), w, FV.p, total, cs, kc, pos, dt_local.p);
    }
    tap_end();
    ++launches;
  }
  // per-case minimum CFL step partials of the slots flagged in `flags`
  void dtmin_reduce(const int* flags) {
    dim3 grid(n_chunks, n_slots);
    if constexpr (sizeof(T) == 4) {
      if (faithful()) {
        faithful_dtmin(grid, kReduceThreads, d_segs.p, cmap(), W.p, flags, kReduceCells, partial.p, n_chunks, kc, stream);
        return;
      }
    }
    k_case_reduce<T, RED_DTMIN><<<grid, kReduceThreads, 0, stream>>>(d_segs.p, cmap(), W.p, nullptr, flags,
                                                                     kReduceCells, partial.p, n_chunks, kc);
  }
  // one time step of every live slot, step index `pos` inside the chunk
  void step_kernels(const Cases<T>& cs, int pos) {
    const bool local = P.dt_mode == ESR_DT_LOCAL;
    switch (P.time_scheme) {
      case ESR_TIME_EE:
        recon(W.p, cs, pos, local);
        flux_dispatch<ST_FIRST>(W.p, nullptr, Wa.p, cs, pos);
        k_commit<T><<<n_blk, block, 0, stream>>>(d_segs.p, d_blk.p, Wa.p, W.p, cs, pos);
        ++launches;
        break;
      case ESR_TIME_RK2:
        recon(W.p, cs, pos, local);
        flux_dispatch<ST_FIRST>(W.p, nullptr, Wa.p, cs, pos);
        recon(Wa.p, cs, pos, false);
        flux_dispatch<ST_RK2_SECOND>(Wa.p, W.p, W.p, cs, pos);
        break;
      default:  // SRK2
        recon(W.p, cs, pos, local);
        flux_dispatch<ST_FIRST>(W.p, nullptr, Wa.p, cs, pos);
        recon(Wa.p, cs, pos, false);
        flux_dispatch<ST_SRK2_SECOND>(Wa.p, W.p, W.p, cs, pos);
        break;
    }
  }
  // One step of the slots active in `cs` written to scratch instead of W
  // (the residual probe); returns the buffer that holds the stepped state.
  V* probe_kernels(const Cases<T>& cs) {
    const bool local = P.dt_mode == ESR_DT_LOCAL;
    recon(W.p, cs, 0, local);
    flux_dispatch<ST_FIRST>(W.p, nullptr, Wa.p, cs, 0);
    if (P.time_scheme == ESR_TIME_EE) return Wa.p;
    recon(Wa.p, cs, 0, false);
    if (P.time_scheme == ESR_TIME_RK2) flux_dispatch<ST_RK2_SECOND>(Wa.p, W.p, Wp.p, cs, 0);
    else flux_dispatch<ST_SRK2_SECOND>(Wa.p, W.p, Wp.p, cs, 0);
    return Wp.p;
  }
  void check_point(int pos) {
    const int tb = 128, nb = (n_slots + tb - 1) / tb;
    k_mark_due<<<nb, tb, 0, stream>>>(ctl(), n_slots, pos, std::max(1, P.check_every));
    dim3 grid(n_chunks, n_slots);
    if (P.stop_rule == ESR_STOP_DENSITY_L2)
      k_case_reduce<T, RED_RESSQ><<<grid, kReduceThreads, 0, stream>>>(d_segs.p, cmap(), W.p, (V*)res.p, due.p,
                                                                       kReduceCells, partial.p, n_chunks, kc);
    else
      k_case_reduce<T, RED_NORM><<<grid, kReduceThreads, 0, stream>>>(d_segs.p, cmap(), W.p, Wref.p, due.p,
                                                                      kReduceCells, partial.p, n_chunks, kc);
    k_forces<T><<<n_slots, 256, 0, stream>>>(d_segs.p, cmap(), W.p, qref.p, forces.p, kc, due.p, eng_track.p);
    k_check<<<nb, tb, 0, stream>>>(ctl(), n_slots, pos, partial.p, n_chunks, d_ncells.p, P.threshold,
                                   std::max(1, P.patience), P.stop_rule, std::max(1, P.check_every));
    launches += 4;
  }
  void issue_run_chunk(int len) {
    const Cases<T> cs = cases(false);
    const int ce = std::max(1, P.check_every);
    for (int i = 0; i < len; ++i) {
      step_kernels(cs, i);
      if ((i + 1) % ce == 0 || i + 1 == len) check_point(i + 1);
    }
    const int tb = 128, nb = (n_slots + tb - 1) / tb;
    k_advance<<<nb, tb, 0, stream>>>(ctl(), n_slots, len, 1);
    ++launches;
  }
  void issue_plain_chunk(int len) {
    const Cases<T> cs = cases(true);
    for (int i = 0; i < len; ++i) step_kernels(cs, i);
    const int tb = 128, nb = (n_slots + tb - 1) / tb;
    tap_begin(2);
    k_advance<<<nb, tb, 0, stream>>>(ctl(), n_slots, len, 0);
    tap_end();
    ++launches;
  }
  int profile(int nsteps, esr_kernel_times* out) {
    if (nsteps <= 0) return fail(ESR_ERR_ARG, "profile_step: nsteps must be > 0");
    std::vector<Tap> v;
    v.reserve((size_t)nsteps * 5 + 4);
    taps = &v;
    issue_plain_chunk(nsteps);
    taps = nullptr;
    cudaError_t e = cudaStreamSynchronize(stream);
    double ms[3] = {0, 0, 0};
    int cnt[3] = {0, 0, 0};
    for (Tap& t : v) {
      float x = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&x, t.a, t.b);
      ms[t.kind] += x;
      cnt[t.kind] += 1;
      cudaEventDestroy(t.a);
      cudaEventDestroy(t.b);
    }
    if (e != cudaSuccess) return fail(ESR_ERR_CUDA, cudaGetErrorString(e));
    out->recon_ms = cnt[0] ? ms[0] / cnt[0] : 0.0;
    out->flux_ms = cnt[1] ? ms[1] / cnt[1] : 0.0;
    out->other_ms = cnt[2] ? ms[2] / cnt[2] : 0.0;
    out->recon_launches = cnt[0];
    out->flux_launches = cnt[1];
    out->other_launches = cnt[2];
    out->reserved = 0;
    return ESR_OK;
  }
  int run_chunk_len() const {
    const int ce = std::max(1, P.check_every);
    if (ce <= kChunkMax) return ce * std::max(1, kChunkMax / ce);
    for (int l = kChunkMax; l >= 1; --l)
      if (ce % l == 0) return l;
    return 1;
  }
  int capture(bool run, int len, cudaGraphExec_t* out) {
    cudaGraph_t graph = nullptr;
    ESR_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    const int64_t before = launches;
    if (run) issue_run_chunk(len); else issue_plain_chunk(len);
    launches = before;  // counted again when the graph is launched
    ESR_CUDA(cudaStreamEndCapture(stream, &graph));
    cudaError_t e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ESR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return ESR_OK;
  }
  int64_t chunk_launches(bool run, int len) {
    const bool muscl = P.reconstruction == ESR_RECON_MUSCL;
    const bool local = P.dt_mode == ESR_DT_LOCAL;
    int per_step;
    if (P.time_scheme == ESR_TIME_EE) per_step = 2 + ((muscl || local) ? 1 : 0);
    else per_step = 2 + (muscl ? 2 : (local ? 1 : 0));
    int64_t n = (int64_t)per_step * len + 1;
    if (run) {
      const int ce = std::max(1, P.check_every);
      int cps = 0;
      for (int i = 0; i < len; ++i) if ((i + 1) % ce == 0 || i + 1 == len) ++cps;
      n += 4LL * cps;
    }
    return n;
  }
  int launch_run_chunk() {
    const int len = run_chunk_len();
    if (P.use_graphs) {
      if (!g_run || g_run_len != len) {
        if (g_run) cudaGraphExecDestroy(g_run);
        g_run = nullptr;
        ESR_TRY(capture(true, len, &g_run));
        g_run_len = len;
      }
      ESR_CUDA(cudaGraphLaunch(g_run, stream));
      launches += chunk_launches(true, len);
    } else {
      issue_run_chunk(len);
    }
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }

  // ------------------------------------------------------------- case setup
  int set_case(int slot, const esr_case* c, const double* W_init, bool defer_dt = false) {
    int m, b;
    ESR_TRY(mesh_of_slot(slot, m, b));
    if (!c) return fail(ESR_ERR_ARG, "set_case: null case");
    if (!(c->tf > 0) && c->max_steps <= 0) return fail(ESR_ERR_ARG, "set_case: tf must be > 0");
    if (!(c->cfl > 0)) return fail(ESR_ERR_ARG, "set_case: cfl must be > 0");
    MeshDev& md = *meshes[m];
    const HostMesh& hm = *md.hm;
    const int N = hm.n_cells;
    // per-slot constants: inlet, sponge strength (helper.py:279-285), force reference
    const V in = mk4<T>((T)c->inlet[0], (T)c->inlet[1], (T)c->inlet[2], (T)c->inlet[3]);
    const T r = in.x, u = in.y / r, v = in.z / r;
    const T p = (in.w - kc.half * r * (u * u + v * v)) * kc.gm1;
    const T U = std::sqrt(u * u + v * v);
    const T a = std::sqrt(kc.gamma * p / r);
    const T Ly = (T)hm.y_max - (T)hm.y_min;   // helper.py:271-277 in the state precision
    const T wdt = (T)0.2 * Ly;
    T str = (T)1.0 * (U + a) / wdt;
    if (!(std::isfinite((double)str))) str = T(0);
    const double cflv = c->cfl;
    const double tfv = c->tf;
    const long long ms = c->max_steps;
    const double q = 0.5 * c->rho_inf * c->u_inf * c->u_inf * c->l_ref;
    const double qv = q > 0 ? q : 1.0;
    ESR_CUDA(cudaMemcpyAsync(inlet.p + slot, &in, sizeof(V), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(strength.p + slot, &str, sizeof(T), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(cfl.p + slot, &cflv, sizeof(double), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(tf.p + slot, &tfv, sizeof(double), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(max_steps.p + slot, &ms, sizeof(long long), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(qref.p + slot, &qv, sizeof(double), cudaMemcpyHostToDevice, stream));
    // engineering criterion: relative tolerances of euler/main.py:72-73
    const int etrack = c->eng_track ? 1 : 0;
    const int epat = std::max(1, c->eng_patience > 0 ? c->eng_patience : P.patience);
    const double4 et = make_double4(c->eng_target_cd, c->eng_target_cl,
                                    c->eng_cd_tol * std::max(std::fabs(c->eng_target_cd), 1e-8),
                                    c->eng_cl_tol * std::max(std::fabs(c->eng_target_cl), 1e-8));
    ESR_CUDA(cudaMemcpyAsync(eng_track.p + slot, &etrack, sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(eng_patience.p + slot, &epat, sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(eng_t.p + slot, &et, sizeof(double4), cudaMemcpyHostToDevice, stream));
    const double th = c->threshold;
    ESR_CUDA(cudaMemcpyAsync(thr.p + slot, &th, sizeof(double), cudaMemcpyHostToDevice, stream));
    const int tb = 256, nb = (N + tb - 1) / tb;
    if (W_init) {
      if (stage_rows.n < (size_t)4 * N) ESR_TRY(stage_rows.alloc((size_t)4 * N));
      ESR_CUDA(cudaMemcpyAsync(stage_rows.p, W_init, (size_t)4 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
      k_scatter_state<T><<<nb, tb, 0, stream>>>(stage_rows.p, md.inv.p, N, W.p, Wref.p, md.off, md.B, b);
    } else {
      k_fill_freestream<T><<<nb, tb, 0, stream>>>(W.p, Wref.p, N, md.off, md.B, b, in);
    }
    launches += 1;
    return reset_slot(slot, defer_dt);
  }
  // counters to zero; dt and N from the slot's current state (now, or with the
  // next flush_fills when deferred so many refills share one reduction)
  std::vector<int> pending_fill;
  int reset_slot(int slot, bool defer = false) {
    const int one = 1, zero = 0;
    for (DevBuf<int>* bfr : {&step, &ref_step, &streak, &streak_start, &stopping, &due})
      ESR_CUDA(cudaMemcpyAsync(bfr->p + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(status.p + slot, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(active.p + slot, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    const double inf = INFINITY;
    ESR_CUDA(cudaMemcpyAsync(last_rel.p + slot, &inf, sizeof(double), cudaMemcpyHostToDevice, stream));
    if (pending_fill.size() != (size_t)n_slots) pending_fill.assign(n_slots, 0);
    pending_fill[slot] = 1;
    return defer ? ESR_OK : flush_fills();
  }
  int flush_fills() {
    if (pending_fill.size() != (size_t)n_slots) return ESR_OK;
    bool any = false;
    for (int v : pending_fill) any |= v != 0;
    if (!any) return ESR_OK;
    ESR_CUDA(cudaMemcpyAsync(fill.p, pending_fill.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_TRY(finish_fill());
    ESR_CUDA(cudaStreamSynchronize(stream));  // pending_fill is reused as the copy source
    std::fill(pending_fill.begin(), pending_fill.end(), 0);
    return ESR_OK;
  }
  // dt + N for every slot flagged in `fill` (one reduction launch for all)
  int finish_fill() {
    dtmin_reduce(fill.p);
    const int tb = 128, nb = (n_slots + tb - 1) / tb;
    k_dt_finish<T><<<nb, tb, 0, stream>>>(fill.p, n_slots, partial.p, n_chunks, cfl.p, tf.p, max_steps.p, dt.p, ctl(),
                                          P.dt_mode == ESR_DT_LOCAL);
    k_forces<T><<<n_slots, 256, 0, stream>>>(d_segs.p, cmap(), W.p, qref.p, forces.p, kc, fill.p, eng_track.p);
    k_eng_init<<<nb, tb, 0, stream>>>(ctl(), fill.p, n_slots);
    launches += 4;
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }
  // ---------------------------------------------- many slots at once
  DevBuf<double> stage_many;            // host rows of set_cases / get_states
  DevBuf<SlotInit<T>> d_init;
  DevBuf<SlotCopy<T>> d_jobs;

  // ------------------------------ overlapped transfers (float32 host fields)
  // The next cases' fields go up on a copy stream while the current chunk
  // runs (stage_in), are placed by one launch on the solver's stream
  // (apply_staged); final fields are gathered on the solver's stream and go
  // down on the copy stream while the next chunk runs (fetch_states). Events
  // order the two streams: a staging buffer is rewritten only after the
  // launches that read it have run.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_in_ready = nullptr, ev_in_consumed = nullptr, ev_out_ready = nullptr, ev_out_done = nullptr;
  DevBuf<float> st_in, st_out;
  DevBuf<SlotInit<T>> st_init;
  DevBuf<SlotCopy<T>> st_jobs_in, st_jobs_out;
  PinnedBuf<SlotInit<T>> h_init;
  PinnedBuf<SlotCopy<T>> h_jobs_in, h_jobs_out;
  int staged_n = 0, staged_max = 0;
  std::vector<int> staged_slots;
  int transfer_setup() {
    if (copy_stream) return ESR_OK;
    ESR_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&ev_in_ready, &ev_in_consumed, &ev_out_ready, &ev_out_done})
      ESR_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return ESR_OK;
  }
  int stage_in(int n, const int32_t* slots, const esr_case* cs, const float* const* W_init) {
    if (n <= 0 || !slots || !cs || !W_init) return fail(ESR_ERR_ARG, "stage_cases: bad arguments");
    ESR_TRY(transfer_setup());
    std::vector<char> seen(n_slots, 0);
    long long rows = 0;
    int max_n = 0;
    // everything is checked before the staging buffers change
    for (int i = 0; i < n; ++i) {
      int m, b;
      ESR_TRY(mesh_of_slot(slots[i], m, b));
      if (seen[slots[i]]) return fail(ESR_ERR_ARG, "stage_cases: a slot is listed twice");
      seen[slots[i]] = 1;
      if (!W_init[i]) return fail(ESR_ERR_ARG, "stage_cases: null field");
      if (!(cs[i].tf > 0) && cs[i].max_steps <= 0) return fail(ESR_ERR_ARG, "stage_cases: tf must be > 0");
      if (!(cs[i].cfl > 0)) return fail(ESR_ERR_ARG, "stage_cases: cfl must be > 0");
      rows += meshes[m]->hm->n_cells;
      max_n = std::max(max_n, meshes[m]->hm->n_cells);
    }
    // the previous staging's copies have finished: its host tables are free
    ESR_CUDA(cudaEventSynchronize(ev_in_ready));
    ESR_TRY(h_init.reserve(n));
    ESR_TRY(h_jobs_in.reserve(n));
    if (st_in.n < (size_t)4 * rows) ESR_TRY(st_in.alloc((size_t)4 * rows));
    if (st_init.n < (size_t)n) ESR_TRY(st_init.alloc(n));
    if (st_jobs_in.n < (size_t)n) ESR_TRY(st_jobs_in.alloc(n));
    long long row = 0;
    for (int i = 0; i < n; ++i) {
      int m, b;
      mesh_of_slot(slots[i], m, b);
      esr_case c = cs[i];
      c.mesh = m;
      SlotInit<T>& x = h_init.p[i];
      x = SlotInit<T>{};
      x.slot = slots[i];
      case_params(c, x.inlet, x.strength, x.qref, x.eng_t, x.eng_track, x.eng_pat);
      x.cfl = c.cfl;
      x.tf = c.tf;
      x.thr = c.threshold;
      x.max_steps = c.max_steps;
      MeshDev& md = *meshes[m];
      h_jobs_in.p[i] = SlotCopy<T>{row, md.inv.p, md.off, md.hm->n_cells, md.B, b, 0, x.inlet};
      row += md.hm->n_cells;
    }
    // the device staging is rewritten once the last placement has read it
    ESR_CUDA(cudaStreamWaitEvent(copy_stream, ev_in_consumed, 0));
    ESR_CUDA(cudaMemcpyAsync(st_init.p, h_init.p, n * sizeof(SlotInit<T>), cudaMemcpyHostToDevice, copy_stream));
    ESR_CUDA(cudaMemcpyAsync(st_jobs_in.p, h_jobs_in.p, n * sizeof(SlotCopy<T>), cudaMemcpyHostToDevice, copy_stream));
    // one copy per run of fields that lie back to back in host memory (the
    // staging rows are consecutive), so a caller with one block for all its
    // fields pays one copy's launch cost, not one per case
    for (int i = 0; i < n;) {
      int j = i + 1;
      size_t len = (size_t)4 * h_jobs_in.p[i].n_cells;
      while (j < n && W_init[j] == W_init[i] + len) len += (size_t)4 * h_jobs_in.p[j++].n_cells;
      ESR_CUDA(cudaMemcpyAsync(st_in.p + 4 * h_jobs_in.p[i].stage_row, W_init[i], len * sizeof(float),
                               cudaMemcpyHostToDevice, copy_stream));
      i = j;
    }
    ESR_CUDA(cudaEventRecord(ev_in_ready, copy_stream));
    staged_n = n;
    staged_max = max_n;
    staged_slots.assign(slots, slots + n);
    return ESR_OK;
  }
  int apply_staged() {
    if (staged_n <= 0) return fail(ESR_ERR_STATE, "apply_staged: nothing staged");
    ESR_CUDA(cudaStreamWaitEvent(stream, ev_in_ready, 0));
    ESR_CUDA(cudaMemsetAsync(fill.p, 0, n_slots * sizeof(int), stream));
    SlotParams<T> sp{dt.p, inlet.p, strength.p, cfl.p, tf.p, max_steps.p, qref.p, eng_track.p, eng_patience.p, eng_t.p, thr.p};
    k_init_slots<T><<<(staged_n + 127) / 128, 128, 0, stream>>>(st_init.p, staged_n, sp, ctl(), fill.p);
    ++launches;
    for (int j0 = 0; j0 < staged_n; j0 += 65535) {
      const int nj = std::min(65535, staged_n - j0);
      k_scatter_slots<T, float><<<dim3((staged_max + 255) / 256, nj), 256, 0, stream>>>(st_in.p, st_jobs_in.p + j0, W.p,
                                                                                        Wref.p);
      ++launches;
    }
    ESR_TRY(finish_fill());
    ESR_CUDA(cudaEventRecord(ev_in_consumed, stream));
    for (int g : staged_slots) hcase_index[g] = g;
    staged_n = 0;
    return ESR_OK;
  }
  int fetch_states(int n, const int32_t* slots, float* const* out) {
    if (n <= 0 || !slots || !out) return fail(ESR_ERR_ARG, "fetch_states: bad arguments");
    ESR_TRY(transfer_setup());
    long long rows = 0;
    int max_n = 0;
    for (int i = 0; i < n; ++i) {
      int m, b;
      ESR_TRY(mesh_of_slot(slots[i], m, b));
      if (!out[i]) return fail(ESR_ERR_ARG, "fetch_states: null output");
      rows += meshes[m]->hm->n_cells;
      max_n = std::max(max_n, meshes[m]->hm->n_cells);
    }
    // the previous download has finished: the gather staging and its table are free
    ESR_CUDA(cudaEventSynchronize(ev_out_done));
    ESR_TRY(h_jobs_out.reserve(n));
    if (st_out.n < (size_t)4 * rows) ESR_TRY(st_out.alloc((size_t)4 * rows));
    if (st_jobs_out.n < (size_t)n) ESR_TRY(st_jobs_out.alloc(n));
    long long row = 0;
    for (int i = 0; i < n; ++i) {
      int m, b;
      mesh_of_slot(slots[i], m, b);
      MeshDev& md = *meshes[m];
      h_jobs_out.p[i] = SlotCopy<T>{row, md.inv.p, md.off, md.hm->n_cells, md.B, b, 0, V{}};
      row += md.hm->n_cells;
    }
    ESR_CUDA(cudaMemcpyAsync(st_jobs_out.p, h_jobs_out.p, n * sizeof(SlotCopy<T>), cudaMemcpyHostToDevice, stream));
    for (int j0 = 0; j0 < n; j0 += 65535) {
      const int nj = std::min(65535, n - j0);
      k_gather_slots<T, float><<<dim3((max_n + 255) / 256, nj), 256, 0, stream>>>(W.p, st_jobs_out.p + j0, st_out.p);
      ++launches;
    }
    ESR_CUDA(cudaEventRecord(ev_out_ready, stream));
    ESR_CUDA(cudaStreamWaitEvent(copy_stream, ev_out_ready, 0));
    for (int i = 0; i < n;) {   // one copy per run of back-to-back outputs, as in stage_in
      int j = i + 1;
      size_t len = (size_t)4 * h_jobs_out.p[i].n_cells;
      while (j < n && out[j] == out[i] + len) len += (size_t)4 * h_jobs_out.p[j++].n_cells;
      ESR_CUDA(cudaMemcpyAsync(out[i], st_out.p + 4 * h_jobs_out.p[i].stage_row, len * sizeof(float),
                               cudaMemcpyDeviceToHost, copy_stream));
      i = j;
    }
    ESR_CUDA(cudaEventRecord(ev_out_done, copy_stream));
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }
  int wait_transfers() {
    if (!copy_stream) return ESR_OK;
    ESR_CUDA(cudaEventSynchronize(ev_in_ready));
    ESR_CUDA(cudaEventSynchronize(ev_out_done));
    return ESR_OK;
  }
  // Upload the slot table and launch fn(table, grid) once per 65,535 slots
  // (the grid's y limit); grid.x covers the largest mesh. The caller
  // synchronises the stream before the host table goes.
  template <typename F>
  int launch_slot_copies(const std::vector<SlotCopy<T>>& jobs, int max_n, F&& fn) {
    const int n = (int)jobs.size();
    if (n == 0 || max_n == 0) return ESR_OK;
    if (d_jobs.n < (size_t)n) ESR_TRY(d_jobs.alloc(n));
    ESR_CUDA(cudaMemcpyAsync(d_jobs.p, jobs.data(), n * sizeof(SlotCopy<T>), cudaMemcpyHostToDevice, stream));
    for (int j0 = 0; j0 < n; j0 += 65535) {
      const int nj = std::min(65535, n - j0);
      fn(d_jobs.p + j0, dim3((max_n + 255) / 256, nj));
      ++launches;
    }
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }
  // S: the type of the caller's host rows (double, or float for float32 fields)
  template <typename S>
  int set_cases(int n, const int32_t* slots, const esr_case* cs, const S* const* W_init) {
    if (n < 0 || (n > 0 && (!slots || !cs))) return fail(ESR_ERR_ARG, "set_cases: bad arguments");
    if (n == 0) return ESR_OK;
    std::vector<SlotInit<T>> hi(n);
    std::vector<char> seen(n_slots, 0);
    std::vector<long long> off(n, -1);
    long long rows = 0;
    for (int i = 0; i < n; ++i) {
      int m, b;
      ESR_TRY(mesh_of_slot(slots[i], m, b));
      if (seen[slots[i]]) return fail(ESR_ERR_ARG, "set_cases: a slot is listed twice");
      seen[slots[i]] = 1;
      esr_case c = cs[i];
      c.mesh = m;   // the slot decides the mesh, as in esr_set_case
      if (!(c.tf > 0) && c.max_steps <= 0) return fail(ESR_ERR_ARG, "set_cases: tf must be > 0");
      if (!(c.cfl > 0)) return fail(ESR_ERR_ARG, "set_cases: cfl must be > 0");
      SlotInit<T>& x = hi[i];
      x.slot = slots[i];
      case_params(c, x.inlet, x.strength, x.qref, x.eng_t, x.eng_track, x.eng_pat);
      x.cfl = c.cfl;
      x.tf = c.tf;
      x.thr = c.threshold;
      x.max_steps = c.max_steps;
      if (W_init && W_init[i]) { off[i] = rows; rows += meshes[m]->hm->n_cells; }
    }
    // every case is valid: only now does the host bookkeeping change
    for (int i = 0; i < n; ++i) hcase_index[slots[i]] = slots[i];
    if (rows > 0 && stage_many.n < (size_t)4 * rows) ESR_TRY(stage_many.alloc((size_t)4 * rows));
    S* stage = reinterpret_cast<S*>(stage_many.p);   // room for 4 rows of doubles is room for floats
    if (d_init.n < (size_t)n) ESR_TRY(d_init.alloc(n));
    ESR_CUDA(cudaMemcpyAsync(d_init.p, hi.data(), n * sizeof(SlotInit<T>), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemsetAsync(fill.p, 0, n_slots * sizeof(int), stream));
    SlotParams<T> sp{dt.p, inlet.p, strength.p, cfl.p, tf.p, max_steps.p, qref.p, eng_track.p, eng_patience.p, eng_t.p, thr.p};
    k_init_slots<T><<<(n + 127) / 128, 128, 0, stream>>>(d_init.p, n, sp, ctl(), fill.p);
    ++launches;
    // every field lands in the staging rows first, then one launch places them all
    std::vector<SlotCopy<T>> jobs(n);
    int max_n = 0;
    for (int i = 0; i < n; ++i) {
      int m, b;
      ESR_TRY(mesh_of_slot(slots[i], m, b));
      MeshDev& md = *meshes[m];
      const int N = md.hm->n_cells;
      if (off[i] >= 0)
        ESR_CUDA(cudaMemcpyAsync(stage + 4 * off[i], W_init[i], (size_t)4 * N * sizeof(S), cudaMemcpyHostToDevice, stream));
      jobs[i] = SlotCopy<T>{off[i] >= 0 ? off[i] : -1, md.inv.p, md.off, N, md.B, b, 0, hi[i].inlet};
      max_n = std::max(max_n, N);
    }
    ESR_TRY(launch_slot_copies(jobs, max_n, [&](const SlotCopy<T>* dj, dim3 grid) {
      k_scatter_slots<T, S><<<grid, 256, 0, stream>>>(stage, dj, W.p, Wref.p);
    }));
    ESR_TRY(finish_fill());
    ESR_CUDA(cudaStreamSynchronize(stream));   // hi and the caller's fields are the copy sources
    return ESR_OK;
  }
  template <typename S>
  int get_states(int n, const int32_t* slots, S* const* out) {
    if (n < 0 || (n > 0 && (!slots || !out))) return fail(ESR_ERR_ARG, "get_states: bad arguments");
    long long rows = 0;
    std::vector<long long> off(n);
    for (int i = 0; i < n; ++i) {
      int m, b;
      ESR_TRY(mesh_of_slot(slots[i], m, b));
      if (!out[i]) return fail(ESR_ERR_ARG, "get_states: null output");
      off[i] = rows;
      rows += meshes[m]->hm->n_cells;
    }
    if (rows > 0 && stage_many.n < (size_t)4 * rows) ESR_TRY(stage_many.alloc((size_t)4 * rows));
    S* stage = reinterpret_cast<S*>(stage_many.p);
    // one launch stages every slot's rows, then one copy per slot
    std::vector<SlotCopy<T>> jobs(n);
    int max_n = 0;
    for (int i = 0; i < n; ++i) {
      int m, b;
      ESR_TRY(mesh_of_slot(slots[i], m, b));
      MeshDev& md = *meshes[m];
      jobs[i] = SlotCopy<T>{off[i], md.inv.p, md.off, md.hm->n_cells, md.B, b, 0, V{}};
      max_n = std::max(max_n, md.hm->n_cells);
    }
    ESR_TRY(launch_slot_copies(jobs, max_n, [&](const SlotCopy<T>* dj, dim3 grid) {
      k_gather_slots<T, S><<<grid, 256, 0, stream>>>(W.p, dj, stage);
    }));
    for (int i = 0; i < n; ++i)
      ESR_CUDA(cudaMemcpyAsync(out[i], stage + 4 * off[i], (size_t)4 * jobs[i].n_cells * sizeof(S),
                               cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    return ESR_OK;
  }
  int clear_slot(int slot) {
    int m, b;
    ESR_TRY(mesh_of_slot(slot, m, b));
    const int zero = 0;
    ESR_CUDA(cudaMemcpyAsync(active.p + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(status.p + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
    hcase_index[slot] = -1;
    return ESR_OK;
  }
  // A caller's device state buffer is read or written by a kernel as 4-value
  // vectors, so it must be memory of this solver's GPU (or managed memory)
  // aligned for them; a host address or another GPU's memory is an argument
  // error here, before any launch.
  int check_state_ptr(const void* p, const char* what) {
    cudaPointerAttributes a{};
    ESR_CUDA(cudaPointerGetAttributes(&a, p));
    const bool dev = (a.type == cudaMemoryTypeDevice && a.device == device) || a.type == cudaMemoryTypeManaged;
    if (!dev) return fail(ESR_ERR_ARG, std::string(what) + ": not device memory of the solver's GPU");
    if ((uintptr_t)p % alignof(V) != 0)
      return fail(ESR_ERR_ARG, std::string(what) + ": state must be aligned to " + std::to_string(alignof(V)) + " bytes");
    return ESR_OK;
  }
  int set_state(int slot, const double* Wh, bool device_src) {
    int m, b;
    ESR_TRY(mesh_of_slot(slot, m, b));
    MeshDev& md = *meshes[m];
    const int N = md.hm->n_cells, tb = 256, nb = (N + tb - 1) / tb;
    if (device_src) {
      ESR_TRY(check_state_ptr(Wh, "set_state_device"));
      k_copy_in_device<T><<<nb, tb, 0, stream>>>((const V*)Wh, md.inv.p, N, W.p, Wref.p, md.off, md.B, b);
    } else {
      if (stage_rows.n < (size_t)4 * N) ESR_TRY(stage_rows.alloc((size_t)4 * N));
      ESR_CUDA(cudaMemcpyAsync(stage_rows.p, Wh, (size_t)4 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
      k_scatter_state<T><<<nb, tb, 0, stream>>>(stage_rows.p, md.inv.p, N, W.p, Wref.p, md.off, md.B, b);
    }
    ++launches;
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }
  int get_state(int slot, double* Wh, bool device_dst) {
    int m, b;
    ESR_TRY(mesh_of_slot(slot, m, b));
    MeshDev& md = *meshes[m];
    const int N = md.hm->n_cells, tb = 256, nb = (N + tb - 1) / tb;
    if (device_dst) {
      ESR_TRY(check_state_ptr(Wh, "get_state_device"));
      k_copy_out_device<T><<<nb, tb, 0, stream>>>(W.p, md.inv.p, N, md.off, md.B, b, (V*)Wh);
      ++launches;
      ESR_CUDA(cudaGetLastError());
      return ESR_OK;
    }
    if (stage_rows.n < (size_t)4 * N) ESR_TRY(stage_rows.alloc((size_t)4 * N));
    k_gather_state<T><<<nb, tb, 0, stream>>>(W.p, md.inv.p, N, md.off, md.B, b, stage_rows.p);
    ++launches;
    ESR_CUDA(cudaMemcpyAsync(Wh, stage_rows.p, (size_t)4 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    return ESR_OK;
  }

  // ----------------------------------------------------------------- runs
  int step_n(int nsteps) {
    if (nsteps < 0) return fail(ESR_ERR_ARG, "step: nsteps < 0");
    ESR_CUDA(cudaEventRecord(ev0, stream));
    int left = nsteps;
    const int L = 32;
    while (left > 0) {
      const int len = std::min(left, L);
      if (P.use_graphs && len == L) {
        if (!g_plain || g_plain_len != L) {
          if (g_plain) cudaGraphExecDestroy(g_plain);
          g_plain = nullptr;
          ESR_TRY(capture(false, L, &g_plain));
          g_plain_len = L;
        }
        ESR_CUDA(cudaGraphLaunch(g_plain, stream));
        launches += chunk_launches(false, L);
      } else {
        issue_plain_chunk(len);
      }
      left -= len;
    }
    ESR_CUDA(cudaEventRecord(ev1, stream));
    ESR_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    last_ms = ms;
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }
  int any_active(int& n_live, std::vector<int>* st = nullptr) {
    std::vector<int> a(n_slots);
    ESR_CUDA(cudaMemcpyAsync(a.data(), active.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    if (st) { st->resize(n_slots); ESR_CUDA(cudaMemcpyAsync(st->data(), status.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream)); }
    ESR_CUDA(cudaStreamSynchronize(stream));
    n_live = 0;
    for (int v : a) n_live += v != 0;
    return ESR_OK;
  }
  int run_all(esr_result* res) {
    ESR_CUDA(cudaEventRecord(ev0, stream));
    int live = 0;
    ESR_TRY(any_active(live));
    int poll = 2;
    while (live > 0) {
      for (int i = 0; i < poll; ++i) ESR_TRY(launch_run_chunk());
      ESR_TRY(any_active(live));
      poll = std::min(poll * 2, 16);
    }
    ESR_CUDA(cudaEventRecord(ev1, stream));
    ESR_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    last_ms = ms;
    if (res) ESR_TRY(results(res));
    return ESR_OK;
  }
  int compute_forces() {
    k_forces<T><<<n_slots, 256, 0, stream>>>(d_segs.p, cmap(), W.p, qref.p, forces.p, kc, nullptr, nullptr);
    ++launches;
    ESR_CUDA(cudaGetLastError());
    return ESR_OK;
  }
  int results(esr_result* out) {
    ESR_TRY(compute_forces());
    std::vector<int> st(n_slots), stp(n_slots), nm(n_slots), sstep(n_slots);
    std::vector<double> lr(n_slots), fo(2 * n_slots);
    std::vector<T> d(n_slots);
    std::vector<long long> ts(n_slots), te(n_slots);
    ESR_CUDA(cudaMemcpyAsync(st.data(), status.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(stp.data(), step.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(nm.data(), nmax.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(sstep.data(), stopping.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(lr.data(), last_rel.p, n_slots * sizeof(double), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(fo.data(), forces.p, 2 * n_slots * sizeof(double), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(d.data(), dt.p, n_slots * sizeof(T), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(ts.data(), t_start.p, n_slots * sizeof(long long), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(te.data(), t_end.p, n_slots * sizeof(long long), cudaMemcpyDeviceToHost, stream));
    std::vector<int> etr(n_slots), est(n_slots), esp(n_slots);
    ESR_CUDA(cudaMemcpyAsync(etr.data(), eng_track.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(est.data(), eng_stop.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(esp.data(), eng_stopping.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    for (int g = 0; g < n_slots; ++g) {
      esr_result& r = out[g];
      r.eng_converged = etr[g] ? est[g] : 0;
      r.eng_stopping_step = etr[g] ? (est[g] ? esp[g] : nm[g]) : 0;
      r.status = st[g];
      r.converged = st[g] == ESR_CASE_CONVERGED;
      r.stopping_step = (st[g] == ESR_CASE_CONVERGED || st[g] == ESR_CASE_MAXSTEP || st[g] == ESR_CASE_NONFINITE) ? sstep[g] : nm[g];
      r.steps = stp[g];
      r.n_max = nm[g];
      r.case_index = hcase_index[g];
      r.dt = P.dt_mode == ESR_DT_LOCAL ? 0.0 : (double)d[g];
      r.last_rel = lr[g];
      r.cd = fo[2 * g];
      r.cl = fo[2 * g + 1];
      r.solve_time_s = (te[g] > ts[g] && st[g] >= ESR_CASE_CONVERGED) ? (double)(te[g] - ts[g]) * 1e-9 : 0.0;
    }
    return ESR_OK;
  }
  DevBuf<V> probe_save;      // residual probe: the state it restores
  DevBuf<double> grad_out;   // gradient export
  int residual_probe(double* rel) {
    // one step of every running slot from the current state without keeping it
    // (euler/main.py:228-230): ||W_probe - W|| / (||W|| + 1e-16)
    DevBuf<V>& save = probe_save;
    ESR_TRY(save.reserve(total));
    ESR_CUDA(cudaMemcpyAsync(save.p, W.p, total * sizeof(V), cudaMemcpyDeviceToDevice, stream));
    std::vector<int> act(n_slots), st(n_slots);
    ESR_CUDA(cudaMemcpyAsync(act.data(), active.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(st.data(), status.p, n_slots * sizeof(int), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    std::vector<int> on(n_slots);
    for (int g = 0; g < n_slots; ++g) on[g] = st[g] != ESR_CASE_EMPTY;
    ESR_CUDA(cudaMemcpyAsync(active.p, on.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    step_kernels(cases(true), 0);
    ESR_CUDA(cudaMemcpyAsync(due.p, on.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    dim3 grid(n_chunks, n_slots);
    k_case_reduce<T, RED_DIFF><<<grid, kReduceThreads, 0, stream>>>(d_segs.p, cmap(), W.p, save.p, due.p, kReduceCells,
                                                                    partial.p, n_chunks, kc);
    ++launches;
    std::vector<double2> pt((size_t)n_slots * n_chunks);
    ESR_CUDA(cudaMemcpyAsync(pt.data(), partial.p, pt.size() * sizeof(double2), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaMemcpyAsync(W.p, save.p, total * sizeof(V), cudaMemcpyDeviceToDevice, stream));
    ESR_CUDA(cudaMemcpyAsync(active.p, act.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    for (int g = 0; g < n_slots; ++g) {
      double s0 = 0, s1 = 0;
      for (int i = 0; i < n_chunks; ++i) { s0 += pt[(size_t)g * n_chunks + i].x; s1 += pt[(size_t)g * n_chunks + i].y; }
      rel[g] = on[g] ? std::sqrt(s0) / (std::sqrt(s1) + 1e-16) : 0.0;
    }
    return ESR_OK;
  }
  int gradients(int slot, double* out) {
    int m, b;
    ESR_TRY(mesh_of_slot(slot, m, b));
    MeshDev& md = *meshes[m];
    const int N = md.hm->n_cells, tb = 128, nb = (N + tb - 1) / tb;
    DevBuf<double>& g = grad_out;
    ESR_TRY(g.reserve((size_t)8 * N));
    k_grad_export<T><<<nb, tb, 0, stream>>>(d_segs.p, m, b, W.p, inlet.p, md.inv.p, slot, kc, g.p);
    ++launches;
    ESR_CUDA(cudaGetLastError());
    ESR_CUDA(cudaMemcpyAsync(out, g.p, (size_t)8 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    return ESR_OK;
  }
  int entropy(double* S) {
    std::vector<int> on(n_slots, 1);
    ESR_CUDA(cudaMemcpyAsync(due.p, on.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    dim3 grid(n_chunks, n_slots);
    k_case_reduce<T, RED_ENTROPY><<<grid, kReduceThreads, 0, stream>>>(d_segs.p, cmap(), W.p, nullptr, due.p, kReduceCells,
                                                                       partial.p, n_chunks, kc);
    ++launches;
    std::vector<double2> pt((size_t)n_slots * n_chunks);
    ESR_CUDA(cudaMemcpyAsync(pt.data(), partial.p, pt.size() * sizeof(double2), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    for (int g = 0; g < n_slots; ++g) {
      double s0 = 0;
      for (int i = 0; i < n_chunks; ++i) s0 += pt[(size_t)g * n_chunks + i].x;
      S[g] = s0;
    }
    return ESR_OK;
  }
  int dts(double* out) {
    std::vector<T> d(n_slots);
    ESR_CUDA(cudaMemcpyAsync(d.data(), dt.p, n_slots * sizeof(T), cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    for (int g = 0; g < n_slots; ++g) out[g] = (double)d[g];
    return ESR_OK;
  }

  // ------------------------------------------- batch with retire / refill
  // Per-case slot parameters (the same values set_case uploads for one slot).
  void case_params(const esr_case& c, V& in, T& str, double& q, double4& et, int& etrack, int& epat) {
    const HostMesh& hm = *meshes[c.mesh]->hm;
    in = mk4<T>((T)c.inlet[0], (T)c.inlet[1], (T)c.inlet[2], (T)c.inlet[3]);
    const T r = in.x, u = in.y / r, v = in.z / r;
    const T p = (in.w - kc.half * r * (u * u + v * v)) * kc.gm1;
    const T U = std::sqrt(u * u + v * v), a = std::sqrt(kc.gamma * p / r);
    const T Ly = (T)hm.y_max - (T)hm.y_min;
    str = (T)1.0 * (U + a) / ((T)0.2 * Ly);
    if (!(std::isfinite((double)str))) str = T(0);
    const double qq = 0.5 * c.rho_inf * c.u_inf * c.u_inf * c.l_ref;
    q = qq > 0 ? qq : 1.0;
    etrack = c.eng_track ? 1 : 0;
    epat = std::max(1, c.eng_patience > 0 ? c.eng_patience : P.patience);
    et = make_double4(c.eng_target_cd, c.eng_target_cl, c.eng_cd_tol * std::max(std::fabs(c.eng_target_cd), 1e-8),
                      c.eng_cl_tol * std::max(std::fabs(c.eng_target_cl), 1e-8));
  }

  // The queue lives on the device: every captured chunk of steps ends with
  // the refill sequence (retire -> assign -> fill -> dt), so the host only
  // polls the done counter.
  struct BatchBufs {
    DevBuf<int> qlist, qoff, qhead, slot_case, retiring, c_eng_track, c_eng_pat, r_status, r_stop, r_steps, r_nmax,
        r_eng_conv, r_eng_stop, n_done;
    DevBuf<V> c_inlet;
    DevBuf<T> c_strength;
    DevBuf<double> c_cfl, c_tf, c_qref, c_thr, r_dt, r_rel, r_cd, r_cl, r_time, r_probe, init, out;
    DevBuf<long long> c_max_steps, init_off, out_off;
    DevBuf<double4> c_eng_t;
  };
  DevBuf<int> perm_all, move_src;
  DevBuf<const int*> perm_ptrs, inv_ptrs;

  void issue_refill(const Queue<T>& q, const SlotParams<T>& sp, bool with_states) {
    const int tb = 128, nb = (n_slots + tb - 1) / tb;
    k_mark_retiring<<<nb, tb, 0, stream>>>(status.p, n_slots, q.slot_case, q.retiring);
    k_forces<T><<<n_slots, 256, 0, stream>>>(d_segs.p, cmap(), W.p, qref.p, forces.p, kc, q.retiring, nullptr);
    k_retire<T><<<nb, tb, 0, stream>>>(ctl(), q, dt.p, forces.p, n_slots, P.dt_mode == ESR_DT_LOCAL);
    // final one-step residual of each retiring case with its own dt
    Cases<T> pc = cases(true);
    pc.active = q.retiring;
    const V* wp = probe_kernels(pc);
    dim3 gr(n_chunks, n_slots);
    k_case_reduce<T, RED_DIFF><<<gr, kReduceThreads, 0, stream>>>(d_segs.p, cmap(), wp, W.p, q.retiring, kReduceCells,
                                                                  partial.p, n_chunks, kc);
    k_probe_finish<T><<<nb, tb, 0, stream>>>(q, partial.p, n_chunks, n_slots);
    int max_cells = 0;
    for (auto& md : meshes) max_cells = std::max(max_cells, md->hm->n_cells);
    dim3 g2(std::min(64, (max_cells + 255) / 256), n_slots);
    if (with_states) k_retire_states<T><<<g2, 256, 0, stream>>>(d_segs.p, cmap(), q, W.p, inv_ptrs.p);
    k_assign<T><<<(int)(meshes.size() + 31) / 32, 32, 0, stream>>>(d_segs.p, (int)meshes.size(), q, sp, ctl(), fill.p);
    k_fill_slots<T><<<g2, 256, 0, stream>>>(d_segs.p, cmap(), q, fill.p, perm_ptrs.p, W.p, Wref.p);
    dtmin_reduce(fill.p);
    k_dt_finish<T><<<nb, tb, 0, stream>>>(fill.p, n_slots, partial.p, n_chunks, cfl.p, tf.p, max_steps.p, dt.p, ctl(),
                                          P.dt_mode == ESR_DT_LOCAL);
    k_forces<T><<<n_slots, 256, 0, stream>>>(d_segs.p, cmap(), W.p, qref.p, forces.p, kc, fill.p, eng_track.p);
    k_eng_init<<<nb, tb, 0, stream>>>(ctl(), fill.p, n_slots);
    // pack running cases into the lowest slots once a mesh's queue is empty
    k_compact_plan<T><<<(int)(meshes.size() + 31) / 32, 32, 0, stream>>>(d_segs.p, (int)meshes.size(), q, move_src.p,
                                                                         d_live.p);
    k_compact_items<T><<<g2, 256, 0, stream>>>(d_segs.p, cmap(), move_src.p, W.p, Wref.p);
    k_compact_slots<T><<<nb, tb, 0, stream>>>(move_src.p, n_slots, q, sp, ctl(), forces.p);
    launches += with_states ? 15 : 14;
  }

  // A batch in flight: its queue and result buffers, the captured chunk graph
  // and the host's polling state, held between esr_batch_submit and
  // esr_batch_results (esr_batch_solve runs the three steps in one call).
  BatchBufs batch_bufs;   // reused by every batch (one pending at a time)
  struct PendingBatch {
    BatchBufs* Bp = nullptr;
    Queue<T> q{};
    SlotParams<T> sp{};
    std::vector<int> case_mesh;
    std::vector<long long> out_off;
    int n = 0;
    bool want_states = false;
    cudaGraphExec_t gexec = nullptr;
    cudaGraphExec_t gexec_tail = nullptr;   // the same chunk with K2 per cell (K2 by patches solvers)
    bool tail = false;                      // few live slots: the tail form runs
    int len = 0;
    int64_t per_chunk = 0;
    int poll = 4;
    long long guard = 0;
    int done = 0;
    ~PendingBatch() {
      if (gexec) cudaGraphExecDestroy(gexec);
      if (gexec_tail) cudaGraphExecDestroy(gexec_tail);
    }
  };
  std::unique_ptr<PendingBatch> pend;

  // Release the pending batch. clear_slots: the batch was abandoned before it
  // finished, so its running cases are stopped (their slots go inactive).
  int batch_cancel(bool clear_slots = true) {
    if (!pend) return ESR_OK;   // nothing pending: nothing changes
    int rc = ESR_OK;
    if (clear_slots && pend->n > 0) cudaMemsetAsync(active.p, 0, n_slots * sizeof(int), stream);
    // every slot is a step kernel's again
    cudaMemcpyAsync(d_live.p, h_live_full.data(), h_live_full.size() * sizeof(int4), cudaMemcpyHostToDevice, stream);
    // nothing of the batch may still run when its buffers are freed
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) rc = fail(ESR_ERR_CUDA, std::string("batch_cancel: ") + cudaGetErrorString(e));
    pend.reset();
    batch_busy = false;
    for (int g = 0; g < n_slots; ++g) hcase_index[g] = -1;
    return rc;
  }

  int batch_submit(const esr_case* cs, int n, const double* const* init, bool want_states) {
    if (pend) return fail(ESR_ERR_STATE, "batch_submit: a batch is already pending");
    const int nm = (int)meshes.size();
    for (int i = 0; i < n; ++i) {
      if (cs[i].mesh < 0 || cs[i].mesh >= nm) return fail(ESR_ERR_ARG, "batch: case mesh out of range");
      if (meshes[cs[i].mesh]->B < 1) return fail(ESR_ERR_ARG, "batch: case mesh has no slots");
      if (!(cs[i].cfl > 0)) return fail(ESR_ERR_ARG, "batch: cfl must be > 0");
      if (!(cs[i].tf > 0) && cs[i].max_steps <= 0) return fail(ESR_ERR_ARG, "batch: tf must be > 0");
    }
    auto owned = std::make_unique<PendingBatch>();
    PendingBatch& pb = *owned;
    pb.Bp = &batch_bufs;
    pb.n = n;
    pb.want_states = want_states;
    if (n == 0) {   // nothing to run: the slots are left as they are
      pend = std::move(owned);
      batch_busy = true;
      return ESR_OK;
    }
    int rc = submit_fill(pb, cs, init);
    if (rc != ESR_OK) {   // owned (and its buffers) go once the stream is idle
      cudaStreamSynchronize(stream);
      return rc;
    }
    pend = std::move(owned);
    batch_busy = true;
    return ESR_OK;
  }

  int submit_fill(PendingBatch& pb, const esr_case* cs, const double* const* init) {
    const int n = pb.n, nm = (int)meshes.size();
    // device copies of the renumbering, once per solver
    if (!perm_ptrs.p) {
      size_t tot = 0;
      for (auto& md : meshes) tot += md->hm->n_cells;
      ESR_TRY(perm_all.alloc(tot));
      std::vector<const int*> pp(nm), ip(nm);
      size_t o = 0;
      for (int m = 0; m < nm; ++m) {
        const HostMesh& hm = *meshes[m]->hm;
        ESR_CUDA(cudaMemcpy(perm_all.p + o, hm.perm.data(), hm.n_cells * sizeof(int), cudaMemcpyHostToDevice));
        pp[m] = perm_all.p + o;
        ip[m] = meshes[m]->inv.p;
        o += hm.n_cells;
      }
      ESR_TRY(perm_ptrs.alloc(nm));
      ESR_TRY(inv_ptrs.alloc(nm));
      ESR_CUDA(cudaMemcpy(perm_ptrs.p, pp.data(), nm * sizeof(const int*), cudaMemcpyHostToDevice));
      ESR_CUDA(cudaMemcpy(inv_ptrs.p, ip.data(), nm * sizeof(const int*), cudaMemcpyHostToDevice));
    }
    BatchBufs& B = *pb.Bp;
    // queue: cases grouped by mesh, submission order inside a mesh
    std::vector<int> qlist, qoff(nm + 1, 0);
    for (int m = 0; m < nm; ++m) {
      qoff[m] = (int)qlist.size();
      for (int i = 0; i < n; ++i) if (cs[i].mesh == m) qlist.push_back(i);
    }
    qoff[nm] = (int)qlist.size();
    std::vector<V> hin(n);
    std::vector<T> hstr(n);
    std::vector<double> hcfl(n), htf(n), hq(n), hthr(n);
    std::vector<long long> hms(n), hinit_off(n, -1), hout_off(n, 0);
    std::vector<int> htr(n), hpat(n);
    std::vector<double4> het(n);
    long long init_rows = 0, out_rows = 0;
    pb.case_mesh.resize(n);
    for (int i = 0; i < n; ++i) {
      case_params(cs[i], hin[i], hstr[i], hq[i], het[i], htr[i], hpat[i]);
      hcfl[i] = cs[i].cfl;
      htf[i] = cs[i].tf;
      hthr[i] = cs[i].threshold;
      hms[i] = cs[i].max_steps;
      pb.case_mesh[i] = cs[i].mesh;
      const int N = meshes[cs[i].mesh]->hm->n_cells;
      if (init && init[i]) { hinit_off[i] = init_rows; init_rows += N; }
      hout_off[i] = out_rows;
      out_rows += N;
    }
    pb.out_off = hout_off;
    const bool want_states = pb.want_states;
    auto up = [&](auto& buf, const auto& v) -> int {
      using E = typename std::decay_t<decltype(v)>::value_type;
      ESR_TRY(buf.reserve(std::max<size_t>(v.size(), 1)));
      if (!v.empty()) ESR_CUDA(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice, stream));
      return ESR_OK;
    };
    ESR_TRY(up(B.qlist, qlist));
    ESR_TRY(up(B.qoff, qoff));
    ESR_TRY(up(B.c_inlet, hin));
    ESR_TRY(up(B.c_strength, hstr));
    ESR_TRY(up(B.c_cfl, hcfl));
    ESR_TRY(up(B.c_tf, htf));
    ESR_TRY(up(B.c_qref, hq));
    ESR_TRY(up(B.c_thr, hthr));
    ESR_TRY(up(B.c_max_steps, hms));
    ESR_TRY(up(B.c_eng_track, htr));
    ESR_TRY(up(B.c_eng_pat, hpat));
    ESR_TRY(up(B.c_eng_t, het));
    ESR_TRY(up(B.init_off, hinit_off));
    ESR_TRY(up(B.out_off, hout_off));
    for (DevBuf<int>* b : {&B.qhead, &B.n_done}) {
      ESR_TRY(b->reserve(std::max(nm, 1)));
      ESR_CUDA(cudaMemsetAsync(b->p, 0, std::max(nm, 1) * sizeof(int), stream));
    }
    ESR_TRY(B.slot_case.reserve(n_slots));
    ESR_TRY(B.retiring.reserve(n_slots));
    std::vector<int> minus(n_slots, -1);
    ESR_CUDA(cudaMemcpyAsync(B.slot_case.p, minus.data(), n_slots * sizeof(int), cudaMemcpyHostToDevice, stream));
    ESR_CUDA(cudaMemsetAsync(B.retiring.p, 0, n_slots * sizeof(int), stream));
    ESR_CUDA(cudaMemsetAsync(active.p, 0, n_slots * sizeof(int), stream));
    ESR_CUDA(cudaMemsetAsync(status.p, 0, n_slots * sizeof(int), stream));
    ESR_CUDA(cudaMemcpyAsync(d_live.p, h_live_full.data(), h_live_full.size() * sizeof(int4), cudaMemcpyHostToDevice,
                             stream));
    for (DevBuf<int>* b : {&B.r_status, &B.r_stop, &B.r_steps, &B.r_nmax, &B.r_eng_conv, &B.r_eng_stop})
      ESR_TRY(b->reserve(n));
    for (DevBuf<double>* b : {&B.r_dt, &B.r_rel, &B.r_cd, &B.r_cl, &B.r_time, &B.r_probe}) ESR_TRY(b->reserve(n));
    if (Wp.n < (size_t)total) ESR_TRY(Wp.alloc(total));
    if (move_src.n < (size_t)n_slots) ESR_TRY(move_src.alloc(n_slots));
    if (init_rows > 0) {
      ESR_TRY(B.init.reserve((size_t)4 * init_rows));
      for (int i = 0; i < n; ++i)
        if (init && init[i])
          ESR_CUDA(cudaMemcpyAsync(B.init.p + 4 * hinit_off[i], init[i],
                                   (size_t)4 * meshes[cs[i].mesh]->hm->n_cells * sizeof(double),
                                   cudaMemcpyHostToDevice, stream));
    }
    if (want_states) ESR_TRY(B.out.reserve((size_t)4 * out_rows));
    ESR_CUDA(cudaStreamSynchronize(stream));   // host vectors above are the copy sources
    pb.q = Queue<T>{nm, B.qlist.p, B.qoff.p, B.qhead.p, B.slot_case.p, B.retiring.p, B.c_inlet.p, B.c_strength.p,
               B.c_cfl.p, B.c_tf.p, B.c_max_steps.p, B.c_qref.p, B.c_eng_track.p, B.c_eng_pat.p, B.c_eng_t.p, B.c_thr.p,
               init_rows > 0 ? B.init.p : nullptr, B.init_off.p, B.r_status.p, B.r_stop.p, B.r_steps.p, B.r_nmax.p,
               B.r_dt.p, B.r_rel.p, B.r_cd.p, B.r_cl.p, B.r_time.p, B.r_eng_conv.p, B.r_eng_stop.p, B.r_probe.p,
               want_states ? B.out.p : nullptr, B.out_off.p, B.n_done.p};
    pb.sp = SlotParams<T>{dt.p, inlet.p, strength.p, cfl.p, tf.p, max_steps.p, qref.p, eng_track.p, eng_patience.p, eng_t.p, thr.p};
    ESR_CUDA(cudaEventRecord(ev0, stream));
    issue_refill(pb.q, pb.sp, want_states);   // first fill of every slot
    // the chunk graph of this batch: steps, checks, then the refill sequence
    pb.len = run_chunk_len();
    if (P.use_graphs) {
      cudaGraph_t graph = nullptr;
      ESR_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      const int64_t before = launches;
      issue_run_chunk(pb.len);
      issue_refill(pb.q, pb.sp, want_states);
      pb.per_chunk = launches - before;
      launches = before;
      ESR_CUDA(cudaStreamEndCapture(stream, &graph));
      cudaError_t e = cudaGraphInstantiate(&pb.gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) { pb.gexec = nullptr; return fail(ESR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)); }
      if (use_patch && n_pblk > 0) {   // the tail form: K2 per cell
        ESR_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        tail_cell_k2 = true;
        const int64_t b2 = launches;
        issue_run_chunk(pb.len);
        issue_refill(pb.q, pb.sp, want_states);
        launches = b2;
        tail_cell_k2 = false;
        ESR_CUDA(cudaStreamEndCapture(stream, &graph));
        e = cudaGraphInstantiate(&pb.gexec_tail, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { pb.gexec_tail = nullptr; return fail(ESR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)); }
      }
    }
    return ESR_OK;
  }

  // One poll: a few chunks (doubling up to 32 per call), then the
  // done counter. A failure abandons the batch.
  int batch_poll(int* n_done) {
    if (!pend) return fail(ESR_ERR_STATE, "batch_poll: no batch pending");
    PendingBatch& pb = *pend;
    int rc = ESR_OK;
    if (pb.done < pb.n) {
      for (int i = 0; i < pb.poll && rc == ESR_OK; ++i) {
        cudaGraphExec_t g = (pb.tail && pb.gexec_tail) ? pb.gexec_tail : pb.gexec;
        if (g) {
          cudaError_t e = cudaGraphLaunch(g, stream);
          if (e != cudaSuccess) rc = fail(ESR_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
          else launches += pb.per_chunk;
        } else {
          tail_cell_k2 = pb.tail;
          issue_run_chunk(pb.len);
          issue_refill(pb.q, pb.sp, pb.want_states);
          tail_cell_k2 = false;
        }
      }
      if (rc == ESR_OK) {
        // the done counter and, for K2 by patches, each mesh's live slots
        const bool watch = use_patch && n_pblk > 0;
        h_live_poll.resize(meshes.size());
        cudaError_t e = cudaMemcpyAsync(&pb.done, pb.Bp->n_done.p, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess && watch)
          e = cudaMemcpyAsync(h_live_poll.data(), d_live.p, meshes.size() * sizeof(int4), cudaMemcpyDeviceToHost,
                              stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) rc = fail(ESR_ERR_CUDA, std::string("batch poll: ") + cudaGetErrorString(e));
        if (rc == ESR_OK && watch) {
          bool few = true;
          for (const int4& L : h_live_poll) few = few && L.x <= kTailSlots;
          pb.tail = few;
        }
      }
      pb.poll = std::min(pb.poll * 2, 32);
      if (rc == ESR_OK && ++pb.guard > (1LL << 40)) rc = fail(ESR_ERR_STATE, "batch: no progress");
    }
    if (rc != ESR_OK) {
      const std::string msg = g_last_error;
      batch_cancel(true);
      return fail(rc, msg);
    }
    if (n_done) *n_done = pb.done;
    return ESR_OK;
  }

  int batch_results(esr_result* out, double* const* finals) {
    if (!pend) return fail(ESR_ERR_STATE, "batch_results: no batch pending");
    PendingBatch& pb = *pend;
    if (pb.done < pb.n) return fail(ESR_ERR_STATE, "batch_results: the batch has not finished");
    if (finals && !pb.want_states) return fail(ESR_ERR_ARG, "batch_results: final states were not requested at submit");
    const int n = pb.n;
    if (n > 0 && !out) return fail(ESR_ERR_ARG, "batch_results: null results");
    if (n == 0) return batch_cancel(false);
    BatchBufs& B = *pb.Bp;
    ESR_CUDA(cudaEventRecord(ev1, stream));
    std::vector<int> st(n), sstop(n), ssteps(n), snmax(n), sec(n), ses(n);
    std::vector<double> sdt(n), srel(n), scd(n), scl(n), stime(n), sprobe(n);
    auto down = [&](auto& v, const auto& buf) -> int {
      using E = typename std::decay_t<decltype(v)>::value_type;
      ESR_CUDA(cudaMemcpyAsync(v.data(), buf.p, v.size() * sizeof(E), cudaMemcpyDeviceToHost, stream));
      return ESR_OK;
    };
    ESR_TRY(down(st, B.r_status)); ESR_TRY(down(sstop, B.r_stop)); ESR_TRY(down(ssteps, B.r_steps));
    ESR_TRY(down(snmax, B.r_nmax)); ESR_TRY(down(sec, B.r_eng_conv)); ESR_TRY(down(ses, B.r_eng_stop));
    ESR_TRY(down(sdt, B.r_dt)); ESR_TRY(down(srel, B.r_rel)); ESR_TRY(down(scd, B.r_cd)); ESR_TRY(down(scl, B.r_cl));
    ESR_TRY(down(stime, B.r_time));
    ESR_TRY(down(sprobe, B.r_probe));
    if (finals)
      for (int i = 0; i < n; ++i)
        if (finals[i])
          ESR_CUDA(cudaMemcpyAsync(finals[i], B.out.p + 4 * pb.out_off[i],
                                   (size_t)4 * meshes[pb.case_mesh[i]]->hm->n_cells * sizeof(double),
                                   cudaMemcpyDeviceToHost, stream));
    ESR_CUDA(cudaStreamSynchronize(stream));
    for (int i = 0; i < n; ++i) {
      esr_result& r = out[i];
      r = esr_result{};
      r.status = st[i];
      r.converged = st[i] == ESR_CASE_CONVERGED;
      r.stopping_step = sstop[i];
      r.steps = ssteps[i];
      r.n_max = snmax[i];
      r.case_index = i;
      r.dt = sdt[i];
      r.last_rel = srel[i];
      r.cd = scd[i];
      r.cl = scl[i];
      r.solve_time_s = stime[i];
      r.eng_converged = sec[i];
      r.eng_stopping_step = ses[i];
      r.final_residual = sprobe[i];
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    last_ms = ms;
    return batch_cancel(false);   // releases the batch's buffers and graph
  }

  int batch(const esr_case* cs, int n, const double* const* init, double* const* finals, esr_result* out) {
    ESR_TRY(batch_submit(cs, n, init, finals != nullptr));
    while (pend && pend->done < pend->n) ESR_TRY(batch_poll(nullptr));
    return batch_results(out, finals);
  }
};

struct esr_solver {
  std::unique_ptr<SolverBase> impl;
  int precision = 0;
};

// ------------------------------------------------------------------- C ABI
#define ESR_GUARD_BEGIN try {
#define ESR_GUARD_END                                                   \
  }                                                                     \
  catch (const std::exception& e) { return fail(ESR_ERR_STATE, e.what()); } \
  catch (...) { return fail(ESR_ERR_STATE, "unknown C++ exception"); }

// dispatch_any: calls that are valid while a submitted batch owns the slots
template <typename F>
static int dispatch_any(esr_solver* s, F&& f) {
  if (!s || !s->impl) return fail(ESR_ERR_ARG, "null solver");
  if (s->precision == ESR_PREC_F64) return f(*static_cast<SolverT<double>*>(s->impl.get()));
  return f(*static_cast<SolverT<float>*>(s->impl.get()));
}
template <typename F>
static int dispatch(esr_solver* s, F&& f) {
  if (s && s->impl && s->impl->batch_busy)
    return fail(ESR_ERR_STATE, "a submitted batch owns the solver's slots: read its results or cancel it first");
  return dispatch_any(s, std::forward<F>(f));
}

extern "C" {

int32_t esr_api_version(void) { return ESR_API_VERSION; }
const char* esr_last_error(void) { return g_last_error.c_str(); }

int esr_mesh_create(const esr_mesh_desc* desc, esr_mesh** out) {
  ESR_GUARD_BEGIN
  if (!desc || !out) return fail(ESR_ERR_ARG, "mesh_create: null argument");
  auto m = std::make_unique<esr_mesh>();
  std::string err;
  int rc = esr::prepare_mesh(*desc, m->hm, err);
  if (rc != ESR_OK) return fail(rc, err);
  *out = m.release();
  return ESR_OK;
  ESR_GUARD_END
}

int esr_mesh_destroy(esr_mesh* mesh) {
  delete mesh;
  return ESR_OK;
}

int esr_mesh_get_info(const esr_mesh* mesh, esr_mesh_info* info) {
  if (!mesh || !info) return fail(ESR_ERR_ARG, "mesh_get_info: null argument");
  const HostMesh& hm = mesh->hm;
  info->n_cells = hm.n_cells;
  info->n_faces = hm.n_faces;
  info->n_wall_faces = (int)hm.wall_cell.size();
  info->n_boundary_slots = hm.n_boundary_slots;
  info->y_min = hm.y_min;
  info->y_max = hm.y_max;
  info->device_bytes_f32 = (int64_t)hm.n_cells * (G_COUNT * 4 + 16);
  info->device_bytes_f64 = (int64_t)hm.n_cells * (G_COUNT * 8 + 16);
  return ESR_OK;
}

int esr_mesh_get_permutation(const esr_mesh* mesh, int32_t* perm) {
  if (!mesh || !perm) return fail(ESR_ERR_ARG, "mesh_get_permutation: null argument");
  std::memcpy(perm, mesh->hm.perm.data(), mesh->hm.perm.size() * sizeof(int32_t));
  return ESR_OK;
}

int esr_mesh_get_patches(const esr_mesh* mesh, int32_t* n_patches, int32_t* start) {
  if (!mesh || !n_patches) return fail(ESR_ERR_ARG, "mesh_get_patches: null argument");
  const auto& ps = mesh->hm.patch_start;
  *n_patches = (int32_t)ps.size() - 1;
  if (start) std::memcpy(start, ps.data(), ps.size() * sizeof(int32_t));
  return ESR_OK;
}

int esr_mesh_get_geometry(const esr_mesh* mesh, int32_t fidelity, int32_t precision, double* geo, double* lsq) {
  if (!mesh || !geo) return fail(ESR_ERR_ARG, "mesh_get_geometry: null argument");
  if (fidelity != ESR_FIDELITY_FAST && fidelity != ESR_FIDELITY_REFERENCE) return fail(ESR_ERR_ARG, "unknown fidelity");
  if (precision != ESR_PREC_F32 && precision != ESR_PREC_F64) return fail(ESR_ERR_ARG, "unknown precision");
  const HostMesh& hm = mesh->hm;
  const bool ref = fidelity == ESR_FIDELITY_REFERENCE;
  for (int c = 0; c < hm.n_cells; ++c) {
    const size_t i = (size_t)hm.inv[c] * G_COUNT;
    for (int f = 0; f < G_COUNT; ++f) {
      double v;
      if (!ref) v = precision == ESR_PREC_F32 ? (double)(float)hm.geo[i + f] : hm.geo[i + f];
      else v = precision == ESR_PREC_F32 ? (double)hm.geo_ref32[i + f] : hm.geo_ref64[i + f];
      geo[(size_t)c * G_COUNT + f] = v;
    }
    if (lsq && ref && precision == ESR_PREC_F32) {
      const LsqRef& L = hm.lsq_ref32[hm.inv[c]];
      double* o = lsq + (size_t)c * 13;
      for (int k = 0; k < 3; ++k) o[k] = L.w[k];
      for (int k = 0; k < 6; ++k) o[3 + k] = L.dx[k];
      for (int k = 0; k < 4; ++k) o[9 + k] = L.a[k];
    }
  }
  return ESR_OK;
}

int esr_solver_create(const esr_mesh* const* meshes, const int32_t* slots_per_mesh, int32_t n_meshes,
                      const esr_params* params, esr_solver** out) {
  ESR_GUARD_BEGIN
  if (!meshes || !slots_per_mesh || n_meshes <= 0 || !params || !out) return fail(ESR_ERR_ARG, "solver_create: null argument");
  for (int m = 0; m < n_meshes; ++m) {
    if (!meshes[m]) return fail(ESR_ERR_ARG, "solver_create: null mesh");
    if (slots_per_mesh[m] <= 0) return fail(ESR_ERR_ARG, "solver_create: slots_per_mesh must be > 0");
  }
  const esr_params& p = *params;
  if (p.precision != ESR_PREC_F32 && p.precision != ESR_PREC_F64) return fail(ESR_ERR_ARG, "unknown precision");
  if (p.flux != ESR_FLUX_HLLC && p.flux != ESR_FLUX_RUSANOV) return fail(ESR_ERR_ARG, "Unknown flux type");
  if (p.reconstruction != ESR_RECON_MUSCL && p.reconstruction != ESR_RECON_CONSTANT) return fail(ESR_ERR_ARG, "Unknown reconstruction scheme");
  if (p.time_scheme < ESR_TIME_SRK2 || p.time_scheme > ESR_TIME_RK2) return fail(ESR_ERR_ARG, "unknown time scheme");
  if (p.dt_mode != ESR_DT_GLOBAL && p.dt_mode != ESR_DT_LOCAL) return fail(ESR_ERR_ARG, "unknown dt mode");
  if (p.stop_rule != ESR_STOP_REFERENCE && p.stop_rule != ESR_STOP_DENSITY_L2 && p.stop_rule != ESR_STOP_ENGINEERING)
    return fail(ESR_ERR_ARG, "unknown stop rule");
  if (!(p.gamma > 1.0)) return fail(ESR_ERR_ARG, "gamma must be > 1");
  if (p.fidelity != ESR_FIDELITY_FAST && p.fidelity != ESR_FIDELITY_REFERENCE) return fail(ESR_ERR_ARG, "unknown fidelity");
  auto s = std::make_unique<esr_solver>();
  s->precision = p.precision;
  int rc;
  if (p.precision == ESR_PREC_F64) {
    auto impl = std::make_unique<SolverT<double>>();
    rc = impl->init(meshes, slots_per_mesh, n_meshes, &p);
    s->impl = std::move(impl);
  } else {
    auto impl = std::make_unique<SolverT<float>>();
    rc = impl->init(meshes, slots_per_mesh, n_meshes, &p);
    s->impl = std::move(impl);
  }
  if (rc != ESR_OK) return rc;
  *out = s.release();
  return ESR_OK;
  ESR_GUARD_END
}

int esr_solver_destroy(esr_solver* solver) {
  delete solver;
  return ESR_OK;
}

int esr_solver_num_slots(const esr_solver* solver, int32_t* n) {
  if (!solver || !n) return fail(ESR_ERR_ARG, "null argument");
  return dispatch_any(const_cast<esr_solver*>(solver), [&](auto& s) { *n = s.n_slots; return ESR_OK; });
}

int esr_solver_tuning(const esr_solver* solver, esr_tuning* out) {
  if (!solver || !out) return fail(ESR_ERR_ARG, "null argument");
  return dispatch_any(const_cast<esr_solver*>(solver), [&](auto& s) { return s.get_tuning(out); });
}

int esr_solver_set_shape(esr_solver* solver, const esr_tuning_variant* shape) {
  if (!solver || !shape) return fail(ESR_ERR_ARG, "null argument");
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.set_shape(shape); });
  ESR_GUARD_END
}

int esr_set_case(esr_solver* solver, int32_t slot, const esr_case* c, const double* W_init) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) {
    int rc = s.set_case(slot, c, W_init);
    if (rc == ESR_OK) s.hcase_index[slot] = slot;
    return rc;
  });
  ESR_GUARD_END
}
int esr_set_cases(esr_solver* solver, int32_t n, const int32_t* slots, const esr_case* cases,
                  const double* const* W_init) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.set_cases(n, slots, cases, W_init); });
  ESR_GUARD_END
}
int esr_get_states(esr_solver* solver, int32_t n, const int32_t* slots, double* const* out) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.get_states(n, slots, out); });
  ESR_GUARD_END
}
int esr_set_cases_f32(esr_solver* solver, int32_t n, const int32_t* slots, const esr_case* cases,
                      const float* const* W_init) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.set_cases(n, slots, cases, W_init); });
  ESR_GUARD_END
}
int esr_get_states_f32(esr_solver* solver, int32_t n, const int32_t* slots, float* const* out) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.get_states(n, slots, out); });
  ESR_GUARD_END
}
int esr_stage_cases_f32(esr_solver* solver, int32_t n, const int32_t* slots, const esr_case* cases,
                        const float* const* W_init) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.stage_in(n, slots, cases, W_init); });
  ESR_GUARD_END
}
int esr_apply_staged(esr_solver* solver) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.apply_staged(); });
  ESR_GUARD_END
}
int esr_fetch_states_f32(esr_solver* solver, int32_t n, const int32_t* slots, float* const* out) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.fetch_states(n, slots, out); });
  ESR_GUARD_END
}
int esr_wait_transfers(esr_solver* solver) {
  ESR_GUARD_BEGIN
  return dispatch_any(solver, [&](auto& s) { return s.wait_transfers(); });
  ESR_GUARD_END
}
int esr_clear_slot(esr_solver* solver, int32_t slot) {
  return dispatch(solver, [&](auto& s) { return s.clear_slot(slot); });
}
int esr_set_state(esr_solver* solver, int32_t slot, const double* W) {
  if (!W) return fail(ESR_ERR_ARG, "set_state: null state");
  return dispatch(solver, [&](auto& s) {
    int rc = s.set_state(slot, W, false);
    return rc != ESR_OK ? rc : s.reset_slot(slot);
  });
}
int esr_get_state(esr_solver* solver, int32_t slot, double* W) {
  if (!W) return fail(ESR_ERR_ARG, "get_state: null output");
  return dispatch(solver, [&](auto& s) { return s.get_state(slot, W, false); });
}
int esr_set_state_device(esr_solver* solver, int32_t slot, const void* d_W) {
  if (!d_W) return fail(ESR_ERR_ARG, "set_state_device: null state");
  return dispatch(solver, [&](auto& s) {
    int rc = s.set_state(slot, (const double*)d_W, true);
    return rc != ESR_OK ? rc : s.reset_slot(slot);
  });
}
int esr_get_state_device(esr_solver* solver, int32_t slot, void* d_W) {
  if (!d_W) return fail(ESR_ERR_ARG, "get_state_device: null output");
  return dispatch(solver, [&](auto& s) { return s.get_state(slot, (double*)d_W, true); });
}
int esr_compute_dt(esr_solver* solver, double* dt_per_slot) {
  if (!dt_per_slot) return fail(ESR_ERR_ARG, "compute_dt: null output");
  return dispatch(solver, [&](auto& s) { return s.dts(dt_per_slot); });
}
int esr_step(esr_solver* solver, int32_t nsteps) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.step_n(nsteps); });
  ESR_GUARD_END
}
int esr_run(esr_solver* solver, esr_result* results) {
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.run_all(results); });
  ESR_GUARD_END
}
int esr_get_results(esr_solver* solver, esr_result* results) {
  if (!results) return fail(ESR_ERR_ARG, "get_results: null output");
  return dispatch(solver, [&](auto& s) { return s.results(results); });
}
int esr_residual_probe(esr_solver* solver, double* rel) {
  if (!rel) return fail(ESR_ERR_ARG, "residual_probe: null output");
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.residual_probe(rel); });
  ESR_GUARD_END
}
int esr_forces(esr_solver* solver, double* cd, double* cl) {
  if (!cd || !cl) return fail(ESR_ERR_ARG, "forces: null output");
  return dispatch(solver, [&](auto& s) {
    int rc = s.compute_forces();
    if (rc != ESR_OK) return rc;
    std::vector<double> fo(2 * s.n_slots);
    cudaError_t e = cudaMemcpyAsync(fo.data(), s.forces.p, fo.size() * sizeof(double), cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess) return fail(ESR_ERR_CUDA, cudaGetErrorString(e));
    for (int g = 0; g < s.n_slots; ++g) { cd[g] = fo[2 * g]; cl[g] = fo[2 * g + 1]; }
    return ESR_OK;
  });
}
int esr_gradients(esr_solver* solver, int32_t slot, double* grad) {
  if (!grad) return fail(ESR_ERR_ARG, "gradients: null output");
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.gradients(slot, grad); });
  ESR_GUARD_END
}
int esr_entropy(esr_solver* solver, double* total) {
  if (!total) return fail(ESR_ERR_ARG, "entropy: null output");
  return dispatch(solver, [&](auto& s) { return s.entropy(total); });
}
int esr_synchronize(esr_solver* solver) {
  return dispatch_any(solver, [&](auto& s) {
    cudaError_t e = cudaStreamSynchronize(s.stream);
    return e == cudaSuccess ? ESR_OK : fail(ESR_ERR_CUDA, cudaGetErrorString(e));
  });
}
int esr_last_elapsed_ms(esr_solver* solver, double* ms) {
  if (!ms) return fail(ESR_ERR_ARG, "null output");
  return dispatch_any(solver, [&](auto& s) { *ms = s.last_ms; return ESR_OK; });
}
int esr_kernel_launches(const esr_solver* solver, int64_t* n) {
  if (!solver || !n) return fail(ESR_ERR_ARG, "null argument");
  *n = solver->impl->launches;
  return ESR_OK;
}
int esr_profile_step(esr_solver* solver, int32_t nsteps, esr_kernel_times* out) {
  if (!out) return fail(ESR_ERR_ARG, "profile_step: null output");
  ESR_GUARD_BEGIN
  return dispatch(solver, [&](auto& s) { return s.profile(nsteps, out); });
  ESR_GUARD_END
}
int esr_batch_solve(esr_solver* solver, const esr_case* cases, int32_t n_cases, const double* const* init_fields,
                    double* const* final_states, esr_result* results) {
  ESR_GUARD_BEGIN
  if (!cases || n_cases < 0 || !results) return fail(ESR_ERR_ARG, "batch_solve: null argument");
  return dispatch(solver, [&](auto& s) { return s.batch(cases, n_cases, init_fields, final_states, results); });
  ESR_GUARD_END
}
int esr_batch_submit(esr_solver* solver, const esr_case* cases, int32_t n_cases, const double* const* init_fields,
                     int32_t want_states) {
  ESR_GUARD_BEGIN
  if (n_cases < 0 || (n_cases > 0 && !cases)) return fail(ESR_ERR_ARG, "batch_submit: null argument");
  return dispatch(solver, [&](auto& s) { return s.batch_submit(cases, n_cases, init_fields, want_states != 0); });
  ESR_GUARD_END
}
int esr_batch_poll(esr_solver* solver, int32_t* n_done) {
  ESR_GUARD_BEGIN
  return dispatch_any(solver, [&](auto& s) {
    int d = 0;
    const int rc = s.batch_poll(&d);
    if (rc == ESR_OK && n_done) *n_done = d;
    return rc;
  });
  ESR_GUARD_END
}
int esr_batch_results(esr_solver* solver, double* const* final_states, esr_result* results) {
  ESR_GUARD_BEGIN
  return dispatch_any(solver, [&](auto& s) { return s.batch_results(results, final_states); });
  ESR_GUARD_END
}
int esr_batch_cancel(esr_solver* solver) {
  ESR_GUARD_BEGIN
  return dispatch_any(solver, [&](auto& s) { return s.batch_cancel(true); });
  ESR_GUARD_END
}

int esr_idw_apply(const float* d_src, int32_t n_src, int32_t n_vars, const int32_t* d_idx, const float* d_dist,
                  int32_t n_dst, int32_t k, float* d_out, void* stream) {
  if (!d_src || !d_idx || !d_dist || !d_out || n_src <= 0 || n_vars <= 0 || n_dst < 0) return fail(ESR_ERR_ARG, "idw: bad argument");
  if (k < 1 || k > 16) return fail(ESR_ERR_ARG, "idw: k must be in [1, 16]");
  if (n_dst == 0) return ESR_OK;
  const int tb = 128, nb = (n_dst + tb - 1) / tb;
  esr::k_idw<<<nb, tb, 0, (cudaStream_t)stream>>>(d_src, n_src, n_vars, d_idx, d_dist, n_dst, k, d_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ESR_OK : fail(ESR_ERR_CUDA, cudaGetErrorString(e));
}

int esr_idw_status(int32_t* bad) {
  if (!bad) return fail(ESR_ERR_ARG, "idw_status: null output");
  int v = 0;
  const int zero = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, esr::g_idw_bad, sizeof(int));
  if (e == cudaSuccess && v) e = cudaMemcpyToSymbol(esr::g_idw_bad, &zero, sizeof(int));
  if (e != cudaSuccess) return fail(ESR_ERR_CUDA, std::string("idw_status: ") + cudaGetErrorString(e));
  *bad = v;
  return ESR_OK;
}

}  // extern "C"
