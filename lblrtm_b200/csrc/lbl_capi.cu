// lbl_capi.cu -- the C ABI of include/lblgpu.h.
//
// A context owns the resident TAPE3 lines, the line-shape tables, the
// continuum table and a grow-only device arena for the per-call work
// buffers.  lbl_forward plans every layer on the host (exact FP64 panel and
// window schedule), lays all layers' buffers out in the arena, runs the
// optical-depth pipeline for all layers in a handful of batched launches,
// then merges the layers bottom-up on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lblgpu.h"
#include "lbl_kernels.cuh"
#include "lbl_plan.h"

using namespace lbl;

namespace {

// Device memory the context holds, against an optional cap
// (lbl_set_memory_limit).  Allocations that would pass the cap fail with
// cudaErrorMemoryAllocation, as a full device does.
struct DevBudget {
  size_t used = 0, limit = 0;  // limit 0: no cap
  cudaError_t alloc(void** p, size_t bytes) {
    *p = nullptr;
    if (limit && used + bytes > limit) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) used += bytes;
    else cudaGetLastError();
    return e;
  }
  void release(void* p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    used -= std::min(used, bytes);
  }
};

// Grow-only device arena; sub-allocations are 256-byte aligned.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  cudaError_t reserve(size_t bytes, DevBudget& b) {
    if (bytes <= cap) return cudaSuccess;
    size_t want = std::max(bytes, cap * 3 / 2);
    b.release(base, cap);
    base = nullptr;
    cap = 0;
    void* p = nullptr;
    cudaError_t e = b.alloc(&p, want);
    if (e != cudaSuccess && want > bytes) e = b.alloc(&p, want = bytes);
    if (e != cudaSuccess) return e;
    base = static_cast<char*>(p);
    cap = want;
    return cudaSuccess;
  }
  void reset() { used = 0; }
  template <typename T>
  T* take(size_t n) {
    size_t off = (used + 255) & ~size_t(255);
    used = off + n * sizeof(T);
    return reinterpret_cast<T*>(base + off);
  }
};

// Pass 1 of a layout computes the size, pass 2 hands out pointers.
struct Layout {
  size_t bytes = 0;
  template <typename T>
  void add(size_t n) {
    bytes = ((bytes + 255) & ~size_t(255)) + n * sizeof(T);
  }
};

// Persistent host workers for the per-layer planning: tasks [0, n) are taken
// from a shared counter by the workers and the calling thread (starting
// threads for every call costs more than planning a profile).
class HostPool {
 public:
  explicit HostPool(int nworkers) {
    for (int t = 0; t < nworkers; t++) th_.emplace_back([this] { work(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      quit_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void run(int n, const std::function<void(int)>& f) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      f_ = &f;
      n_ = n;
      next_.store(0);
      active_ = (int)th_.size();
      gen_++;
    }
    cv_.notify_all();
    for (int i; (i = next_.fetch_add(1)) < n;) f(i);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [this] { return active_ == 0; });
  }

 private:
  void work() {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int)>* f;
      int n;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
        if (quit_) return;
        seen = gen_;
        f = f_;
        n = n_;
      }
      for (int i; (i = next_.fetch_add(1)) < n;) (*f)(i);
      std::lock_guard<std::mutex> lk(mu_);
      if (--active_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* f_ = nullptr;
  int n_ = 0;
  std::atomic<int> next_{0};
  int active_ = 0;
  uint64_t gen_ = 0;
  bool quit_ = false;
};

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Page-locked host memory (cudaMallocHost or registered).
bool is_pinned(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

struct lbl_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // lines: host copies for planning, device copies for the kernels
  std::vector<double> h_vnu;
  std::vector<float> h_sp, h_pshift;
  std::vector<int32_t> h_mol, h_iflg;
  std::vector<int64_t> h_bs;
  double max_abs_pshift = 0.;
  DevLines dl{};
  void* line_mem = nullptr;
  size_t line_cap = 0;  // bytes of line_mem (grow-only)
  // pinned copies of each optical-depth pass's device status and work
  // counters (one slot per pass queued since the last synchronisation),
  // read after the caller's final synchronisation
  struct StatSlot {
    int32_t status[4];
    int32_t pad[4];
    unsigned long long cnt[8];
  };
  static constexpr int kStatSlots = 512;
  StatSlot* h_slots = nullptr;
  int nslot = 0;
  DevBudget mem;
  // pinned image of the plan tables and the event of its last upload
  // two images alternate, so that the host writes the next batch's plan
  // while the previous upload (or captured graph) may still read the other
  char* stage_host[2] = {nullptr, nullptr};
  size_t stage_cap[2] = {0, 0};
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  bool stage_ev_set[2] = {false, false};
  int stage_next = 0;
  // the executable graph of the last captured group (lbl_forward_batch)
  cudaGraphExec_t gexec = nullptr;
  bool have_lines = false;
  // fused panel kernel variant chosen by the autotuner (-1: not yet tuned)
  // kernel variants chosen by the autotuner per precision (-1: not tuned)
  int panel_variant[2] = {-1, -1};
  int far_variant[2] = {-1, -1};
  // tables
  DevShapes sh{};
  void* shape_mem = nullptr;
  DevMtckd ck{};
  void* ck_mem = nullptr;
  size_t ck_bytes = 0;
  // small pinned staging for per-call tables (layer offsets, channel
  // bounds): a ring of buffers, each reused once the copy that last read it
  // is done (small_ev is the event of the buffer handed out last)
  static constexpr int kSmallRing = 4;
  char* small_host[kSmallRing] = {};
  size_t small_cap[kSmallRing] = {};
  cudaEvent_t small_evs[kSmallRing] = {};
  bool small_used[kSmallRing] = {};
  int small_next = 0;
  cudaEvent_t small_ev = nullptr;
  // Jacobian work space (grow-only)
  char* jac_mem = nullptr;
  size_t jac_cap = 0;
  bool have_ck = false;
  Arena arena;
  std::unique_ptr<HostPool> pool;  // planning workers, created on first use
  // the result's copy-out, overlapped with the last merge launch
  static constexpr int kOutChunks = 4;
  cudaStream_t cstream = nullptr;
  cudaStream_t gstream = nullptr;  // the batched groups are captured here
  cudaEvent_t cev[kOutChunks + 1] = {};
  // merge buffers (ping-pong)
  double* mbuf[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t mcap = 0;
  // stage timing / work counters
  bool prof = false;
  struct Stage {
    std::string name;
    double ms = 0., work = 0.;
    int64_t launches = 0;
  };
  std::vector<Stage> stages;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> event_pool;
  size_t event_next = 0;
  Stage& stage(const char* nm) {
    for (auto& s : stages)
      if (s.name == nm) return s;
    stages.push_back(Stage{nm});
    return stages.back();
  }
  int stage_index(const char* nm) {
    for (size_t i = 0; i < stages.size(); i++)
      if (stages[i].name == nm) return (int)i;
    stages.push_back(Stage{nm});
    return (int)stages.size() - 1;
  }
  cudaEvent_t next_event() {
    if (event_next >= event_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      event_pool.push_back(e);
    }
    return event_pool[event_next++];
  }
};

namespace {
// Brackets one stage's launches with events when profiling is on.
struct StageTimer {
  lbl_ctx* c;
  int idx;
  cudaEvent_t a = nullptr;
  StageTimer(lbl_ctx* ctx, const char* nm, int64_t launches) : c(ctx) {
    idx = c->stage_index(nm);
    c->stages[idx].launches += launches;
    if (c->prof) {
      a = c->next_event();
      cudaEventRecord(a, c->stream);
    }
  }
  ~StageTimer() {
    if (c->prof) {
      cudaEvent_t b = c->next_event();
      cudaEventRecord(b, c->stream);
      c->pending.push_back({idx, {a, b}});
    }
  }
};
// Resolve recorded event pairs after the stream has been synchronised.
void harvest(lbl_ctx* c) {
  for (auto& p : c->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess)
      c->stages[p.first].ms += ms;
  }
  c->pending.clear();
  c->event_next = 0;
}
}  // namespace

namespace {

int fail(lbl_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

// A failed runtime call returns LBL_E_CUDA with the call and its message;
// an allocation that failed (device full or the context's cap reached)
// returns LBL_E_NOMEM.
#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      cudaGetLastError(); /* a later launch must not report this error again */       \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? LBL_E_NOMEM : LBL_E_CUDA,    \
                  std::string(#call) + ": " + cudaGetErrorString(e_));               \
    }                                                                                 \
  } while (0)

// Device view of one batch of planned layers.
struct Batch {
  std::vector<LayerPlan> plans;
  std::vector<LayerDev> ld;
  Work w{};
  LayerDev* d_ld = nullptr;
  int32_t* d_win_layer = nullptr;
  int32_t* d_win_order = nullptr;  // far-wing windows, most expensive first
  int32_t* d_panel_layer = nullptr;
  int64_t* d_panel_base = nullptr;
  int64_t* d_panel_rng = nullptr;  // candidate near-wing lines of every panel
  double* d_panel_segs = nullptr;  // RADFNI segments of every panel
  int32_t* d_panel_nseg = nullptr;
  int64_t* d_blk_base = nullptr;
  int64_t nblk_total = 0;
  int32_t nwin_total = 0;
  int64_t npanel_total = 0, max_far = 0;
  int64_t od_total = 0;
  int stage_k = 0;          // staging image holding the plan
  size_t upload_bytes = 0;  // bytes of the plan image
};

// Plan layers [0,n) on the host into `plans`.  The JRAD switch runs
// through the layers from jrad_in (one profile).
int plan_layers(lbl_ctx* ctx, const lbl_run& R, const lbl_layer* layers, int n, int jrad_in,
                int* jrad_out, std::vector<LayerPlan>& plans,
                const lbl_layer* chain = nullptr) {
  HostLines H{ctx->h_vnu.data(), ctx->h_sp.data(), ctx->h_pshift.data(), ctx->h_mol.data(),
              ctx->h_iflg.data(), (int64_t)ctx->h_vnu.size(), ctx->h_bs.data(),
              (int64_t)ctx->h_bs.size() - 1, ctx->max_abs_pshift};
  plans.resize(n);
  // the JRAD switch carries from layer to layer (OPDPTH :6211); everything
  // else in a layer's plan depends on that layer alone, so layers are
  // planned on several host threads
  std::vector<int> jin(n);
  int jrad = jrad_in;
  for (int l = 0; l < n; l++) {
    jin[l] = jrad;
    jrad = next_jrad(R, chain ? chain[l] : layers[l], jrad);
  }
  if (jrad_out) *jrad_out = jrad;
  std::vector<int> rcs(n, LBL_OK);
  std::vector<std::string> errs(n);
  const std::function<void(int)> plan_one = [&](int l) {
    rcs[l] = plan_layer(R, layers[l], jin[l], H, &plans[l], &errs[l]);
  };
  if (n < 8) {
    for (int l = 0; l < n; l++) plan_one(l);
  } else {
    if (!ctx->pool) {
      const int hw = (int)std::thread::hardware_concurrency();
      ctx->pool = std::make_unique<HostPool>(std::max(1, std::min(hw - 1, 7)));
    }
    ctx->pool->run(n, plan_one);
  }
  for (int l = 0; l < n; l++)
    if (rcs[l] != LBL_OK) return fail(ctx, rcs[l], "layer " + std::to_string(l) + ": " + errs[l]);
  for (int l = 0; l < n; l++)
    if (plans[l].d.n_r1 >= (int64_t(1) << 31) - 64)
      return fail(ctx, LBL_E_RANGE, "layer " + std::to_string(l) + ": more than 2^31 points");
  return LBL_OK;
}

// Device bytes one planned layer adds to a batch's arena (the per-layer
// terms of upload_batch's layout; the fixed part is under 64 KB).
size_t layer_arena_bytes(const LayerDev& d) {
  const size_t npanel = (size_t)d.npanel, nwin = (size_t)d.nwin;
  const size_t nfar = (size_t)(d.far_hi - d.far_lo), nnear = (size_t)(d.near_hi - d.near_lo);
  const size_t nblk = (size_t)(d.blk_hi - d.blk_lo), nfblk = (size_t)(d.fblk_hi - d.fblk_lo);
  const size_t nabs = (size_t)(d.icntnm ? d.nptabs : 0) + 8;
  return sizeof(LayerDev) + 64 + npanel * (8 + 4 + 4 + 16 + 8 * 3 * kPanelSegMax + 4) +
         nwin * (sizeof(WinDev) + 8 + 8 * kR4Stride) + nfar * 83 + 16 * (nfar / 1000 + 2) +
         nnear * (96 + sizeof(NearRec) + 8) + 16 * nblk + 8 * nabs + 8 * (size_t)d.npts +
         (8 * kSegMaxBlk + 16) * nfblk;
}

int upload_batch(lbl_ctx* ctx, Batch& B, bool defer = false);
int enqueue_upload(lbl_ctx* ctx, Batch& B);

// Plan layers [0,n), lay their buffers out in the arena, upload the plans.
// The JRAD chain follows `chain` when given (the nominal layers of a
// perturbed pass), else the layers themselves.
int prepare_batch(lbl_ctx* ctx, const lbl_run& R, const lbl_layer* layers, int n, int jrad_in,
                  int* jrad_out, Batch& B, const lbl_layer* chain = nullptr) {
  const auto t_host = std::chrono::steady_clock::now();
  int rc = plan_layers(ctx, R, layers, n, jrad_in, jrad_out, B.plans, chain);
  if (rc) return rc;
  rc = upload_batch(ctx, B);
  if (ctx->prof)
    ctx->stage("host_plan").ms +=
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host)
            .count();
  return rc;
}

// Lay the planned layers of B out in the arena and upload their plans (with
// `defer`, only write the plan image; enqueue_upload queues the copy).
int upload_batch(lbl_ctx* ctx, Batch& B, bool defer) {
  const int n = (int)B.plans.size();
  // offsets
  int64_t o_nblk = 0;
  int64_t o_r1 = 0, o_r2 = 0, o_r3 = 0, o_od = 0, o_pan = 0, o_win = 0, o_far = 0, o_near = 0,
          o_b9 = 0, o_abs = 0;
  B.ld.resize(n);
  std::vector<int64_t> blk_base(n + 1, 0);
  for (int l = 0; l < n; l++) {
    LayerDev& d = B.plans[l].d;
    d.off_r1 = o_r1;
    d.off_r2 = o_r2;
    d.off_r3 = o_r3;
    d.off_od = o_od;
    d.off_panel = o_pan;
    d.off_win = o_win;
    d.off_r4 = o_win * kR4Stride;
    d.off_far = o_far;
    d.off_shr = o_far;
    d.off_near = o_near;
    d.off_nblk = o_nblk;
    o_nblk += d.blk_hi - d.blk_lo;
    d.off_blk9 = o_b9;
    d.off_abs = o_abs;
    d.off_seg = blk_base[l];
    blk_base[l + 1] = blk_base[l] + (d.fblk_hi - d.fblk_lo);
    o_r1 += d.n_r1 + 1;
    o_r2 += d.n_r2 + 1;
    o_r3 += d.n_r3 + 1;
    o_od += d.npts;
    o_pan += d.npanel;
    o_win += d.nwin;
    const int64_t nfar = d.far_hi - d.far_lo;
    o_far += nfar;
    o_near += d.near_hi - d.near_lo;
    o_b9 += nfar / 1000 + 2;
    o_abs += (d.icntnm ? d.nptabs : 0) + 8;
    B.max_far = std::max(B.max_far, nfar);
    B.ld[l] = d;
  }
  B.nwin_total = (int32_t)o_win;
  B.npanel_total = o_pan;
  B.od_total = o_od;
  B.nblk_total = blk_base[n];
  const int64_t nbt = B.nblk_total + 1;
  // arena layout
  Layout lay;
  lay.add<LayerDev>(n);
  lay.add<double>(o_pan);
  lay.add<int32_t>(o_pan);
  lay.add<int32_t>(o_pan);
  lay.add<int64_t>(n + 1);
  lay.add<WinDev>(std::max<int64_t>(o_win, 1));
  lay.add<int32_t>(std::max<int64_t>(o_win, 1));
  lay.add<int32_t>(std::max<int64_t>(o_win, 1));
  lay.add<int64_t>(n + 1);
  lay.add<double>(std::max<int64_t>(o_win, 1) * kR4Stride);
  for (int k = 0; k < 5; k++) lay.add<double>(o_far + 1);
  lay.add<int8_t>(o_far + 1);
  lay.add<int8_t>(o_far + 1);
  for (int k = 0; k < 5; k++) lay.add<double>(o_far + 1);
  lay.add<int8_t>(o_far + 1);
  lay.add<int64_t>(n);
  lay.add<int64_t>(o_b9 + 1);
  lay.add<double>(o_b9 + 1);
  lay.add<int64_t>(n);
  lay.add<double>(o_near + 1);
  lay.add<double>(5 * (o_near + 1));
  lay.add<double>(o_near + 1);
  lay.add<NearPre>(o_near + 1);
  lay.add<int2>(o_nblk + 1);
  lay.add<NearRec>(o_near + 1);
  lay.add<double>(o_near + 1);
  lay.add<int32_t>(o_nblk + 1);
  lay.add<int32_t>(n);
  lay.add<int32_t>(n);
  lay.add<double>(o_abs);
  lay.add<double>(o_od);
  lay.add<int64_t>(2 * o_pan + 2);
  lay.add<double>(3 * kPanelSegMax * (o_pan + 1));
  lay.add<int32_t>(o_pan + 1);
  lay.add<int32_t>(8);
  lay.add<int32_t>(nbt * kSegMaxBlk);
  lay.add<int32_t>(nbt * kSegMaxBlk);
  lay.add<int32_t>(nbt);
  lay.add<int32_t>(nbt);
  lay.add<int64_t>(nbt);
  lay.add<int64_t>(n);
  lay.add<unsigned long long>(8);
  CK(ctx->arena.reserve(lay.bytes + 4096, ctx->mem));
  Arena& A = ctx->arena;
  A.reset();
  Work& w = B.w;
  B.d_ld = A.take<LayerDev>(n);
  double* d_vft = A.take<double>(o_pan);
  int32_t* d_win_of = A.take<int32_t>(o_pan);
  B.d_panel_layer = A.take<int32_t>(o_pan);
  B.d_panel_base = A.take<int64_t>(n + 1);
  WinDev* d_win = A.take<WinDev>(std::max<int64_t>(o_win, 1));
  B.d_win_layer = A.take<int32_t>(std::max<int64_t>(o_win, 1));
  B.d_win_order = A.take<int32_t>(std::max<int64_t>(o_win, 1));
  B.d_blk_base = A.take<int64_t>(n + 1);
  // everything up to here is the plan, uploaded in one copy
  const size_t upload_bytes = (size_t)(reinterpret_cast<char*>(B.d_blk_base + n + 1) - A.base);
  w.r4 = A.take<double>(std::max<int64_t>(o_win, 1) * kR4Stride);
  w.f_vnu = A.take<double>(o_far + 1);
  w.f_sp = A.take<double>(o_far + 1);
  w.f_alfa = A.take<double>(o_far + 1);
  w.f_epp = A.take<double>(o_far + 1);
  w.f_spp = A.take<double>(o_far + 1);
  w.f_ok = A.take<int8_t>(o_far + 1);
  w.f_co2 = A.take<int8_t>(o_far + 1);
  w.s_vnu = A.take<double>(o_far + 1);
  w.s_sp = A.take<double>(o_far + 1);
  w.s_alfa = A.take<double>(o_far + 1);
  w.s_epp = A.take<double>(o_far + 1);
  w.s_spp = A.take<double>(o_far + 1);
  w.s_co2 = A.take<int8_t>(o_far + 1);
  w.s_count = A.take<int64_t>(n);
  w.b9_start = A.take<int64_t>(o_b9 + 1);
  w.b9_vnuhi = A.take<double>(o_b9 + 1);
  w.b9_count = A.take<int64_t>(n);
  w.n_zslope = A.take<double>(o_near + 1);
  w.n_str = A.take<double>(5 * (o_near + 1));
  w.n_sppsp = A.take<double>(o_near + 1);
  w.n_pre = A.take<NearPre>(o_near + 1);
  w.n_blk = A.take<int2>(o_nblk + 1);
  w.n_rec = A.take<NearRec>(o_near + 1);
  w.n_rvnu = A.take<double>(o_near + 1);
  w.n_boff = A.take<int32_t>(o_nblk + 1);
  w.n_cnt = A.take<int32_t>(n);
  w.n_hw3 = A.take<int32_t>(n);
  w.absrb = A.take<double>(o_abs);
  w.od = A.take<double>(o_od);
  B.d_panel_rng = A.take<int64_t>(2 * o_pan + 2);
  B.d_panel_segs = A.take<double>(3 * kPanelSegMax * (o_pan + 1));
  B.d_panel_nseg = A.take<int32_t>(o_pan + 1);
  w.status = A.take<int32_t>(8);
  w.c_raw = A.take<int32_t>(nbt * kSegMaxBlk);
  w.c_out = A.take<int32_t>(nbt * kSegMaxBlk);
  w.seg_blk = A.take<int32_t>(nbt);
  w.seg_nblk = A.take<int32_t>(nbt);
  w.seg_out = A.take<int64_t>(nbt);
  w.seg_count = A.take<int64_t>(n);
  w.counters = A.take<unsigned long long>(8);
  w.L = B.d_ld;
  w.nlay = n;
  w.vft = d_vft;
  w.win_of = d_win_of;
  w.win = d_win;
  // The plan tables are written into a pinned host image of the start of
  // the arena and sent in one copy; the image is reused once the previous
  // call's copy has completed.
  cudaStream_t s = ctx->stream;
  const int sk = ctx->stage_next;
  ctx->stage_next ^= 1;
  B.stage_k = sk;
  B.upload_bytes = upload_bytes;
  if (ctx->stage_ev_set[sk]) CK(cudaEventSynchronize(ctx->stage_ev[sk]));
  if (upload_bytes > ctx->stage_cap[sk]) {
    if (ctx->stage_host[sk]) cudaFreeHost(ctx->stage_host[sk]);
    ctx->stage_host[sk] = nullptr;
    ctx->stage_cap[sk] = 0;
    void* hp = nullptr;
    CK(cudaMallocHost(&hp, upload_bytes));
    ctx->stage_host[sk] = static_cast<char*>(hp);
    ctx->stage_cap[sk] = upload_bytes;
  }
  auto host = [&](const void* dptr) {
    return ctx->stage_host[sk] + (reinterpret_cast<const char*>(dptr) - A.base);
  };
  std::memcpy(host(B.d_ld), B.ld.data(), sizeof(LayerDev) * n);
  double* h_vft = reinterpret_cast<double*>(host(d_vft));
  int32_t* h_wof = reinterpret_cast<int32_t*>(host(d_win_of));
  int32_t* h_play = reinterpret_cast<int32_t*>(host(B.d_panel_layer));
  int64_t* h_pbase = reinterpret_cast<int64_t*>(host(B.d_panel_base));
  WinDev* h_win = reinterpret_cast<WinDev*>(host(d_win));
  int32_t* h_wlay = reinterpret_cast<int32_t*>(host(B.d_win_layer));
  int32_t* h_word = reinterpret_cast<int32_t*>(host(B.d_win_order));
  std::memcpy(host(B.d_blk_base), blk_base.data(), sizeof(int64_t) * (n + 1));
  for (int l = 0; l < n; l++) {
    const LayerPlan& P = B.plans[l];
    const LayerDev& d = B.ld[l];
    h_pbase[l] = d.off_panel;
    std::memcpy(h_vft + d.off_panel, P.vft.data(), sizeof(double) * d.npanel);
    std::memcpy(h_wof + d.off_panel, P.win_of.data(), sizeof(int32_t) * d.npanel);
    std::fill(h_play + d.off_panel, h_play + d.off_panel + d.npanel, l);
    for (int k = 0; k < d.nwin; k++) {
      h_win[d.off_win + k] = P.win[k];
      h_wlay[d.off_win + k] = l;
    }
  }
  h_pbase[n] = o_pan;
  // Far-wing windows are launched most expensive first so that the long
  // ones do not start last.  Cost estimate: lines within the window's reach
  // (each is decided in order) times a fixed per-line decision cost plus the
  // points one line covers.
  {
    std::vector<double> cost(o_win);
    const double* vb = ctx->h_vnu.data();
    const double* ve = vb + ctx->h_vnu.size();
    for (int64_t k = 0; k < o_win; k++) {
      const WinDev& W = h_win[k];
      const LayerDev& d = B.ld[h_wlay[k]];
      const double nl = double(std::lower_bound(vb, ve, W.vnulst) - std::lower_bound(vb, ve, W.vlo));
      const double span = std::min<double>(W.nptr4, 2. * d.bound4 / d.dvr4 + 1.);
      cost[k] = nl * (span + 8000.);
      h_word[k] = (int32_t)k;
    }
    std::stable_sort(h_word, h_word + o_win,
                     [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
  }
  if (defer) return LBL_OK;
  const int rc = enqueue_upload(ctx, B);
  if (rc) return rc;
  CK(cudaEventRecord(ctx->stage_ev[sk], s));
  ctx->stage_ev_set[sk] = true;
  return LBL_OK;
}

// The device side of a batch's upload: the plan image in one copy, the
// status and counters cleared.  Queued directly, or inside a captured graph
// (the caller then records the staging image's event after the graph).
int enqueue_upload(lbl_ctx* ctx, Batch& B) {
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(ctx->arena.base, ctx->stage_host[B.stage_k], B.upload_bytes,
                     cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(B.w.status, 0, 4 * sizeof(int32_t), s));
  CK(cudaMemsetAsync(B.w.counters, 0, 8 * sizeof(unsigned long long), s));
  return LBL_OK;
}

// The second stream (plan-only kernels beside the far wing; the result's
// copy-out) and its events, created on first use.
int ensure_copy_stream(lbl_ctx* ctx) {
  if (ctx->cstream) return LBL_OK;
  CK(cudaStreamCreateWithFlags(&ctx->gstream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking));
  for (auto& e : ctx->cev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return LBL_OK;
}

int finish_od(lbl_ctx* ctx);

// The autotuner: on the context's first batch of at least kTuneMinPanels
// panels (kTuneMinWindows far-wing windows) in a precision, every variant of
// the fused panel kernel (records staged per batch, CTAs per SM) and of the
// far-wing kernel (adders per window CTA) runs once on that batch, timed by
// CUDA events on the context's stream, and the fastest is kept for the
// context's later calls in that precision (the far wing's tuning launches
// are the batch's own: the chosen variant runs once more unless it ran
// last).  LBL_PANEL_VARIANT / LBL_FAR_VARIANT (0-2) fix a variant.
constexpr int64_t kTuneMinPanels = 4096;
constexpr int64_t kTuneMinWindows = 128;

template <typename Launch>
int tune(lbl_ctx* ctx, int nvar, const char* env, const char* const* names, Launch launch,
         int* chosen, bool keep_result) {
  if (const char* e = std::getenv(env)) {
    const int v = std::atoi(e);
    if (v >= 0 && v < nvar) {
      *chosen = v;
      return LBL_OK;
    }
  }
  cudaStream_t s = ctx->stream;
  std::vector<cudaEvent_t> ev(nvar + 1);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  CK(cudaEventRecord(ev[0], s));
  for (int v = 0; v < nvar; v++) {
    CK(launch(v));
    CK(cudaEventRecord(ev[v + 1], s));
  }
  CK(cudaEventSynchronize(ev[nvar]));
  int best = 0;
  float best_ms = 1e30f;
  std::vector<float> ms(nvar, 0.f);
  for (int v = 0; v < nvar; v++) {
    CK(cudaEventElapsedTime(&ms[v], ev[v], ev[v + 1]));
    if (ms[v] < best_ms) {
      best_ms = ms[v];
      best = v;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  *chosen = best;
  // keep_result: the tuning launches produce the batch's result, which
  // must then be the chosen variant's (in the split form the far-wing
  // variants' FP32 chunk sums are not bit-identical), so that a first call
  // gives what every later call gives
  if (keep_result && best != nvar - 1) CK(launch(best));
  // reported with the stage times: each variant's time and the choice
  for (int v = 0; v < nvar; v++) {
    lbl_ctx::Stage& st = ctx->stage(names[v]);
    st.ms += ms[v];
    st.work = (v == best) ? 1. : 0.;
  }
  return LBL_OK;
}

int tune_panels(lbl_ctx* ctx, Batch& B, int precision) {
  static const char* names[2][kPanelVariants] = {
      {"tune_panel_s32_b4", "tune_panel_s64_b4", "tune_panel_s32_b5"},
      {"tune_panel32_s32_b4", "tune_panel32_s64_b4", "tune_panel32_s32_b5"}};
  const int pk = precision == LBL_PREC_SPLIT ? 1 : 0;
  return tune(ctx, kPanelVariants, "LBL_PANEL_VARIANT", names[pk],
              [&](int v) {
                return launch_panels(B.w, ctx->sh, B.npanel_total, B.d_panel_layer,
                                     B.d_panel_base, B.d_panel_rng, B.d_panel_segs,
                                     B.d_panel_nseg, precision, v, ctx->stream);
              },
              &ctx->panel_variant[pk], false);
}

int tune_far(lbl_ctx* ctx, Batch& B, int precision) {
  static const char* names[2][kFarVariants] = {
      {"tune_far_a160_d3", "tune_far_a128_d4", "tune_far_a192_d2"},
      {"tune_far32_a160_d3", "tune_far32_a128_d4", "tune_far32_a192_d2"}};
  const int pk = precision == LBL_PREC_SPLIT ? 1 : 0;
  return tune(ctx, kFarVariants, "LBL_FAR_VARIANT", names[pk],
              [&](int v) {
                return launch_far_wing(B.w, B.nwin_total, B.d_win_order, B.d_win_layer,
                                       precision, v, ctx->stream);
              },
              &ctx->far_variant[pk], true);
}

// A pinned host buffer of at least `bytes` for a table about to be copied
// to the device; the caller records ctx->small_ev after its copy.
int small_pinned(lbl_ctx* ctx, size_t bytes, void** out) {
  const int k = ctx->small_next;
  ctx->small_next = (k + 1) % lbl_ctx::kSmallRing;
  if (!ctx->small_evs[k])
    CK(cudaEventCreateWithFlags(&ctx->small_evs[k], cudaEventDisableTiming));
  if (ctx->small_used[k]) CK(cudaEventSynchronize(ctx->small_evs[k]));
  if (bytes > ctx->small_cap[k]) {
    if (ctx->small_host[k]) cudaFreeHost(ctx->small_host[k]);
    ctx->small_host[k] = nullptr;
    ctx->small_cap[k] = 0;
    void* hp = nullptr;
    CK(cudaMallocHost(&hp, std::max<size_t>(bytes, 1 << 16)));
    ctx->small_host[k] = static_cast<char*>(hp);
    ctx->small_cap[k] = std::max<size_t>(bytes, 1 << 16);
  }
  ctx->small_used[k] = true;
  ctx->small_ev = ctx->small_evs[k];
  *out = ctx->small_host[k];
  return LBL_OK;
}

// Optical depth of every layer of the batch into B.w.od.
int run_od(lbl_ctx* ctx, const lbl_run& R, Batch& B, int precision) {
  cudaStream_t s = ctx->stream;
  const Work& w = B.w;
  int64_t max_near = 0, max_panel = 0, max_win = 0, max_nblk = 0;
  for (const LayerDev& d : B.ld) {
    max_near = std::max<int64_t>(max_near, d.near_hi - d.near_lo);
    max_panel = std::max<int64_t>(max_panel, d.npanel);
    max_win = std::max<int64_t>(max_win, d.nwin);
    max_nblk = std::max<int64_t>(max_nblk, d.blk_hi - d.blk_lo);
  }
  if (near_walk_smem(max_panel, max_win) > kNearWalkSmemMax)
    return fail(ctx, LBL_E_RANGE, "layer grid too long for the near-wing panel walk");
  if (R.icntnm && !ctx->have_ck) return fail(ctx, LBL_E_NOTREADY, "continuum table not uploaded");
  int rc = ensure_copy_stream(ctx);
  if (rc) return rc;
  {
    StageTimer t(ctx, "far_scale", 1);
    CK(launch_far_scale(w, ctx->dl, B.max_far, s));
  }
  // The work that needs only the plans and the lines (near-wing line
  // scaling, the continuum, the panels' candidate ranges and radiation
  // segments) runs on a second stream beside SHRINK and the far wing; it
  // starts after the far-wing line scaling, which heads the longer chain.
  cudaStream_t s2 = ctx->cstream;
  CK(cudaEventRecord(ctx->cev[0], s));
  CK(cudaStreamWaitEvent(s2, ctx->cev[0], 0));
  CK(launch_near_lines(w, ctx->dl, max_near, s2));
  if (R.icntnm) CK(launch_continuum(w, ctx->ck, R.xself, R.xfrgn, R.xrayl, R.xco2c, R.xo2cn, R.xn2cn, s2));
  CK(launch_panel_segs(w, B.npanel_total, B.d_panel_layer, B.d_panel_base, B.d_panel_segs,
                       B.d_panel_nseg, s2));
  CK(cudaEventRecord(ctx->cev[1], s2));
  {
    StageTimer t(ctx, "shrink", 3);
    CK(launch_shrink(w, ctx->dl.bs, B.d_blk_base, B.nblk_total, s));
  }
  {
    StageTimer t(ctx, "far_wing", B.nwin_total > 0 ? 1 : 0);
    const int fk = precision == LBL_PREC_SPLIT ? 1 : 0;
    if (ctx->far_variant[fk] < 0 && B.nwin_total >= kTuneMinWindows) {
      const int rc3 = tune_far(ctx, B, precision);
      if (rc3) return rc3;
    } else {
      CK(launch_far_wing(w, B.nwin_total, B.d_win_order, B.d_win_layer, precision,
                         ctx->far_variant[fk], s));
    }
  }
  CK(cudaStreamWaitEvent(s, ctx->cev[1], 0));
  {
    // the walk and the window limits; the per-line part ran on the second stream
    StageTimer t(ctx, "near_scale", 3 + (R.icntnm ? 1 : 0) + 2 + 1);
    // the walk, then the window limits and packed records of the accepted lines
    CK(launch_near_walk(w, ctx->dl, max_panel, max_win, max_nblk, s));
    // every panel's candidate records
    CK(launch_panel_ranges(w, B.npanel_total, B.d_panel_layer, B.d_panel_base, B.d_panel_rng, s));
  }
  const int pk = precision == LBL_PREC_SPLIT ? 1 : 0;
  if (ctx->panel_variant[pk] < 0 && B.npanel_total >= kTuneMinPanels) {
    const int rc3 = tune_panels(ctx, B, precision);
    if (rc3) return rc3;
  }
  {
    // near-wing sums, PANEL combination and optical depth in one pass
    StageTimer t(ctx, "panels", 1);
    CK(launch_panels(w, ctx->sh, B.npanel_total, B.d_panel_layer, B.d_panel_base, B.d_panel_rng,
                     B.d_panel_segs, B.d_panel_nseg, precision, ctx->panel_variant[pk], s));
  }
  if (ctx->nslot >= lbl_ctx::kStatSlots) {
    // every slot holds a pass not yet read: drain them
    CK(cudaStreamSynchronize(s));
    const int rc2 = finish_od(ctx);
    if (rc2) return rc2;
  }
  lbl_ctx::StatSlot* sl = ctx->h_slots + ctx->nslot++;
  CK(cudaMemcpyAsync(sl->status, w.status, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(sl->cnt, w.counters, 8 * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, s));
  return LBL_OK;
}

// After the stream has been synchronised: the device status of the last
// run_od and its work counters.
int finish_od(lbl_ctx* ctx) {
  int32_t st = 0;
  for (int k = 0; k < ctx->nslot; k++) {
    const lbl_ctx::StatSlot& sl = ctx->h_slots[k];
    ctx->stage("far_wing").work += (double)sl.cnt[0];
    ctx->stage("panels").work += (double)sl.cnt[1];
    if (!st) st = sl.status[0];
  }
  ctx->nslot = 0;
  if (st == 2)
    return fail(ctx, LBL_E_RANGE,
                "far-wing line file too sparse: a LINF4 segment spans more than 48 TAPE3 panels");
  if (st != 0) return fail(ctx, LBL_E_CUDA, "device status " + std::to_string(st));
  return LBL_OK;
}

int copy_out(lbl_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (is_device_ptr(dst)) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  }
  return LBL_OK;
}

int check_run(lbl_ctx* ctx, const lbl_run* R) {
  if (!R) return fail(ctx, LBL_E_ARG, "run is NULL");
  if (R->ihirac != 1) return fail(ctx, LBL_E_ARG, "only IHIRAC=1 (Voigt) is supported");
  if (R->ilblf4 < 0 || R->ilblf4 > 2) return fail(ctx, LBL_E_ARG, "ILBLF4 must be 0, 1 or 2");
  if (!(R->v2 > R->v1)) return fail(ctx, LBL_E_ARG, "V2 must exceed V1");
  if (R->v2 - R->v1 > 2020.) return fail(ctx, LBL_E_RANGE, "V2-V1 above 2020 cm-1");
  if (R->v1 - 32. * 1e-9 <= 0.) return fail(ctx, LBL_E_RANGE, "V1 must be positive");
  if (!(R->sample > 0.) || !(R->alfal0 > 0.)) return fail(ctx, LBL_E_ARG, "SAMPLE/ALFAL0");
  if (R->iemit != 0 && R->iemit != 1) return fail(ctx, LBL_E_ARG, "IEMIT must be 0 or 1");
  if (R->iemit == 1 && R->ipathl != 1 && R->ipathl != 2 && R->ipathl != 3)
    return fail(ctx, LBL_E_ARG,
                "IPATHL must be 1 (looking down), 2 (tangent path) or 3 (looking up)");
  if (!(R->bndrfl >= 0. && R->bndrfl <= 1.))
    return fail(ctx, LBL_E_ARG, "BNDRFL must lie in [0, 1] (no reflectivity file)");
  if (!ctx->have_lines) return fail(ctx, LBL_E_NOTREADY, "lines not uploaded");
  return LBL_OK;
}

int ensure_merge_buffers(lbl_ctx* ctx, size_t n) {
  if (n <= ctx->mcap) return LBL_OK;
  for (int k = 0; k < 4; k++) {
    ctx->mem.release(ctx->mbuf[k], ctx->mcap * sizeof(double));
    ctx->mbuf[k] = nullptr;
  }
  ctx->mcap = 0;
  for (int k = 0; k < 4; k++) {
    void* p = nullptr;
    CK(ctx->mem.alloc(&p, n * sizeof(double)));
    ctx->mbuf[k] = static_cast<double*>(p);
  }
  ctx->mcap = n;
  return LBL_OK;
}

// Where the merged radiance and transmittance go (host or device memory);
// dev < 0: ask the runtime which memory each pointer is.
struct OutSink {
  double* rad;
  double* tr;  // may be null
  int rad_dev = -1, tr_dev = -1;
};

// Merge every layer of the batch bottom-up; result in mbuf[res], mbuf[res+1].
// With a sink, the last launch runs in kOutChunks pieces and each piece is
// copied to the sink on a second stream while the next one is merged; the
// main stream waits for the copies.
int run_merge(lbl_ctx* ctx, const lbl_run& R, const lbl_layer* layers, Batch& B, int n,
              int* res, int precision, const OutSink* sink = nullptr, int l0 = 0) {
  // the profile is layers [l0, l0+n) of the batch; `layers` points at its first
  const LayerDev* ld = B.ld.data() + l0;
  size_t mx = 0;
  for (auto& d : B.ld) mx = std::max<size_t>(mx, d.npts);
  int rc = ensure_merge_buffers(ctx, mx + 8);
  if (rc) return rc;
  // Consecutive layers on one grid go to one launch (at most kMergeRunMax).
  std::vector<std::pair<int, int>> runs;
  for (int l = 0; l < n;) {
    const LayerDev& d = ld[l];
    if (l > 0 && d.dv > ld[l - 1].dv) return fail(ctx, LBL_E_ITYPE, " RADMRG; ITYPE LT 0 ");
    int e = l + 1;
    while (e < n && e - l < kMergeRunMax && ld[e].dv == d.dv && ld[e].npts == d.npts) e++;
    runs.push_back({l, e});
    l = e;
  }
  if (sink) {
    const int rc2 = ensure_copy_stream(ctx);
    if (rc2) return rc2;
  }
  const int nchunk = sink ? lbl_ctx::kOutChunks : 1;
  int cur = 0;
  double dv_old = 0.;
  int64_t n_old = 0;
  StageTimer tm(ctx, "merge", (int64_t)runs.size() + nchunk - 1);
  for (size_t ri = 0; ri < runs.size(); ri++) {
    const int l = runs[ri].first, e = runs[ri].second;
    const LayerDev& d = ld[l];
    if (n_old >= (int64_t(1) << 31)) return fail(ctx, LBL_E_RANGE, "layer grid of 2^31 or more points");
    MergeRun m{};
    m.nl = e - l;
    m.first = (l == 0);
    m.itype = (l == 0 || dv_old == d.dv) ? 0 : (int32_t)(long)(d.dv / (dv_old - d.dv) + 0.5);
    m.n_old = (int32_t)n_old;
    // looking up (IPATHL=3): EMIN's level temperature is the lower level's
    // (XKTA, src/xmerge.f90:2405-2424), the merge adds the farther layer
    // seen through the nearer ones, and the boundary TMPBND lies beyond
    // the last layer (XMERGE :136-141)
    const bool down = R.ipathl == 3;
    m.down = down ? 1 : 0;
    m.tbnd_last = (down && e == n && n > 1) ? R.tmpbnd : 0.;
    // the symmetric tangent path (IPATHL=2, IANT=0): each layer's far
    // crossing radiates at its lower level's temperature (XKTB,
    // src/xmerge.f90:2417-2420, 2771-2773)
    m.tangent = R.ipathl == 2 ? 1 : 0;
    // the reflected atmosphere (IPATHL=1 with a boundary reflectivity: the
    // reference's IPATHL=-1, src/xmerge.f90:2389, 2725)
    m.refl = (R.iemit == 1 && R.ipathl == 1 && R.bndrfl > 0.) ? R.bndrfl : 0.;
    const bool use_b = m.tangent || m.refl > 0.;
    for (int k = l; k < e; k++) {
      m.od_off[k - l] = ld[k].off_od;
      m.t[k - l] = emin_temps(ld[k].tave, down ? layers[k].tzl : layers[k].tzu);
      const double tzl = layers[k].tzl;
      m.tb_xkt[k - l] = (use_b && tzl > 0.) ? tzl / kRADCN2 : 0.;
      m.tb_rk[k - l] = (use_b && tzl > 0.) ? kRADCN2 / tzl : 0.;
      ctx->stage("merge").work += (double)ld[k].npts;
    }
    const int nxt = cur ^ 2;
    const double tbnd = (l == 0 && R.ipathl == 1) ? R.tmpbnd : 0.;
    const bool last = ri + 1 == runs.size();
    if (!(last && sink)) {
      CK(launch_merge_run(m, B.w.vft + d.off_panel, B.w.od, d.npts, d.dv, ctx->mbuf[cur],
                          ctx->mbuf[cur + 1], ctx->mbuf[nxt], ctx->mbuf[nxt + 1], tbnd, R.bndemi,
                          R.iemit, ctx->stream, precision));
    } else {
      const bool rdev = sink->rad_dev >= 0 ? sink->rad_dev != 0 : is_device_ptr(sink->rad);
      const bool tdev = sink->tr && (sink->tr_dev >= 0 ? sink->tr_dev != 0 : is_device_ptr(sink->tr));
      const cudaMemcpyKind kr = rdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
      const cudaMemcpyKind kt = tdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
      const int64_t step = ((d.npts + nchunk - 1) / nchunk + 2399) / 2400 * 2400;
      // all pieces are queued before the first copy: a copy to pageable
      // host memory returns only when it is done
      for (int c = 0; c < nchunk; c++) {
        const int64_t lo = std::min<int64_t>(d.npts, c * step);
        const int64_t hi = std::min<int64_t>(d.npts, lo + step);
        CK(launch_merge_run(m, B.w.vft + d.off_panel, B.w.od, d.npts, d.dv, ctx->mbuf[cur],
                            ctx->mbuf[cur + 1], ctx->mbuf[nxt], ctx->mbuf[nxt + 1], tbnd,
                            R.bndemi, R.iemit, ctx->stream, precision, lo, hi));
        CK(cudaEventRecord(ctx->cev[c], ctx->stream));
      }
      for (int c = 0; c < nchunk; c++) {
        const int64_t lo = std::min<int64_t>(d.npts, c * step);
        const int64_t hi = std::min<int64_t>(d.npts, lo + step);
        if (hi == lo) continue;
        CK(cudaStreamWaitEvent(ctx->cstream, ctx->cev[c], 0));
        CK(cudaMemcpyAsync(sink->rad + lo, ctx->mbuf[nxt] + lo, sizeof(double) * (hi - lo), kr,
                           ctx->cstream));
        if (sink->tr)
          CK(cudaMemcpyAsync(sink->tr + lo, ctx->mbuf[nxt + 1] + lo, sizeof(double) * (hi - lo),
                             kt, ctx->cstream));
      }
      CK(cudaEventRecord(ctx->cev[nchunk], ctx->cstream));
      CK(cudaStreamWaitEvent(ctx->stream, ctx->cev[nchunk], 0));
    }
    cur = nxt;
    dv_old = d.dv;
    n_old = d.npts;
  }
  *res = cur;
  return LBL_OK;
}

}  // namespace

namespace {

// Device bytes a group of profiles may take in the arena: under the
// context's cap, what the cap leaves beside the other buffers; otherwise
// most of the device's free memory.
size_t group_budget(lbl_ctx* ctx, size_t merge_bytes) {
  size_t avail;
  const size_t others = ctx->mem.used - std::min(ctx->mem.used, ctx->arena.cap);
  if (ctx->mem.limit) {
    avail = ctx->mem.limit > others ? ctx->mem.limit - others : 0;
  } else {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    avail = fr + ctx->arena.cap;
    const size_t keep = (size_t)2 << 30;  // left to the caller and the runtime
    avail = avail > keep ? (avail - keep) / 10 * 9 : 0;
    // a group larger than this gains nothing (a few profiles fill the
    // device) and would leave the caller and the other work spaces no room
    avail = std::min(avail, tot / 10 * 4);
  }
  return avail > merge_bytes ? avail - merge_bytes : 0;
}

// Pinned staging of results bound for pageable host memory, so that the
// copies out stay asynchronous and the host goes on planning; two buffers
// alternate between groups.
struct Bounce {
  double* buf = nullptr;
  size_t cap = 0;  // doubles
  cudaEvent_t ev = nullptr;
  struct Out {
    double* dst;
    size_t off, n;
  };
  std::vector<Out> pend;
};

// Copy a bounce buffer's pending results to their host destinations once
// its group's copies are done.
int bounce_flush(lbl_ctx* ctx, Bounce& b) {
  if (b.pend.empty()) return LBL_OK;
  CK(cudaEventSynchronize(b.ev));
  for (const Bounce::Out& o : b.pend) std::memcpy(o.dst, b.buf + o.off, o.n * sizeof(double));
  b.pend.clear();
  return LBL_OK;
}

// The batched layer loop over profiles [lay0 index p] .. : profiles are
// planned on the host one after another and gathered into groups that fit
// the device budget; each group is uploaded in one copy, its optical depths
// computed by one set of launches for all its layers, and its profiles
// merged one after another, results going straight to device or pinned
// destinations (pageable ones through a pinned bounce buffer).  Every
// device step of a group is queued without a host wait, so the host plans
// the next group while the device computes this one.
int forward_groups(lbl_ctx* ctx, const lbl_run& R, lbl_layer* layers,
                   const std::vector<int64_t>& lay0, const int64_t* offsets, double* rad,
                   double* tr, int precision) {
  const int nprof = (int)lay0.size() - 1;
  size_t mx = 0;
  for (int p = 0; p < nprof; p++)
    for (int64_t l = lay0[p]; l < lay0[p + 1]; l++)
      mx = std::max<size_t>(mx, (size_t)layer_npts(R, layers[l].dv));
  int rc = ensure_merge_buffers(ctx, mx + 8);
  if (rc) return rc;
  rc = ensure_copy_stream(ctx);
  if (rc) return rc;
  const size_t budget = group_budget(ctx, 0);
  const bool rad_dev = is_device_ptr(rad), tr_dev = tr && is_device_ptr(tr);
  const bool rad_host = !rad_dev && !is_pinned(rad);
  const bool tr_host = tr && !tr_dev && !is_pinned(tr);
  // each group's device work is captured in a CUDA graph and launched as
  // one unit (LBL_BATCH_GRAPHS=0 launches it directly)
  const char* ge = std::getenv("LBL_BATCH_GRAPHS");
  const bool graphs_on = !(ge && ge[0] == '0');
  Bounce bounce[2];
  int bi = 0;
  std::vector<LayerPlan> cur;      // plans of the open group
  std::vector<int> cur_prof;       // its profiles
  size_t cur_bytes = 0;
  auto t_host = std::chrono::steady_clock::now();
  double host_ms = 0.;
  auto flush = [&]() -> int {
    if (cur_prof.empty()) return LBL_OK;
    host_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host)
                   .count();
    Batch B;
    B.plans = std::move(cur);
    cur.clear();
    int64_t npan = 0, nwin = 0;
    for (const LayerPlan& P : B.plans) {
      npan += P.d.npanel;
      nwin += P.d.nwin;
    }
    // a group is captured once the panel kernel's variant is settled (the
    // autotuner synchronises), without stage timing, and with a free status
    // slot (draining them synchronises)
    const bool graph = graphs_on && !ctx->prof &&
                       (ctx->panel_variant[precision == LBL_PREC_SPLIT ? 1 : 0] >= 0 ||
                        npan < kTuneMinPanels) &&
                       (ctx->far_variant[precision == LBL_PREC_SPLIT ? 1 : 0] >= 0 ||
                        nwin < kTuneMinWindows);
    if (graph && ctx->nslot + 1 >= lbl_ctx::kStatSlots) {
      CK(cudaStreamSynchronize(ctx->stream));
      const int rcs = finish_od(ctx);
      if (rcs) return rcs;
    }
    int rc2 = upload_batch(ctx, B, graph);
    if (rc2) return rc2;
    // results of this group bound for pageable memory go to bounce[bi]
    Bounce& bb = bounce[bi];
    size_t need = 0;
    for (int p : cur_prof)
      need += (size_t)(offsets[p + 1] - offsets[p]) * ((rad_host ? 1 : 0) + (tr_host ? 1 : 0));
    if (need) {
      rc2 = bounce_flush(ctx, bb);
      if (rc2) return rc2;
      if (need > bb.cap) {
        if (bb.buf) cudaFreeHost(bb.buf);
        bb.buf = nullptr;
        bb.cap = 0;
        void* hp = nullptr;
        CK(cudaMallocHost(&hp, need * sizeof(double)));
        bb.buf = static_cast<double*>(hp);
        bb.cap = need;
      }
      if (!bb.ev) CK(cudaEventCreateWithFlags(&bb.ev, cudaEventDisableTiming));
    }
    // The group is captured on the context's own capture stream (the
    // caller's stream may be the legacy default stream, which cannot be
    // captured); the graph is then launched on the caller's stream.
    cudaStream_t user = ctx->stream;
    if (graph) {
      CK(cudaStreamBeginCapture(ctx->gstream, cudaStreamCaptureModeThreadLocal));
      ctx->stream = ctx->gstream;
    }
    // ends a capture that an error interrupted, so the streams stay usable
    auto abandon = [&](int code) {
      if (graph) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(ctx->gstream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        ctx->stream = user;
      }
      return code;
    };
    if (graph && (rc2 = enqueue_upload(ctx, B))) return abandon(rc2);
    if ((rc2 = run_od(ctx, R, B, precision))) return abandon(rc2);
    size_t boff = 0;
    int l0 = 0;
    for (int p : cur_prof) {
      const int n = (int)(lay0[p + 1] - lay0[p]);
      const size_t np = (size_t)(offsets[p + 1] - offsets[p]);
      OutSink sink{rad + offsets[p], tr ? tr + offsets[p] : nullptr, rad_dev ? 1 : 0,
                   tr_dev ? 1 : 0};
      if (rad_host) {
        bb.pend.push_back({rad + offsets[p], boff, np});
        sink.rad = bb.buf + boff;
        sink.rad_dev = 0;
        boff += np;
      }
      if (tr_host) {
        bb.pend.push_back({tr + offsets[p], boff, np});
        sink.tr = bb.buf + boff;
        sink.tr_dev = 0;
        boff += np;
      }
      int res = 0;
      rc2 = run_merge(ctx, R, layers + lay0[p], B, n, &res, precision, &sink, l0);
      if (rc2) return abandon(rc2);
      l0 += n;
    }
    if (graph) {
      cudaGraph_t g = nullptr;
      ctx->stream = user;
      CK(cudaStreamEndCapture(ctx->gstream, &g));
      cudaGraphExecUpdateResultInfo info;
      if (!ctx->gexec || cudaGraphExecUpdate(ctx->gexec, g, &info) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
        ctx->gexec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ctx->gexec, g, 0);
        if (ie != cudaSuccess) {
          cudaGraphDestroy(g);
          ctx->gexec = nullptr;
          return fail(ctx, LBL_E_CUDA, std::string("cudaGraphInstantiate: ") +
                                           cudaGetErrorString(ie));
        }
      }
      cudaGraphDestroy(g);
      CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
      // the staging image may be rewritten once the graph has run
      CK(cudaEventRecord(ctx->stage_ev[B.stage_k], ctx->stream));
      ctx->stage_ev_set[B.stage_k] = true;
      ctx->stage("graph_groups").launches += 1;
    }
    if (need) CK(cudaEventRecord(bb.ev, ctx->stream));
    bi ^= 1;
    cur_prof.clear();
    cur_bytes = 0;
    t_host = std::chrono::steady_clock::now();
    return LBL_OK;
  };
  for (int p = 0; p < nprof && rc == LBL_OK; p++) {
    std::vector<LayerPlan> plans;
    const int n = (int)(lay0[p + 1] - lay0[p]);
    rc = plan_layers(ctx, R, layers + lay0[p], n, R.jrad, nullptr, plans);
    if (rc) break;
    size_t bytes = 0;
    for (const LayerPlan& P : plans) bytes += layer_arena_bytes(P.d);
    if (!cur_prof.empty() && cur_bytes + bytes > budget) {
      rc = flush();
      if (rc) break;
    }
    if (bytes > budget) {
      rc = fail(ctx, LBL_E_NOMEM, "profile " + std::to_string(p) + " needs " +
                                      std::to_string(bytes >> 20) + " MiB of work space, " +
                                      std::to_string(budget >> 20) + " MiB available");
      break;
    }
    for (LayerPlan& P : plans) cur.push_back(std::move(P));
    cur_prof.push_back(p);
    cur_bytes += bytes;
  }
  if (rc == LBL_OK) rc = flush();
  if (ctx->prof) ctx->stage("host_plan").ms += host_ms;
  cudaError_t se = cudaStreamSynchronize(ctx->stream);
  for (Bounce& b : bounce) {
    if (rc == LBL_OK && se == cudaSuccess) rc = bounce_flush(ctx, b);
    if (b.buf) cudaFreeHost(b.buf);
    if (b.ev) cudaEventDestroy(b.ev);
  }
  if (rc) return rc;
  if (se != cudaSuccess) return fail(ctx, LBL_E_CUDA, cudaGetErrorString(se));
  harvest(ctx);
  return finish_od(ctx);
}

}  // namespace

namespace {

int check_jac_args(lbl_ctx* ctx, const lbl_run* run, const lbl_layer* layers,
                   const int32_t* nlay, int nprof, const int32_t* mols, int nq, int mode) {
  int rc = check_run(ctx, run);
  if (rc) return rc;
  if (!layers || !nlay || nprof < 1 || nq < 0 || nq >= kJacMaxParams || (nq > 0 && !mols))
    return fail(ctx, LBL_E_ARG, "Jacobians: bad argument");
  if (mode != LBL_JAC_CENTRAL && mode != LBL_JAC_REFERENCE)
    return fail(ctx, LBL_E_ARG, "Jacobians: mode must be LBL_JAC_CENTRAL or LBL_JAC_REFERENCE");
  if (run->iemit != 1 || run->ipathl != 1 || run->bndrfl != 0.)
    return fail(ctx, LBL_E_ARG,
                "Jacobians: upwelling radiance only (IEMIT=1, IPATHL=1, no reflectivity)");
  for (int p = 0; p < nprof; p++)
    if (nlay[p] < 1) return fail(ctx, LBL_E_ARG, "Jacobians: profile without layers");
  for (int k = 0; k < nq; k++)
    if (mols[k] < 1 || mols[k] > LBL_WKDIM)
      return fail(ctx, LBL_E_ARG, "Jacobians: molecule number out of range");
  return LBL_OK;
}

// Device results of jac_profile (pointers into the Jacobian work space).
struct JacOut {
  double* rad = nullptr;   // TOA radiance on the top grid (npts)
  double* rows = nullptr;  // rows (k - k0)*nlay*npts + l*npts + i
  int64_t npts = 0;
  int nlay = 0;
  std::vector<double> top_vft;     // panel origins of the top layer
  double top_dv = 0.;
  double* chan_rad = nullptr;      // channel means (jac_channels)
  double* chan_rows = nullptr;
};

// Sizes of one profile's Jacobian work space for nk parameters at once.
struct JacSizes {
  int64_t ntot, npts;
  int a;  // layers a..nlay-1 share the top grid
  size_t bytes(int nk, int nlay, int64_t nchan) const {
    const size_t rows = (size_t)nk * nlay * npts, low = (size_t)nk * std::max(a, 1) * npts;
    const size_t chan = nchan > 0 ? (size_t)(nk * nlay + 2) * nchan + 32 : 0;
    return 8 * ((size_t)nk * ntot + ntot + rows + 2 * low + 4 * (size_t)npts + nlay + chan) +
           16 * 256;
  }
};

JacSizes jac_sizes(const lbl_run& R, const lbl_layer* layers, int nlay) {
  JacSizes z{0, layer_npts(R, layers[nlay - 1].dv), 0};
  for (int l = 0; l < nlay; l++) {
    z.ntot += layer_npts(R, layers[l].dv);
    if (l > 0 && layers[l].dv != layers[l - 1].dv) z.a = l;
  }
  return z;
}

// Parameters one profile can take at once within the memory budget (the
// optical-depth passes are recomputed for each chunk of parameters when not
// all fit); 0 when even one does not.
int jac_chunk(lbl_ctx* ctx, const lbl_run& R, const lbl_layer* layers, int nlay, int np,
              int64_t nchan) {
  const JacSizes z = jac_sizes(R, layers, nlay);
  // arena of one pass: estimated from the layer grids and the line count
  const size_t arena = (size_t)z.ntot * 16 + (size_t)nlay * ctx->h_vnu.size() * 200 +
                       ((size_t)64 << 20);
  size_t avail;
  const size_t held = ctx->mem.used - std::min(ctx->mem.used, ctx->arena.cap + ctx->jac_cap);
  if (ctx->mem.limit) {
    avail = ctx->mem.limit > held ? ctx->mem.limit - held : 0;
  } else {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    avail = fr + ctx->arena.cap + ctx->jac_cap;
    const size_t keep = (size_t)2 << 30;
    avail = avail > keep ? avail - keep : 0;
  }
  avail = avail > arena ? avail - arena : 0;
  for (int nk = np; nk >= 1; nk--)
    if (z.bytes(nk, nlay, nchan) <= avail) return nk;
  return 0;
}

// One profile's TOA radiance and the Jacobian rows of parameters [k0, k1)
// (0: temperature, k: molecule mols[k-1]) on its top grid, left in the
// Jacobian work space.  Every step is queued on the stream without a host
// wait (the caller synchronises), so the host plans each optical-depth pass
// while the device runs the previous one.
//   LBL_JAC_CENTRAL:   dtau/dp by central differences of whole-profile
//                      optical depths (T +-0.1 K, amount +-1 %; a layer's
//                      depth depends only on its own parameters, so one pass
//                      serves every layer), merged with the exact derivative
//                      of EMIN/EMINIT/RADNN;
//   LBL_JAC_REFERENCE: the reference's analytic-Jacobian definitions
//                      (src/lblrtm.f90:2855-3067): one pass at T + 1 K and one
//                      per molecule with that molecule alone (other amounts
//                      zero, WK(7) added to WBROAD), merged by the
//                      TDERIVup/QDERIVup rows (src/xmerge.f90:5786-6144).
// Each layer's row is carried to the top through the later layers' regrid
// and transmittance.
int jac_profile(lbl_ctx* ctx, const lbl_run& R, lbl_layer* layers, int nlay,
                const int32_t* mols, int k0, int k1, int mode, int precision, int64_t nchan,
                JacOut& o) {
  const int nk = k1 - k0;
  const JacSizes z = jac_sizes(R, layers, nlay);
  const int64_t npts = z.npts, ntot = z.ntot;
  const int a = z.a;
  std::vector<int64_t> off(nlay + 1, 0);
  for (int l = 0; l < nlay; l++) off[l + 1] = off[l] + layer_npts(R, layers[l].dv);
  const size_t need = z.bytes(nk, nlay, nchan);
  if (need > ctx->jac_cap) {
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->mem.release(ctx->jac_mem, ctx->jac_cap);
    ctx->jac_mem = nullptr;
    ctx->jac_cap = 0;
    void* m = nullptr;
    if (ctx->mem.alloc(&m, need) != cudaSuccess) {
      // the arena of an earlier batch may hold the room: release it (the
      // passes below reserve what they need) and try once more
      ctx->mem.release(ctx->arena.base, ctx->arena.cap);
      ctx->arena.base = nullptr;
      ctx->arena.cap = 0;
      CK(ctx->mem.alloc(&m, need));
    }
    ctx->jac_mem = static_cast<char*>(m);
    ctx->jac_cap = need;
  }
  size_t used = 0;
  auto take = [&](size_t n) {
    used = (used + 255) & ~size_t(255);
    double* p = reinterpret_cast<double*>(ctx->jac_mem + used);
    used += n * 8;
    return p;
  };
  const size_t n_rows = (size_t)nk * nlay * npts, n_low = (size_t)nk * std::max(a, 1) * npts;
  double* dtau = take((size_t)nk * ntot);
  double* tmp = take(ntot);
  double* rows = take(n_rows);
  double* low[2] = {take(n_low), take(n_low)};
  double* rt[4] = {take(npts), take(npts), take(npts), take(npts)};
  int64_t* d_off = reinterpret_cast<int64_t*>(take(nlay));
  // channel means, then the channel bounds (nchan + 1 entries)
  o.chan_rows = take(nchan > 0 ? (size_t)nk * nlay * nchan + nchan + 9 : 0);
  o.chan_rad = take(nchan > 0 ? (size_t)nchan + 8 : 0);
  cudaStream_t s = ctx->stream;
  int rc;
  std::vector<lbl_layer> Lp(layers, layers + nlay), Lm(layers, layers + nlay);
  const double dT = 0.1, dq = 0.01;
  for (int k = k0; k < k1; k++) {
    double* dst = dtau + (size_t)(k - k0) * ntot;
    for (int l = 0; l < nlay; l++) {
      Lp[l] = layers[l];
      Lm[l] = layers[l];
      if (mode == LBL_JAC_CENTRAL) {
        if (k == 0) {
          Lp[l].tave += dT;
          Lm[l].tave -= dT;
        } else {
          Lp[l].wk[mols[k - 1] - 1] *= 1. + dq;
          Lm[l].wk[mols[k - 1] - 1] *= 1. - dq;
        }
      } else if (k == 0) {
        Lp[l].tave += 1.;
      } else {
        const int m = mols[k - 1];
        for (int j = 0; j < LBL_WKDIM; j++) Lp[l].wk[j] = 0.;
        Lp[l].wk[m - 1] = layers[l].wk[m - 1];
        Lp[l].wbroad = layers[l].wbroad + layers[l].wk[6];
      }
    }
    const int nside = mode == LBL_JAC_CENTRAL ? 2 : 1;
    for (int side = 0; side < nside; side++) {
      Batch Bs;
      // every pass keeps the nominal JRAD chain of the layers
      rc = prepare_batch(ctx, R, side ? Lm.data() : Lp.data(), nlay, R.jrad, nullptr, Bs,
                         layers);
      if (rc) return rc;
      rc = run_od(ctx, R, Bs, precision);
      if (rc) return rc;
      CK(cudaMemcpyAsync(side ? tmp : dst, Bs.w.od, 8 * ntot, cudaMemcpyDeviceToDevice, s));
    }
    if (mode == LBL_JAC_CENTRAL) {
      const double h = k == 0 ? 2. * dT : std::log(1. + dq) - std::log(1. - dq);
      CK(launch_jac_diff(dst, tmp, ntot, 1. / h, s));
    }
  }
  // nominal optical depths, kept in the batch for the merge
  Batch B;
  rc = prepare_batch(ctx, R, layers, nlay, R.jrad, nullptr, B);
  if (rc) return rc;
  rc = run_od(ctx, R, B, precision);
  if (rc) return rc;
  {
    int64_t* hoff = nullptr;
    rc = small_pinned(ctx, 8 * (size_t)nlay, reinterpret_cast<void**>(&hoff));
    if (rc) return rc;
    for (int l = 0; l < nlay; l++) hoff[l] = B.ld[l].off_od;
    CK(cudaMemcpyAsync(d_off, hoff, 8 * nlay, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(ctx->small_ev, s));
  }
  int cur = 0;
  {
    StageTimer t(ctx, "jacobian", 0);
    int lc = 0;
    double dv_old = 0.;
    int64_t n_old = 0;
    for (int l = 0; l < nlay; l++) {
      const LayerDev& d = B.ld[l];
      if (l > 0 && d.dv > dv_old) return fail(ctx, LBL_E_ITYPE, " RADMRG; ITYPE LT 0 ");
      // carry the rows of layers below l onto layer l's grid
      if (l > 0 && l <= a) {
        for (int k = 0; k < nk; k++)
          CK(launch_jac_prop(B.d_ld + l, B.w.od + d.off_od, d.npts, dv_old, n_old,
                             low[lc] + (size_t)k * a * npts, low[lc ^ 1] + (size_t)k * a * npts,
                             npts, l, s));
        lc ^= 1;
      }
      double* dp[kJacMaxParams];
      const double* tp[kJacMaxParams];
      for (int k = 0; k < nk; k++) {
        dp[k] = (l < a) ? low[lc] + ((size_t)k * a + l) * npts
                        : rows + ((size_t)k * nlay + l) * npts;
        tp[k] = dtau + (size_t)k * ntot + off[l];
      }
      const int nxt = cur ^ 2;
      const double tbnd = (l == 0) ? R.tmpbnd : 0.;
      CK(launch_jac_layer(B.d_ld + l, B.w.vft + d.off_panel, B.w.od + d.off_od, d.npts, l == 0,
                          dv_old, n_old, rt[cur], rt[cur + 1], rt[nxt], rt[nxt + 1], tbnd,
                          R.bndemi, layers[l].tzu, dp, tp, nk, mode, k0, s));
      cur = nxt;
      dv_old = d.dv;
      n_old = d.npts;
    }
    CK(launch_jac_top(B.w.od, d_off, nlay, a, nk, npts, rows, low[lc], s));
  }
  o.rad = rt[cur];
  o.rows = rows;
  o.npts = npts;
  o.nlay = nlay;
  o.top_vft = B.plans[nlay - 1].vft;
  o.top_dv = B.ld[nlay - 1].dv;
  return LBL_OK;
}

// Means of the radiance and of `nrows` rows over channels [V1 + c dv_chan,
// V1 + (c+1) dv_chan), c < nchan, of the top grid (the points of a channel
// are those whose wavenumber lies in it).
int jac_channels(lbl_ctx* ctx, const lbl_run& R, JacOut& o, int nrows, double dv_chan,
                 int64_t nchan) {
  int64_t* cb = nullptr;
  int rc = small_pinned(ctx, 8 * (size_t)(nchan + 1), reinterpret_cast<void**>(&cb));
  if (rc) return rc;
  const double DV = o.top_dv;
  auto vpt = [&](int64_t f) {
    const int64_t p = f / 2400;
    return (o.top_vft[p] + double(33 - 1) * DV) + double(f - 2400 * p) * DV;
  };
  for (int64_t c = 0; c <= nchan; c++) {
    const double vc = R.v1 + double(c) * dv_chan;
    int64_t lo = 0, hi = o.npts;
    while (lo < hi) {
      const int64_t m = (lo + hi) / 2;
      if (vpt(m) < vc) lo = m + 1;
      else hi = m;
    }
    cb[c] = lo;
  }
  for (int64_t c = 0; c < nchan; c++)
    if (cb[c + 1] <= cb[c]) return fail(ctx, LBL_E_ARG, "a channel holds no grid point");
  // the bounds go in the rows' space, which the channel means no longer need
  int64_t* d_cb = reinterpret_cast<int64_t*>(o.chan_rows + (size_t)nrows * nchan);
  static_assert(sizeof(int64_t) == sizeof(double), "bounds stored in a double array");
  CK(cudaMemcpyAsync(d_cb, cb, 8 * (nchan + 1), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaEventRecord(ctx->small_ev, ctx->stream));
  CK(launch_chan_mean(o.rad, o.npts, 1, d_cb, nchan, o.chan_rad, ctx->stream));
  CK(launch_chan_mean(o.rows, o.npts, nrows, d_cb, nchan, o.chan_rows, ctx->stream));
  return LBL_OK;
}

}  // namespace

// ==========================================================================
extern "C" {

int lbl_ctx_create(int device, lbl_ctx** out) {
  if (!out) return LBL_E_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LBL_E_NODEVICE;
  }
  if (device < 0 || device >= ndev) return LBL_E_ARG;
  lbl_ctx* ctx = new lbl_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return LBL_E_CUDA;
  }
  upload_voicon();
  init_kernel_attributes();
  void* hs = nullptr;
  const size_t slot_bytes = sizeof(lbl_ctx::StatSlot) * lbl_ctx::kStatSlots;
  if (cudaMallocHost(&hs, slot_bytes) != cudaSuccess) {
    delete ctx;
    return LBL_E_NOMEM;
  }
  std::memset(hs, 0, slot_bytes);
  ctx->h_slots = static_cast<lbl_ctx::StatSlot*>(hs);
  if (cudaEventCreateWithFlags(&ctx->stage_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->stage_ev[1], cudaEventDisableTiming) != cudaSuccess) {
    cudaFreeHost(hs);
    delete ctx;
    return LBL_E_CUDA;
  }
  ShapeTables* t = new ShapeTables;
  build_shape_tables(t);
  const size_t nd = kNfmx + 1;
  char* mem = nullptr;
  // FP64 tables, the packed R1 records, and their FP32 copies
  if (cudaMalloc(&mem, 13 * nd * sizeof(double) + 4096) != cudaSuccess) {
    delete t;
    delete ctx;
    return LBL_E_NOMEM;
  }
  ctx->shape_mem = mem;
  const double* src[5] = {t->f1, t->f2, t->f3, t->fg, t->xver};
  double* dd = reinterpret_cast<double*>(mem);
  double* pk = dd + ((5 * nd + 3) & ~size_t(3));  // records 32-byte aligned
  for (int k = 0; k < 5; k++)
    cudaMemcpy(dd + k * nd, src[k], nd * sizeof(double), cudaMemcpyHostToDevice);
  std::vector<double> rec(4 * nd, 0.);
  for (size_t i = 0; i < nd; i++) {
    rec[4 * i] = t->f1[i];
    rec[4 * i + 1] = t->fg[i];
    rec[4 * i + 2] = t->xver[i];
  }
  cudaMemcpy(pk, rec.data(), 4 * nd * sizeof(double), cudaMemcpyHostToDevice);
  // FP32: F1, FG, XVER, 0 per index (16-byte records), then F2 and F3
  float* fk = reinterpret_cast<float*>(pk + 4 * nd);
  std::vector<float> rec32(4 * nd, 0.f), f23(2 * nd);
  for (size_t i = 0; i < nd; i++) {
    rec32[4 * i] = (float)t->f1[i];
    rec32[4 * i + 1] = (float)t->fg[i];
    rec32[4 * i + 2] = (float)t->xver[i];
    f23[i] = (float)t->f2[i];
    f23[nd + i] = (float)t->f3[i];
  }
  cudaMemcpy(fk, rec32.data(), 4 * nd * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(fk + 4 * nd, f23.data(), 2 * nd * sizeof(float), cudaMemcpyHostToDevice);
  delete t;
  ctx->sh = DevShapes{dd, dd + nd, dd + 2 * nd, dd + 3 * nd, dd + 4 * nd, pk,
                      reinterpret_cast<const float4*>(fk), fk + 4 * nd, fk + 5 * nd};
  if (cudaGetLastError() != cudaSuccess) {
    lbl_ctx_destroy(ctx);
    return LBL_E_CUDA;
  }
  *out = ctx;
  return LBL_OK;
}

int lbl_ctx_destroy(lbl_ctx* ctx) {
  if (!ctx) return LBL_E_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->h_slots) cudaFreeHost(ctx->h_slots);
  for (int k = 0; k < 2; k++) {
    if (ctx->stage_host[k]) cudaFreeHost(ctx->stage_host[k]);
    if (ctx->stage_ev[k]) cudaEventDestroy(ctx->stage_ev[k]);
  }
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  for (int k = 0; k < lbl_ctx::kSmallRing; k++) {
    if (ctx->small_host[k]) cudaFreeHost(ctx->small_host[k]);
    if (ctx->small_evs[k]) cudaEventDestroy(ctx->small_evs[k]);
  }
  ctx->mem.release(ctx->jac_mem, ctx->jac_cap);
  ctx->mem.release(ctx->line_mem, ctx->line_cap);
  if (ctx->shape_mem) cudaFree(ctx->shape_mem);
  ctx->mem.release(ctx->ck_mem, ctx->ck_bytes);
  ctx->mem.release(ctx->arena.base, ctx->arena.cap);
  for (int k = 0; k < 4; k++) ctx->mem.release(ctx->mbuf[k], ctx->mcap * sizeof(double));
  for (auto e : ctx->event_pool) cudaEventDestroy(e);
  for (auto e : ctx->cev)
    if (e) cudaEventDestroy(e);
  if (ctx->cstream) cudaStreamDestroy(ctx->cstream);
  if (ctx->gstream) cudaStreamDestroy(ctx->gstream);
  delete ctx;
  return LBL_OK;
}

const char* lbl_last_error(const lbl_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int lbl_set_stream(lbl_ctx* ctx, void* stream) {
  if (!ctx) return LBL_E_ARG;
  ctx->stream = reinterpret_cast<cudaStream_t>(stream);
  return LBL_OK;
}

}  // extern "C"

namespace {
// The host-side checks of a line list (the conditions RDLIN assumes or
// STOPs on): ascending centres, coupling records after their line, TAPE3
// panels of at most 250 records.  Fills the searchable centres (coupling
// records repeat the previous line's centre) and the panel starts.
int validate_lines(lbl_ctx* ctx, const lbl_lines* L, std::vector<double>* vs_out,
                   std::vector<int64_t>* bs_out) {
  if (!L || L->n < 0) return fail(ctx, LBL_E_ARG, "bad lines");
  const int64_t n = L->n;
  if (n >= (int64_t(1) << 31) - 8) return fail(ctx, LBL_E_RANGE, "more than 2^31 line records");
  if (n > 0 && (!L->vnu || !L->sp || !L->alfa || !L->epp || !L->mol || !L->hwhms ||
                !L->tmpalf || !L->pshift || !L->iflg))
    return fail(ctx, LBL_E_ARG, "NULL line array");
  // Line-coupling records (IFLG < 0) follow their line and carry Y/G
  // coefficients in the centre field (RDLIN :818-837, LNCOR1 :1039-1061):
  // they are skipped in the order check, and the searchable copy of the
  // centres repeats the previous line's there.
  std::vector<double>& vs = *vs_out;
  vs.assign(L->vnu, L->vnu + n);
  {
    double last = 0.;
    bool have = false;
    for (int64_t i = 0; i < n; i++) {
      if (L->iflg[i] < 0) {
        if (i == 0 || (L->iflg[i - 1] != 1 && L->iflg[i - 1] != 3))
          return fail(ctx, LBL_E_FORMAT,
                      "coupling record without a coupled line at record " + std::to_string(i));
        vs[i] = last;
        continue;
      }
      if (have && !(L->vnu[i] >= last))
        return fail(ctx, LBL_E_UNSORTED,
                    "line centres not ascending at record " + std::to_string(i));
      last = L->vnu[i];
      have = true;
    }
    for (int64_t i = 0; i < n; i++)
      if ((L->iflg[i] == 1 || L->iflg[i] == 3) && (i + 1 >= n || L->iflg[i + 1] >= 0))
        return fail(ctx, LBL_E_FORMAT,
                    "coupled line without its coefficient record at record " + std::to_string(i));
  }
  std::vector<int64_t>& bs = *bs_out;
  bs.clear();
  if (L->nblock > 0 && L->block_start) {
    bs.assign(L->block_start, L->block_start + L->nblock + 1);
    if (bs.front() != 0 || bs.back() != n) return fail(ctx, LBL_E_ARG, "block_start must span 0..n");
  } else {
    for (int64_t s = 0; s < n; s += 250) bs.push_back(s);
    bs.push_back(n);
  }
  for (size_t b = 0; b + 1 < bs.size(); b++) {
    if (bs[b + 1] < bs[b]) return fail(ctx, LBL_E_ARG, "block_start not increasing");
    if (bs[b + 1] - bs[b] > 250) return fail(ctx, LBL_E_NREC, "RDLIN; NREC GT LIMIN");
  }
  return LBL_OK;
}
}  // namespace

extern "C" {

int lbl_lines_upload(lbl_ctx* ctx, const lbl_lines* L) {
  if (!ctx) return LBL_E_ARG;
  std::vector<double> vs;
  std::vector<int64_t> bs;
  const int vrc = validate_lines(ctx, L, &vs, &bs);
  if (vrc) return vrc;
  const int64_t n = L->n;
  ctx->h_vnu = vs;
  ctx->h_sp.assign(L->sp, L->sp + n);
  ctx->h_pshift.assign(L->pshift, L->pshift + n);
  ctx->h_mol.assign(L->mol, L->mol + n);
  ctx->h_iflg.assign(L->iflg, L->iflg + n);
  ctx->h_bs = bs;
  ctx->max_abs_pshift = 0.;
  for (int64_t i = 0; i < n; i++)
    ctx->max_abs_pshift = std::max(ctx->max_abs_pshift, std::fabs((double)L->pshift[i]));
  cudaSetDevice(ctx->device);
  const size_t nn = (size_t)std::max<int64_t>(n, 1) + 2;  // +2: coupling record reads
  size_t bytes = nn * (2 * 8 + 6 * 4 + 2 * 4) + bs.size() * 8 + 16 * 256;  // 11 aligned arrays
  // the line buffer grows only; work already queued on the stream that
  // reads the old lines is ordered before the copies below
  if (!ctx->line_mem || bytes > ctx->line_cap) {
    if (ctx->line_mem) {
      CK(cudaStreamSynchronize(ctx->stream));
      ctx->mem.release(ctx->line_mem, ctx->line_cap);
    }
    ctx->line_mem = nullptr;
    ctx->line_cap = 0;
    ctx->have_lines = false;
    void* nm = nullptr;
    CK(ctx->mem.alloc(&nm, bytes));
    ctx->line_mem = nm;
    ctx->line_cap = bytes;
  }
  char* m = static_cast<char*>(ctx->line_mem);
  CK(cudaMemsetAsync(m, 0, bytes, ctx->stream));
  size_t off = 0;
  auto take = [&](size_t b) {
    off = (off + 255) & ~size_t(255);
    char* p = m + off;
    off += b;
    return p;
  };
  DevLines d;
  d.vnu = reinterpret_cast<double*>(take(nn * 8));
  d.vraw = reinterpret_cast<double*>(take(nn * 8));
  d.sp = reinterpret_cast<float*>(take(nn * 4));
  d.alfa = reinterpret_cast<float*>(take(nn * 4));
  d.epp = reinterpret_cast<float*>(take(nn * 4));
  d.hwhms = reinterpret_cast<float*>(take(nn * 4));
  d.tmpalf = reinterpret_cast<float*>(take(nn * 4));
  d.pshift = reinterpret_cast<float*>(take(nn * 4));
  d.mol = reinterpret_cast<int32_t*>(take(nn * 4));
  d.iflg = reinterpret_cast<int32_t*>(take(nn * 4));
  d.bs = reinterpret_cast<int64_t*>(take(bs.size() * 8));
  d.n = n;
  d.nblk = (int64_t)bs.size() - 1;
  cudaStream_t st = ctx->stream;
  if (n > 0) {
    CK(cudaMemcpyAsync((void*)d.vnu, ctx->h_vnu.data(), n * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.vraw, L->vnu, n * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.sp, L->sp, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.alfa, L->alfa, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.epp, L->epp, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.hwhms, L->hwhms, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.tmpalf, L->tmpalf, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.pshift, L->pshift, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.mol, L->mol, n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void*)d.iflg, L->iflg, n * 4, cudaMemcpyHostToDevice, st));
  }
  CK(cudaMemcpyAsync((void*)d.bs, bs.data(), bs.size() * 8, cudaMemcpyHostToDevice, st));
  // the caller's arrays (and bs) must outlive the copies
  CK(cudaStreamSynchronize(st));
  ctx->dl = d;
  ctx->have_lines = true;
  return LBL_OK;
}

int lbl_mtckd_upload(lbl_ctx* ctx, const lbl_mtckd* T) {
  if (!ctx || !T || T->n < 4 || !T->self_absco_ref || !T->for_absco_ref || !T->self_texp ||
      !(T->dv > 0.))
    return fail(ctx, LBL_E_ARG, "bad continuum table");
  cudaSetDevice(ctx->device);
  ctx->mem.release(ctx->ck_mem, ctx->ck_bytes);
  ctx->ck_mem = nullptr;
  ctx->have_ck = false;
  void* vm = nullptr;
  CK(ctx->mem.alloc(&vm, 3 * T->n * sizeof(double)));
  ctx->ck_bytes = 3 * T->n * sizeof(double);
  double* m = static_cast<double*>(vm);
  CK(cudaMemcpy(m, T->self_absco_ref, T->n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m + T->n, T->for_absco_ref, T->n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m + 2 * T->n, T->self_texp, T->n * 8, cudaMemcpyHostToDevice));
  ctx->ck_mem = m;
  CK(cudaMemcpy(m, T->self_absco_ref, T->n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m + T->n, T->for_absco_ref, T->n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m + 2 * T->n, T->self_texp, T->n * 8, cudaMemcpyHostToDevice));
  ctx->ck = DevMtckd{m, m + T->n, m + 2 * T->n, T->v0, T->dv, T->ref_press, T->ref_temp, T->n};
  ctx->have_ck = true;
  return LBL_OK;
}

int lbl_dv_rule(const lbl_run* run, lbl_layer* layers, int32_t nlay) {
  if (!run || !layers || nlay < 1) return LBL_E_ARG;
  std::string e;
  return dv_rule(*run, layers, nlay, &e);
}

int64_t lbl_layer_npts(const lbl_run* run, double dv) {
  if (!run || !(dv > 0.) || !(run->v2 > run->v1)) return -1;
  return layer_npts(*run, dv);
}

int lbl_layer_od(lbl_ctx* ctx, const lbl_run* run, const lbl_layer* layer, int32_t* jrad,
                 double* od, int64_t npts, int32_t precision) {
  if (!ctx) return LBL_E_ARG;
  int rc = check_run(ctx, run);
  if (rc) return rc;
  if (!layer || !jrad || !od) return fail(ctx, LBL_E_ARG, "NULL argument");
  cudaSetDevice(ctx->device);
  if (layer_npts(*run, layer->dv) != npts) return fail(ctx, LBL_E_ARG, "npts does not match the layer grid");
  Batch B;
  int jout = 0;
  rc = prepare_batch(ctx, *run, layer, 1, *jrad, &jout, B);
  if (rc) return rc;
  rc = run_od(ctx, *run, B, precision);
  if (rc) return rc;
  rc = copy_out(ctx, od, B.w.od, sizeof(double) * npts);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  harvest(ctx);
  rc = finish_od(ctx);
  if (rc) return rc;
  *jrad = jout;
  return LBL_OK;
}

int lbl_merge_layer(lbl_ctx* ctx, const lbl_run* run, const lbl_layer* layer, int32_t first,
                    double dv_old, const double* rad_in, const double* tr_in, int64_t n_old,
                    const double* od, double* rad_out, double* tr_out, int64_t n_new) {
  if (!ctx) return LBL_E_ARG;
  // bit 0: the first layer (EMINIT); bit 1: the last layer (looking up, the
  // boundary beyond it)
  const bool last = (first & 2) != 0;
  first &= 1;
  int rc = check_run(ctx, run);
  if (rc) return rc;
  if (!layer || !od || !rad_out || (run->iemit == 1 && !tr_out)) return fail(ctx, LBL_E_ARG, "NULL argument");
  if (!first && (!rad_in || (run->iemit == 1 && !tr_in) || n_old < 1))
    return fail(ctx, LBL_E_ARG, "accumulated input missing");
  if (!first && layer->dv > dv_old) return fail(ctx, LBL_E_ITYPE, " RADMRG; ITYPE LT 0 ");
  cudaSetDevice(ctx->device);
  if (layer_npts(*run, layer->dv) != n_new) return fail(ctx, LBL_E_ARG, "n_new does not match the layer grid");
  HostLines H{ctx->h_vnu.data(), ctx->h_sp.data(), ctx->h_pshift.data(), ctx->h_mol.data(),
              ctx->h_iflg.data(), (int64_t)ctx->h_vnu.size(), ctx->h_bs.data(),
              (int64_t)ctx->h_bs.size() - 1, ctx->max_abs_pshift};
  LayerPlan P;
  std::string e;
  rc = plan_layer(*run, *layer, run->jrad, H, &P, &e);
  if (rc) return fail(ctx, rc, e);
  const size_t nn = (size_t)std::max(n_new, n_old) + 8;
  rc = ensure_merge_buffers(ctx, nn);
  if (rc) return rc;
  CK(ctx->arena.reserve(sizeof(LayerDev) + P.vft.size() * 8 + n_new * 8 + 4096, ctx->mem));
  ctx->arena.reset();
  LayerDev* dL = ctx->arena.take<LayerDev>(1);
  double* dv = ctx->arena.take<double>(P.vft.size());
  double* dod = ctx->arena.take<double>(n_new);
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(dL, &P.d, sizeof(LayerDev), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dv, P.vft.data(), P.vft.size() * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dod, od, n_new * 8, cudaMemcpyDefault, s));
  if (!first) {
    CK(cudaMemcpyAsync(ctx->mbuf[0], rad_in, n_old * 8, cudaMemcpyDefault, s));
    if (run->iemit == 1) CK(cudaMemcpyAsync(ctx->mbuf[1], tr_in, n_old * 8, cudaMemcpyDefault, s));
  }
  const double refl = (run->iemit == 1 && run->ipathl == 1 && run->bndrfl > 0.) ? run->bndrfl : 0.;
  if (run->iemit == 1 && (run->ipathl == 2 || refl > 0.) && !(layer->tzl > 0.))
    return fail(ctx, LBL_E_ARG, "the tangent path and the reflected atmosphere need TZL > 0");
  const double tbnd = (first && run->ipathl == 1) ? run->tmpbnd : 0.;
  const bool down = run->ipathl == 3;
  const double tbnd_last = (down && last && !first) ? run->tmpbnd : 0.;
  CK(launch_merge(dL, dv, dod, n_new, first, dv_old, n_old, ctx->mbuf[0], ctx->mbuf[1],
                  ctx->mbuf[2], ctx->mbuf[3], tbnd, run->bndemi, run->iemit,
                  down ? layer->tzl : layer->tzu, s, LBL_PREC_FP64, down ? 1 : 0, tbnd_last,
                  (run->ipathl == 2 || refl > 0.) ? layer->tzl : 0., refl));
  CK(cudaMemcpyAsync(rad_out, ctx->mbuf[2], n_new * 8, cudaMemcpyDefault, s));
  if (tr_out) CK(cudaMemcpyAsync(tr_out, ctx->mbuf[3], n_new * 8, cudaMemcpyDefault, s));
  CK(cudaStreamSynchronize(s));
  return LBL_OK;
}

int64_t lbl_pnlint_npts(const lbl_run* run, double dv, double dvout) {
  if (!run || !(run->v2 > run->v1) || run->v2 - run->v1 > 2020. || !(run->v1 > 0.))
    return -LBL_E_ARG;
  PnlPlan P;
  std::string e;
  int rc = pnlint_plan(*run, dv, dvout, &P, &e);
  if (rc) return -rc;
  return P.n_out;
}

int lbl_pnlint(lbl_ctx* ctx, const lbl_run* run, double dv, double dvout, const double* od_in,
               int64_t n_in, double* od_out, int64_t n_out) {
  if (!ctx) return LBL_E_ARG;
  if (!run || !od_in || !od_out) return fail(ctx, LBL_E_ARG, "NULL argument");
  if (!(run->v2 > run->v1) || run->v2 - run->v1 > 2020. || !(run->v1 > 0.))
    return fail(ctx, LBL_E_ARG, "V1/V2");
  PnlPlan P;
  std::string e;
  int rc = pnlint_plan(*run, dv, dvout, &P, &e);
  if (rc) return fail(ctx, rc, e);
  if (layer_npts(*run, dv) != n_in) return fail(ctx, LBL_E_ARG, "n_in does not match the layer grid");
  if (P.n_out != n_out) return fail(ctx, LBL_E_ARG, "n_out does not match the DVOUT grid");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  if (P.copy) {
    CK(cudaMemcpyAsync(od_out, od_in, n_in * 8, cudaMemcpyDefault, s));
    CK(cudaStreamSynchronize(s));
    return LBL_OK;
  }
  const bool in_dev = is_device_ptr(od_in), out_dev = is_device_ptr(od_out);
  const size_t nseg = P.seg.size();
  size_t bytes = nseg * sizeof(PnlSeg) + sizeof(P.a) + 3 * 256;
  if (!in_dev) bytes += n_in * 8 + 256;
  if (!out_dev) bytes += n_out * 8 + 256;
  CK(ctx->arena.reserve(bytes, ctx->mem));
  ctx->arena.reset();
  PnlSeg* dseg = ctx->arena.take<PnlSeg>(nseg);
  double* da = ctx->arena.take<double>(4 * 101);
  const double* din = od_in;
  double* dout = od_out;
  if (!in_dev) {
    double* t = ctx->arena.take<double>(n_in);
    CK(cudaMemcpyAsync(t, od_in, n_in * 8, cudaMemcpyHostToDevice, s));
    din = t;
  }
  if (!out_dev) dout = ctx->arena.take<double>(n_out);
  CK(cudaMemcpyAsync(dseg, P.seg.data(), nseg * sizeof(PnlSeg), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(da, P.a, sizeof(P.a), cudaMemcpyHostToDevice, s));
  const double ratdv = dvout / dv;
  CK(launch_pnlint(dseg, (int64_t)nseg, da, din, n_in, ratdv, dout, n_out, s));
  if (!out_dev) CK(cudaMemcpyAsync(od_out, dout, n_out * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return LBL_OK;
}

int64_t lbl_scan_npts(const lbl_scan* sc, double dv_in, double* dvout) {
  if (!sc) return -LBL_E_ARG;
  ScanPlan P;
  std::string e;
  int rc = scan_plan(*sc, dv_in, &P, &e);
  // a spectrum coarser than DVINT is scanned on DVINT after SCNINT
  if (rc == LBL_E_RANGE && P.dvint > 0. && dv_in > P.dvint) rc = scan_plan(*sc, P.dvint, &P, &e);
  if (rc) return -rc;
  if (dvout) *dvout = P.dvo;
  return P.n_out;
}

namespace {
int scan_core(lbl_ctx* ctx, const lbl_scan* sc, const ScanPlan& P, const double* spec, int64_t n,
              double v1_in, double dv_in, double* out, int64_t n_out);
}

int lbl_scan_spectrum(lbl_ctx* ctx, const lbl_scan* sc, const double* spec, int64_t n,
                      double v1_in, double dv_in, double* out, int64_t n_out) {
  if (!ctx) return LBL_E_ARG;
  if (!sc || !spec || !out || n < 1) return fail(ctx, LBL_E_ARG, "NULL argument or empty spectrum");
  ScanPlan P;
  std::string e;
  int rc = scan_plan(*sc, dv_in, &P, &e);
  if (!(rc == LBL_E_RANGE && P.dvint > 0. && dv_in > P.dvint)) {
    if (rc) return fail(ctx, rc, e);
    return scan_core(ctx, sc, P, spec, n, v1_in, dv_in, out, n_out);
  }
  // SCANFN :322-345: the spectrum is first interpolated onto DVINT (SCNINT),
  // then scanned there
  const double dvint = P.dvint;
  rc = scan_plan(*sc, dvint, &P, &e);
  if (rc) return fail(ctx, rc, e);
  if (P.n_out != n_out) return fail(ctx, LBL_E_ARG, "n_out does not match the output grid");
  std::vector<ScnChunk> chunks;
  int64_t n_fine = 0;
  rc = scnint_plan(n, v1_in, dv_in, dvint, &chunks, &n_fine, &e);
  if (rc) return fail(ctx, rc, e);
  static_assert(sizeof(ScnChunk) == sizeof(ScnChunkDev), "chunk layouts");
  std::vector<double> coef(4 * 203);
  scnint_coefs(coef.data());
  cudaSetDevice(ctx->device);
  const bool in_dev = is_device_ptr(spec);
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_fine = up((size_t)n_fine * 8), b_in = in_dev ? 0 : up((size_t)n * 8),
               b_ch = up(chunks.size() * sizeof(ScnChunk)), b_co = up(coef.size() * 8);
  const size_t bytes = b_fine + b_in + b_ch + b_co;
  void* mem = nullptr;
  CK(ctx->mem.alloc(&mem, bytes));
  struct Release {
    lbl_ctx* c;
    void* m;
    size_t b;
    ~Release() { c->mem.release(m, b); }
  } guard{ctx, mem, bytes};
  char* base = static_cast<char*>(mem);
  double* fine = reinterpret_cast<double*>(base);
  double* din = in_dev ? const_cast<double*>(spec) : reinterpret_cast<double*>(base + b_fine);
  ScnChunkDev* dch = reinterpret_cast<ScnChunkDev*>(base + b_fine + b_in);
  double* dco = reinterpret_cast<double*>(base + b_fine + b_in + b_ch);
  cudaStream_t s = ctx->stream;
  if (!in_dev) CK(cudaMemcpyAsync(din, spec, (size_t)n * 8, cudaMemcpyHostToDevice, s));
  if (!chunks.empty())
    CK(cudaMemcpyAsync(dch, chunks.data(), chunks.size() * sizeof(ScnChunk),
                       cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dco, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice, s));
  CK(launch_scnint(dch, (int64_t)chunks.size(), din, n, dco, dvint / dv_in, fine, s));
  rc = scan_core(ctx, sc, P, fine, n_fine, v1_in, dvint, out, n_out);
  // the pageable copies above and the kernel finished before scan_core
  // returned (it synchronises the stream)
  CK(cudaStreamSynchronize(s));
  return rc;
}

namespace {
int scan_core(lbl_ctx* ctx, const lbl_scan* sc, const ScanPlan& P, const double* spec, int64_t n,
              double v1_in, double dv_in, double* out, int64_t n_out) {
  if (P.n_out != n_out) return fail(ctx, LBL_E_ARG, "n_out does not match the output grid");
  cudaSetDevice(ctx->device);
  if (P.jfn == 0 || P.jfn == 5 || P.jfn == 6) {
    // CNVRCT/CNVVRC/CNVVRL: every box, with both of its end points, inside
    // the input (the first box's left edge, the last box's right edge)
    const double b2 = P.bfov * P.bfov, vlast0 = sc->v1 + double(P.n_out - 1) * P.dvo;
    const double vfirst = P.jfn == 0 ? sc->v1 - P.hwhm
                          : P.jfn == 5 ? sc->v1 * (1. - b2 / 4.) : sc->v1;
    const double vlast = P.jfn == 0 ? vlast0 + P.hwhm
                         : P.jfn == 5 ? vlast0 * (1. + b2 / 4.) : vlast0 * (1. + b2 / 2.);
    if (v1_in > vfirst - dv_in || v1_in + double(n - 1) * dv_in < vlast + dv_in)
      return fail(ctx, LBL_E_RANGE, "scan: the boxes must lie inside the spectrum");
    const bool in_dev = is_device_ptr(spec), out_dev = is_device_ptr(out);
    size_t bytes = 256;
    if (!in_dev) bytes += n * 8 + 256;
    if (!out_dev) bytes += n_out * 8 + 256;
    CK(ctx->arena.reserve(bytes, ctx->mem));
    ctx->arena.reset();
    cudaStream_t s = ctx->stream;
    const double* din = spec;
    if (!in_dev) {
      double* t = ctx->arena.take<double>(n);
      CK(cudaMemcpyAsync(t, spec, n * 8, cudaMemcpyHostToDevice, s));
      din = t;
    }
    double* dout = out_dev ? out : ctx->arena.take<double>(n_out);
    CK(launch_scan_rect(din, n, sc->jabs ? 1 : 0, P.jfn, sc->v1, P.dvo, P.hwhm, P.bfov, v1_in,
                        dv_in, dout, n_out, s));
    if (!out_dev) CK(cudaMemcpyAsync(out, dout, n_out * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return LBL_OK;
  }
  // SHRKSC: full groups of IRATSH points; the compressed input's first
  // wavenumber and the CONVSC range from VBOT/VTOP (src/postsub.f90:1330-1355)
  const int64_t nc = n / P.iratsh;
  const double v1i = v1_in + P.v1shft;
  int64_t ilo = (int64_t)(((P.vbot - v1i) / P.dvsc) + 1.5);
  ilo = std::max<int64_t>(ilo, 1);
  int64_t ihi = (int64_t)(((P.vtop - v1i) / P.dvsc) + 1.5);
  ihi = std::min<int64_t>(ihi, nc);
  const double zint = (v1i - P.vft0) / P.dvo;
  const bool in_dev = is_device_ptr(spec), out_dev = is_device_ptr(out);
  size_t bytes = (nc + 1) * 8 + P.xf.size() * 8 + 4 * 256;
  if (!in_dev) bytes += n * 8 + 256;
  if (!out_dev) bytes += n_out * 8 + 256;
  CK(ctx->arena.reserve(bytes, ctx->mem));
  ctx->arena.reset();
  cudaStream_t s = ctx->stream;
  double* dsc = ctx->arena.take<double>(nc + 1);
  double* dxf = ctx->arena.take<double>(P.xf.size());
  const double* din = spec;
  if (!in_dev) {
    double* t = ctx->arena.take<double>(n);
    CK(cudaMemcpyAsync(t, spec, n * 8, cudaMemcpyHostToDevice, s));
    din = t;
  }
  double* dout = out_dev ? out : ctx->arena.take<double>(n_out);
  CK(cudaMemcpyAsync(dxf, P.xf.data(), P.xf.size() * 8, cudaMemcpyHostToDevice, s));
  CK(launch_scan(din, n, (int)P.iratsh, sc->jabs ? 1 : 0, dsc, ilo, ihi, zint, P.ratio, P.zbound,
                 P.zslope, P.xnorm, dxf, P.nfmax, dout, n_out, s));
  if (!out_dev) CK(cudaMemcpyAsync(out, dout, n_out * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return LBL_OK;
}
}  // namespace

int lbl_forward(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers, int32_t nlay, double* rad,
                double* tr, int64_t npts, int32_t precision) {
  if (!ctx) return LBL_E_ARG;
  int rc = check_run(ctx, run);
  if (rc) return rc;
  if (!layers || nlay < 1 || !rad) return fail(ctx, LBL_E_ARG, "NULL argument");
  cudaSetDevice(ctx->device);
  std::string e;
  rc = dv_rule(*run, layers, nlay, &e);
  if (rc) return fail(ctx, rc, e);
  if (layer_npts(*run, layers[nlay - 1].dv) != npts)
    return fail(ctx, LBL_E_ARG, "npts does not match the last layer's grid");
  Batch B;
  rc = prepare_batch(ctx, *run, layers, nlay, run->jrad, nullptr, B);
  if (rc) return rc;
  rc = run_od(ctx, *run, B, precision);
  if (rc) return rc;
  int res = 0;
  const OutSink sink{rad, tr};
  rc = run_merge(ctx, *run, layers, B, nlay, &res, precision, &sink);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  harvest(ctx);
  return finish_od(ctx);
}

int lbl_forward_batch(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers, const int32_t* nlay,
                      int32_t nprof, double* rad, double* tr, int64_t* offsets,
                      int64_t npts_total, int32_t precision) {
  if (!ctx) return LBL_E_ARG;
  int rc = check_run(ctx, run);
  if (rc) return rc;
  if (!layers || !nlay || nprof < 1 || !rad || !offsets) return fail(ctx, LBL_E_ARG, "NULL argument");
  cudaSetDevice(ctx->device);
  std::vector<int64_t> lay0(nprof + 1, 0);
  offsets[0] = 0;
  for (int p = 0; p < nprof; p++) {
    if (nlay[p] < 1) return fail(ctx, LBL_E_ARG, "profile without layers");
    std::string e;
    rc = dv_rule(*run, layers + lay0[p], nlay[p], &e);
    if (rc) return fail(ctx, rc, "profile " + std::to_string(p) + ": " + e);
    offsets[p + 1] = offsets[p] + layer_npts(*run, layers[lay0[p] + nlay[p] - 1].dv);
    lay0[p + 1] = lay0[p] + nlay[p];
  }
  if (offsets[nprof] > npts_total) return fail(ctx, LBL_E_ARG, "output buffer too small");
  return forward_groups(ctx, *run, layers, lay0, offsets, rad, tr, precision);
}

int lbl_jacobian(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers, int32_t nlay,
                 const int32_t* mols, int32_t nq, double* rad, double* jac, int64_t npts,
                 int32_t precision) {
  if (!ctx) return LBL_E_ARG;
  int rc = check_jac_args(ctx, run, layers, &nlay, 1, mols, nq, LBL_JAC_CENTRAL);
  if (rc) return rc;
  if (!jac) return fail(ctx, LBL_E_ARG, "lbl_jacobian: NULL output");
  cudaSetDevice(ctx->device);
  std::string e;
  rc = dv_rule(*run, layers, nlay, &e);
  if (rc) return fail(ctx, rc, e);
  if (layer_npts(*run, layers[nlay - 1].dv) != npts)
    return fail(ctx, LBL_E_ARG, "npts does not match the last layer's grid");
  const int np = 1 + nq;
  const int chunk = jac_chunk(ctx, *run, layers, nlay, np, 0);
  if (chunk < 1) return fail(ctx, LBL_E_NOMEM, "lbl_jacobian: work space");
  for (int k0 = 0; k0 < np; k0 += chunk) {
    const int k1 = std::min(np, k0 + chunk);
    JacOut o;
    rc = jac_profile(ctx, *run, layers, nlay, mols, k0, k1, LBL_JAC_CENTRAL, precision, 0, o);
    if (rc) return rc;
    if (rad && k0 == 0) {
      rc = copy_out(ctx, rad, o.rad, sizeof(double) * npts);
      if (rc) return rc;
    }
    rc = copy_out(ctx, jac + (size_t)k0 * nlay * npts, o.rows,
                  sizeof(double) * (size_t)(k1 - k0) * nlay * npts);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  harvest(ctx);
  return finish_od(ctx);
}

int lbl_adjoint_batch(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers, const int32_t* nlay,
                      int32_t nprof, const int32_t* mols, int32_t nq, int32_t mode,
                      double dv_chan, double* rad, int64_t* offsets, int64_t rad_cap,
                      double* jac, int64_t* jac_off, int64_t jac_cap, int32_t precision) {
  if (!ctx) return LBL_E_ARG;
  int rc = check_jac_args(ctx, run, layers, nlay, nprof, mols, nq, mode);
  if (rc) return rc;
  if (!rad || !offsets || !jac || !jac_off || !(dv_chan >= 0.))
    return fail(ctx, LBL_E_ARG, "lbl_adjoint_batch: bad argument");
  cudaSetDevice(ctx->device);
  const int np = 1 + nq;
  std::vector<int64_t> lay0(nprof + 1, 0), nout(nprof);
  const int64_t nchan = dv_chan > 0. ? (int64_t)std::floor((run->v2 - run->v1) / dv_chan + 1e-9) : 0;
  if (dv_chan > 0. && nchan < 1) return fail(ctx, LBL_E_ARG, "channel wider than the run");
  offsets[0] = 0;
  jac_off[0] = 0;
  for (int p = 0; p < nprof; p++) {
    std::string e;
    rc = dv_rule(*run, layers + lay0[p], nlay[p], &e);
    if (rc) return fail(ctx, rc, "profile " + std::to_string(p) + ": " + e);
    lay0[p + 1] = lay0[p] + nlay[p];
    nout[p] = dv_chan > 0. ? nchan : layer_npts(*run, layers[lay0[p + 1] - 1].dv);
    offsets[p + 1] = offsets[p] + nout[p];
    jac_off[p + 1] = jac_off[p] + (int64_t)np * nlay[p] * nout[p];
  }
  if (offsets[nprof] > rad_cap || jac_off[nprof] > jac_cap)
    return fail(ctx, LBL_E_ARG, "output buffer too small");
  for (int p = 0; p < nprof; p++) {
    lbl_layer* L = layers + lay0[p];
    const int nl = nlay[p];
    const int chunk = jac_chunk(ctx, *run, L, nl, np, nchan);
    if (chunk < 1)
      return fail(ctx, LBL_E_NOMEM, "profile " + std::to_string(p) + ": Jacobian work space");
    for (int k0 = 0; k0 < np; k0 += chunk) {
      const int k1 = std::min(np, k0 + chunk);
      JacOut o;
      rc = jac_profile(ctx, *run, L, nl, mols, k0, k1, mode, precision, nchan, o);
      if (rc) return rc;
      const double* rsrc = o.rad;
      const double* jsrc = o.rows;
      if (dv_chan > 0.) {
        // channel means of the radiance and of each row, into the work space
        rc = jac_channels(ctx, *run, o, nl * (k1 - k0), dv_chan, nchan);
        if (rc) return rc;
        rsrc = o.chan_rad;
        jsrc = o.chan_rows;
      }
      if (k0 == 0) {
        rc = copy_out(ctx, rad + offsets[p], rsrc, sizeof(double) * nout[p]);
        if (rc) return rc;
      }
      rc = copy_out(ctx, jac + jac_off[p] + (int64_t)k0 * nl * nout[p], jsrc,
                    sizeof(double) * (size_t)(k1 - k0) * nl * nout[p]);
      if (rc) return rc;
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  harvest(ctx);
  return finish_od(ctx);
}

int lbl_set_memory_limit(lbl_ctx* ctx, int64_t bytes) {
  if (!ctx || bytes < 0) return fail(ctx, LBL_E_ARG, "memory limit must be >= 0");
  // the grow-only work buffers are released; later calls allocate them again
  // within the cap
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->mem.release(ctx->arena.base, ctx->arena.cap);
  ctx->arena.base = nullptr;
  ctx->arena.cap = 0;
  ctx->mem.release(ctx->jac_mem, ctx->jac_cap);
  ctx->jac_mem = nullptr;
  ctx->jac_cap = 0;
  for (int k = 0; k < 4; k++) {
    ctx->mem.release(ctx->mbuf[k], ctx->mcap * sizeof(double));
    ctx->mbuf[k] = nullptr;
  }
  ctx->mcap = 0;
  ctx->mem.limit = (size_t)bytes;
  return LBL_OK;
}

int64_t lbl_memory_used(const lbl_ctx* ctx) { return ctx ? (int64_t)ctx->mem.used : -1; }

int lbl_profile(lbl_ctx* ctx, int32_t enable) {
  if (!ctx) return LBL_E_ARG;
  ctx->prof = enable != 0;
  return LBL_OK;
}

int lbl_profile_read(lbl_ctx* ctx, lbl_stage_stat* out, int32_t cap, int32_t* n) {
  if (!ctx || !n || (cap > 0 && !out)) return LBL_E_ARG;
  int32_t k = 0;
  for (auto& s : ctx->stages) {
    if (k < cap) {
      std::memset(&out[k], 0, sizeof(lbl_stage_stat));
      std::strncpy(out[k].name, s.name.c_str(), sizeof(out[k].name) - 1);
      out[k].ms = s.ms;
      out[k].launches = s.launches;
      out[k].work = s.work;
    }
    k++;
  }
  *n = std::min(k, cap);
  ctx->stages.clear();
  return LBL_OK;
}

int lbl_brightness_temperature(const double* rad, int64_t n, double v1, double dv, double* bt) {
  if (!rad || !bt || n < 0) return LBL_E_ARG;
  const double c1 = 1.191042722E-12, c2 = 1.4387752;
  for (int64_t i = 0; i < n; i++) {
    const double v = v1 + double(i) * dv;
    bt[i] = c2 * v / std::log(c1 * v * v * v / rad[i] + 1.);
  }
  return LBL_OK;
}

}  // extern "C"

// ---- TAPE3 file input ------------------------------------------------------
extern "C" int lbl_tape3_parse(const char* path, std::vector<double>* vnu, std::vector<float>* sp,
                               std::vector<float>* alfa, std::vector<float>* epp,
                               std::vector<int32_t>* mol, std::vector<float>* hw,
                               std::vector<float>* tmp, std::vector<float>* psh,
                               std::vector<int32_t>* iflg, std::vector<int64_t>* bs,
                               std::string* err);

extern "C" int lbl_lines_load_tape3(lbl_ctx* ctx, const char* path, int64_t* nlines) {
  if (!path) return fail(ctx, LBL_E_ARG, "NULL path");
  std::vector<double> vnu;
  std::vector<float> sp, alfa, epp, hw, tmp, psh;
  std::vector<int32_t> mol, iflg;
  std::vector<int64_t> bs;
  std::string e;
  int rc = lbl_tape3_parse(path, &vnu, &sp, &alfa, &epp, &mol, &hw, &tmp, &psh, &iflg, &bs, &e);
  if (rc) return fail(ctx, rc, e);
  lbl_lines L;
  L.n = (int64_t)vnu.size();
  L.vnu = vnu.data();
  L.sp = sp.data();
  L.alfa = alfa.data();
  L.epp = epp.data();
  L.mol = mol.data();
  L.hwhms = hw.data();
  L.tmpalf = tmp.data();
  L.pshift = psh.data();
  L.iflg = iflg.data();
  L.nblock = (int64_t)bs.size() - 1;
  L.block_start = bs.data();
  if (!ctx) {
    // no context: read and check the file only
    std::vector<double> vs;
    std::vector<int64_t> bchk;
    rc = validate_lines(nullptr, &L, &vs, &bchk);
    if (rc == LBL_OK && nlines) *nlines = L.n;
    return rc;
  }
  rc = lbl_lines_upload(ctx, &L);
  if (rc == LBL_OK && nlines) *nlines = L.n;
  return rc;
}
