// gd_server.cu -- the serving form: a request loop with continuous batching.
//
// Docking requests (a ligand ensemble + pocket template against one of the
// server's resident proteins, with its own MC parameters) are queued by
// gd_server_submit and admitted by a scheduler thread while the HBM budget
// and the slot count allow.  Requests are grouped by launch shape into lanes,
// each with its own stream; a lane advances all its requests in one launch,
// each by a number of MC steps balanced by its cost (plan_steps), and is
// relaunched as soon as that launch ends, with the requests admitted in the
// meantime joining it; lanes never wait for one another.  Each request keeps
// its own step counter and step count (KItem.step0 / n_run), replica state
// and random stream, so requests that arrived at different times share
// launches and a request's results do not depend on what else is running.
// Finished requests are copied out and their memory returns to the budget.
//
// There is no counterpart in the reference (Run() handles one complex per
// process, run.cu:41-353); the semantics of every request are those of Run.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "gd_common.h"

using namespace gd;
using Clock = std::chrono::steady_clock;

namespace {

enum ReqState { RQ_QUEUED, RQ_ACTIVE, RQ_DONE, RQ_CANCELLED, RQ_FAILED };

// A protein resident for the server's lifetime (device tables + host copy of
// the point properties for validating requests).
struct SrvProtein {
  gd_dcomplex *dcx = nullptr;
  std::vector<float> x, y, z, ele, hpp;
  std::vector<int> t, c, seq3r, hflag;
  gd_protein prt{};
  size_t bytes = 0;
};

struct Lane;

struct Req {
  uint64_t id = 0;
  int protein = 0;
  ReqState state = RQ_QUEUED;
  gd_status err = GD_OK;
  bool cancel = false;
  // owned host copy of the request
  std::vector<float> lx, ly, lz, lc, psp, kx, ky, kz, mx, my, mz, tcc, mb;
  std::vector<int> lt, ln, kt;
  gd_enepara ff{};
  gd_complex cx{};
  gd_mc_params mc{};
  int n_rep = 0;
  size_t bytes = 0;
  Clock::time_point t_submit, t_start, t_done;
  // device side while active
  gd_dcomplex *dcx = nullptr;
  float *d_m_old = nullptr, *d_e_old = nullptr, *d_mb = nullptr, *d_cmcc = nullptr;
  int *d_idx = nullptr, *d_acs = nullptr, *d_acx = nullptr;
  gd_record *d_rec = nullptr;     // [n_rep][steps_total] with GD_MC_RECORD
  Lane *lane = nullptr;            // its launch shape
  cudaStream_t stream = nullptr;  // the lane's stream
  int step = 0;
  int n_run = 0;      // MC steps of the current launch
  double cost = 0.0;  // ligand-size bucket x protein points (time per MC step)
  KItem item{};
  // results
  std::vector<float> energy, movematrix;
  std::vector<int> acs, idx, acx;
  std::vector<gd_record> rec;
};

// A launch shape of the server (tile, staging, group layout, exchange
// interval) with its own stream.  The requests of a lane advance together in
// rolling launches; lanes never wait for one another, so a shape whose
// requests are cheap is relaunched as soon as its own kernel ends while
// other shapes are still running.
struct Lane {
  Tile tile;
  int ns = 0, res = 0, gm = 0, spe = 0;
  int split = 1;                    // CTAs (a cluster) per request unit
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  // the lane's kernel error word, in pinned host memory the kernels write
  // directly (read after `done`)
  int *h_err = nullptr;
  bool busy = false;                // a launch is in flight
  std::vector<Req *> members;       // active requests of this shape
  std::vector<Req *> fresh;         // admitted, not yet initialised
  std::vector<Req *> in_flight;     // the requests of the launch in flight
  // Launch descriptors in pinned host memory that the kernels read directly
  // (no copy in the lane's stream, so a launch is one or two kernels and an
  // event): one set for the INIT launch and one for the MC launch that
  // follows it on the stream.  A set is rewritten only when the lane's
  // previous launch has ended.
  struct Desc {
    KItem *items = nullptr;
    int *cta = nullptr;  // [3][cap_cta]
    KGroup *groups = nullptr;
    size_t cap_items = 0, cap_cta = 0, cap_groups = 0;
  } desc[2];
};

// (A, P, NA, stages, resident, group-major, steps per exchange, split, sub-lane)
using LaneKey = std::tuple<int, int, int, int, int, int, int, int, int>;
constexpr int kMaxLanes = 512;
// Lanes per launch shape.  A lane relaunches only when the slowest CTA of its
// launch has finished, so its other SMs wait meanwhile unless other lanes'
// CTAs are queued; requests of one shape dealt over several lanes (each
// with its own stream) keep more CTAs queued.
constexpr int kSubLanes = 4;

}  // namespace

struct gd_server {
  gd_ctx *ctx = nullptr;
  size_t budget = 0;
  int max_active = 0;
  int steps_per_launch = 0;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;       // scheduler wake-up
  std::condition_variable done_cv;  // request completion
  bool stop = false;
  std::vector<std::unique_ptr<SrvProtein>> proteins;
  size_t protein_bytes = 0;
  std::deque<Req *> queue;
  std::vector<Req *> active;
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
  uint64_t next_id = 1;
  size_t bytes_in_use = 0;
  // statistics
  uint64_t n_done = 0, n_iter = 0, n_launch = 0;
  double busy_s = 0.0;
  // scheduler-thread state
  std::map<LaneKey, std::unique_ptr<Lane>> lanes;
  // error words of the lanes (device, zeroed) and their pinned host copies,
  // allocated once with the server
  int *h_err_pool = nullptr;  // lanes' error words (pinned, written by kernels)
  // nanoseconds the server's CTAs spent on their SMs (all launches)
  unsigned long long *d_busy_ns = nullptr;
  // the scheduler thread's time spent issuing launches (written by the
  // scheduler thread only, read by gd_server_get_stats)
  std::atomic<double> host_launch_s{0.0};
};

namespace {

// Device bytes a request holds while active (tables + replica state, and
// its per-step record with GD_MC_RECORD).
size_t request_bytes(const gd_complex *cx, const gd_mc_params *mc, int n_rep) {
  size_t b = (size_t)TAB_ROWS * GD_NPT * 24;
  b += (size_t)cx->lig.n_conf * cx->lig.lna * 16 + (size_t)cx->lig.lna * 8;
  b += (size_t)GD_NLT * cx->psp.n_col * 4;
  b += (size_t)cx->kde.pnk * 16 + (GD_NLT + 1) * 4;
  b += (size_t)cx->mcs.pos * cx->lig.lna * 16 + (size_t)cx->mcs.pos * 8;
  b += (size_t)n_rep * (6 + GD_NTERM + 3) * 4 + 3 * MAX_TMP * 4;
  // MCC reference map: one bit per (atom, padded point)
  b += (size_t)cx->lig.lna * ((cx->prt.pnp + TILE_PTS - 1) / TILE_PTS) * (TILE_PTS / 8);
  if (mc->flags & GD_MC_RECORD) b += (size_t)n_rep * mc->steps_total * sizeof(gd_record);
  return b;
}

template <typename T>
std::vector<T> vcopy(const T *p, size_t n) {
  return p ? std::vector<T>(p, p + n) : std::vector<T>();
}

void release_device(Req *r) {
  cudaStream_t s = r->stream;
  if (r->d_m_old) cudaFreeAsync(r->d_m_old, s);
  if (r->d_e_old) cudaFreeAsync(r->d_e_old, s);
  if (r->d_cmcc) cudaFreeAsync(r->d_cmcc, s);
  if (r->d_mb) cudaFreeAsync(r->d_mb, s);
  if (r->d_idx) cudaFreeAsync(r->d_idx, s);
  if (r->d_acs) cudaFreeAsync(r->d_acs, s);
  if (r->d_acx) cudaFreeAsync(r->d_acx, s);
  if (r->d_rec) cudaFreeAsync(r->d_rec, s);
  r->d_m_old = r->d_e_old = r->d_mb = r->d_cmcc = nullptr;
  r->d_idx = r->d_acs = r->d_acx = nullptr;
  r->d_rec = nullptr;
  if (r->dcx) {
    cudaStreamSynchronize(s);
    dcx_release(r->dcx);
    r->dcx = nullptr;
  }
}

// Grows a lane's pinned descriptor buffer (only while the lane is idle).
template <typename T>
gd_status grow(T **p, size_t *cap, size_t need) {
  if (need <= *cap) return GD_OK;
  size_t n = std::max<size_t>(need, *cap * 2 + 64);
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  GD_CUDA(cudaMallocHost((void **)p, n * sizeof(T)));
  *cap = n;
  return GD_OK;
}

// The lane of a request's launch shape, created on first use.
gd_status lane_for(gd_server *S, const Req *r, Lane **out) {
  const KTables &T = r->dcx->T;
  Tile t = tile_for(S->ctx, T);
  // a request is a run of its own
  const int split =
      split_for(S->ctx, T, units_of(T.n_prt, T.n_lig, r->mc.n_tmp), kServeSplitCost);
  int ns, res;
  pick_stages(T, t, &ns, &res, split);
  const bool gm = (32 % r->mc.n_tmp) == 0;
  const int spe = r->mc.steps_per_exchange;
  // the shape's least loaded lane; a new one while that lane holds requests
  // and the shape has fewer than kSubLanes
  Lane *best = nullptr;
  int n_sub = 0;
  for (int sub = 0; sub < kSubLanes; ++sub) {
    auto it = S->lanes.find(LaneKey{t.A, t.P, t.NA, ns, res, gm ? 1 : 0, spe, split, sub});
    if (it == S->lanes.end()) break;
    ++n_sub;
    Lane *L = it->second.get();
    if (!best || L->members.size() + L->fresh.size() < best->members.size() + best->fresh.size())
      best = L;
  }
  if (best && ((best->members.empty() && best->fresh.empty()) || n_sub == kSubLanes)) {
    *out = best;
    return GD_OK;
  }
  const LaneKey key{t.A, t.P, t.NA, ns, res, gm ? 1 : 0, spe, split, n_sub};
  auto L = std::make_unique<Lane>();
  L->tile = t;
  L->ns = ns;
  L->res = res;
  L->gm = gm ? 1 : 0;
  L->spe = spe;
  L->split = split;
  const int slot = (int)S->lanes.size();
  if (slot >= kMaxLanes) return fail(GD_ENOMEM, "more than %d lanes in the server", kMaxLanes);
  GD_CUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
  GD_CUDA(cudaEventCreateWithFlags(&L->done, cudaEventDisableTiming));
  L->h_err = S->h_err_pool + slot;
  *out = L.get();
  S->lanes[key] = std::move(L);
  return GD_OK;
}

// Uploads the request's tables, allocates its state on its lane's stream and
// fills its KItem.
gd_status admit(gd_server *S, Req *r) {
  NvtxRange nvtx("gd_server admit");
  SrvProtein &P = *S->proteins[r->protein];
  GD_TRY(gd_complex_upload_shared(S->ctx, &r->cx, P.dcx, 0, P.prt.n_conf, &r->dcx));
  Lane *L = nullptr;
  GD_TRY(lane_for(S, r, &L));
  r->lane = L;
  r->stream = L->stream;
  cudaStream_t s = L->stream;
  const size_t n = (size_t)r->n_rep;
  if (injected_alloc_failure(S->ctx))
    return fail(GD_ENOMEM, "request state: out of memory (injected)");
  GD_CUDA(cudaMallocAsync(&r->d_m_old, n * 6 * sizeof(float), s));
  GD_CUDA(cudaMallocAsync(&r->d_e_old, n * GD_NTERM * sizeof(float), s));
  GD_CUDA(cudaMallocAsync(&r->d_cmcc, n * sizeof(float), s));
  GD_CUDA(cudaMallocAsync(&r->d_mb, MAX_TMP * sizeof(float), s));
  GD_CUDA(cudaMallocAsync(&r->d_idx, n * sizeof(int), s));
  GD_CUDA(cudaMallocAsync(&r->d_acs, n * sizeof(int), s));
  GD_CUDA(cudaMallocAsync(&r->d_acx, MAX_TMP * sizeof(int), s));
  GD_CUDA(cudaMemsetAsync(r->d_acx, 0, MAX_TMP * sizeof(int), s));
  const bool record = (r->mc.flags & GD_MC_RECORD) != 0;
  if (record) {
    const size_t nr = n * (size_t)r->mc.steps_total * sizeof(gd_record);
    GD_CUDA(cudaMallocAsync((void **)&r->d_rec, nr, s));
    GD_CUDA(cudaMemsetAsync(r->d_rec, 0, nr, s));
  }
  GD_CUDA(cudaMemcpyAsync(r->d_mb, r->mb.data(), r->mb.size() * sizeof(float),
                          cudaMemcpyHostToDevice, s));
  KItem &I = r->item;
  std::memset(&I, 0, sizeof(I));
  I.T = r->dcx->T;
  I.rep_base = 0;
  I.n_tmp = r->mc.n_tmp;
  I.n_lig_conf = I.T.n_lig;
  I.n_prt = I.T.n_prt;
  I.n_rep = r->n_rep;
  I.steps_per_dump = r->mc.steps_per_dump;
  I.spe = r->mc.steps_per_exchange;
  for (int k = 0; k < 6; ++k) I.move_scale[k] = r->mc.move_scale[k];
  I.seed = r->mc.seed;
  I.stream_id = r->mc.stream_id;
  I.flags = r->mc.flags;
  I.minus_beta = r->d_mb;
  I.acs_exchg = r->d_acx;
  I.record = r->d_rec;  // steps 0 .. steps_total-1 (no ring)
  I.rec_steps = record ? r->mc.steps_total : 0;
  I.rec_ring = 0;
  I.m_old = r->d_m_old;
  I.e_old = r->d_e_old;
  I.cmcc = r->d_cmcc;
  I.idx_tmp = r->d_idx;
  I.acs_mc = r->d_acs;
  r->step = 0;
  // time per MC step: the unit's pairs over the CTAs that share them
  r->cost = (double)lna_bucket(I.T.lna) * I.T.pnp / r->lane->split;
  return GD_OK;
}

// One launch of a lane over the given requests (KRun item_step: each request
// at its own step, for its own step count), plus the exchange kernel for
// groups that do not fit a CTA.  Asynchronous on the lane's stream.
gd_status launch_lane(gd_server *S, Lane &L, const std::vector<Req *> &rs, int mode) {
  NvtxRange nvtx(mode == KMODE_INIT ? "gd_server lane init" : "gd_server lane launch");
  if (rs.empty()) return GD_OK;
  cudaStream_t s = L.stream;
  std::vector<KItem> items;
  items.reserve(rs.size());
  std::vector<std::tuple<double, int, int, int>> ctas;  // cost, item, rep0/group, n
  std::vector<KGroup> groups;
  for (size_t i = 0; i < rs.size(); ++i) {
    Req *r = rs[i];
    r->item.step0 = r->step;
    r->item.n_run = mode == KMODE_REMC ? r->n_run : 1;
    items.push_back(r->item);
    const KItem &I = r->item;
    const int nt = I.n_tmp, nl = I.n_lig_conf;
    if (L.gm) {
      const int G = 32 / nt;
      for (int p = 0; p < I.n_prt; ++p)
        for (int l0 = 0; l0 < nl; l0 += G)
          ctas.emplace_back(r->cost * r->item.n_run, (int)i, p * nl + l0,
                            std::min(G, nl - l0) * nt);
    } else {
      const int per_p = nt * nl;
      for (int p = 0; p < I.n_prt; ++p)
        for (int j = 0; j < per_p; j += 32)
          ctas.emplace_back(r->cost * r->item.n_run, (int)i, p * per_p + j,
                            std::min(32, per_p - j));
      if (mode == KMODE_REMC && (I.flags & GD_MC_EXCHANGE))
        for (int p = 0; p < I.n_prt; ++p)
          for (int l = 0; l < nl; ++l) groups.push_back(KGroup{(int)i, p, l, 0});
    }
  }
  // costliest CTAs first, so the longest ones start first
  std::stable_sort(ctas.begin(), ctas.end(),
                   [](const auto &a, const auto &b) { return std::get<0>(a) > std::get<0>(b); });
  const size_t n_cta = ctas.size();
  // the lane's previous launch has ended, so its descriptor set is free
  Lane::Desc &D = L.desc[mode == KMODE_INIT ? 0 : 1];
  GD_TRY(grow(&D.items, &D.cap_items, items.size()));
  GD_TRY(grow(&D.cta, &D.cap_cta, 3 * n_cta));
  GD_TRY(grow(&D.groups, &D.cap_groups, std::max<size_t>(groups.size(), 1)));
  std::memcpy(D.items, items.data(), items.size() * sizeof(KItem));
  for (size_t c = 0; c < n_cta; ++c) {
    D.cta[c] = std::get<1>(ctas[c]);
    D.cta[n_cta + c] = std::get<2>(ctas[c]);
    D.cta[2 * n_cta + c] = std::get<3>(ctas[c]);
  }
  if (!groups.empty()) std::memcpy(D.groups, groups.data(), groups.size() * sizeof(KGroup));
  KRun R{};
  R.mode = mode;
  R.A = L.tile.A;
  R.P = L.tile.P;
  R.n_stages = L.ns;
  R.resident = L.res;
  R.items = D.items;
  R.cta_item = D.cta;
  R.cta_rep0 = D.cta + n_cta;
  R.cta_nrep = D.cta + 2 * n_cta;
  R.group_major = L.gm;
  R.fused_exchange = L.gm;
  R.spe = L.spe;
  R.step0 = 0;
  R.n_steps = 0;  // per item (item_step)
  R.item_step = 1;
  R.err = L.h_err;
  R.busy_ns = S->d_busy_ns;
  R.split = L.split;
  for (const Req *r : rs) R.hb_pairs = std::max(R.hb_pairs, hb_pairs_of(r->item.T, L.tile.A));
  GD_CUDA(launch_dock(R, L.tile.NA, (int)n_cta * L.split, s));
  S->ctx->launches += 1;
  S->n_launch += 1;
  if (!groups.empty()) {
    // per-item mode (step0 < 0): each group uses its item's step and spe
    GD_CUDA(launch_exchange(D.items, D.groups, (int)groups.size(), 1, -1, nullptr, s));
    S->ctx->launches += 1;
    S->n_launch += 1;
  }
  return GD_OK;
}

// MC steps of every request of a lane's next launch.  A request's CTAs take
// time proportional to its cost per step, so the most expensive one advances
// steps_per_launch steps (rounded to its exchange interval) and the others
// proportionally more, in whole exchange intervals and at most their
// remaining steps: the launch's CTAs run about equally long.  Requests whose
// exchange runs as a separate kernel advance one interval.
void plan_steps(gd_server *S, const std::vector<Req *> &rs) {
  double quantum = 0.0;
  for (Req *r : rs) {
    const int spe = r->mc.steps_per_exchange;
    const int n = std::max(spe, S->steps_per_launch / spe * spe);
    quantum = std::max(quantum, r->cost * n);
  }
  for (Req *r : rs) {
    const int spe = r->mc.steps_per_exchange;
    const int left = r->mc.steps_total - r->step;
    int n;
    if ((r->mc.flags & GD_MC_EXCHANGE) && 32 % r->mc.n_tmp != 0) {
      n = spe;
    } else {
      const double k = std::floor(quantum / (r->cost * spe));
      n = (int)std::min<double>(std::max(1.0, k), (double)(left / spe)) * spe;
    }
    r->n_run = std::max(spe, std::min(n, left));
  }
}

gd_status copy_out(Req *r) {
  cudaStream_t s = r->stream;
  const size_t n = (size_t)r->n_rep;
  r->energy.resize(n * GD_NTERM);
  r->movematrix.resize(n * 6);
  r->acs.resize(n);
  r->idx.resize(n);
  r->acx.resize(r->mc.n_tmp);
  GD_CUDA(cudaMemcpyAsync(r->energy.data(), r->d_e_old, n * GD_NTERM * 4, cudaMemcpyDeviceToHost,
                          s));
  GD_CUDA(cudaMemcpyAsync(r->movematrix.data(), r->d_m_old, n * 24, cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaMemcpyAsync(r->acs.data(), r->d_acs, n * 4, cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaMemcpyAsync(r->idx.data(), r->d_idx, n * 4, cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaMemcpyAsync(r->acx.data(), r->d_acx, r->mc.n_tmp * 4, cudaMemcpyDeviceToHost, s));
  if (r->d_rec) {
    r->rec.resize(n * (size_t)r->mc.steps_total);
    GD_CUDA(cudaMemcpyAsync(r->rec.data(), r->d_rec, r->rec.size() * sizeof(gd_record),
                            cudaMemcpyDeviceToHost, s));
  }
  GD_CUDA(cudaStreamSynchronize(s));
  return GD_OK;
}

// Called with S->mu held.
void finish(gd_server *S, Req *r, ReqState st, gd_status err) {
  release_device(r);
  r->state = st;
  r->err = err;
  r->t_done = Clock::now();
  S->bytes_in_use -= r->bytes;
  if (st == RQ_DONE) S->n_done += 1;
  S->active.erase(std::remove(S->active.begin(), S->active.end(), r), S->active.end());
}

// The scheduler thread.  Each round it admits queued requests while the HBM
// budget and the slot count allow, collects the lanes whose launch has ended
// (advancing their requests, finishing the completed ones), and relaunches
// every idle lane with its current members plus the newly admitted requests
// of its shape (initialised first, on the same stream).
void scheduler(gd_server *S) {
  cudaSetDevice(S->ctx->device);
  auto t_busy = Clock::now();
  bool was_busy = false;
  for (;;) {
    std::vector<Req *> admitted;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->stop) break;
      for (auto it = S->queue.begin(); it != S->queue.end();) {
        if ((*it)->cancel) {
          (*it)->state = RQ_CANCELLED;
          (*it)->t_done = Clock::now();
          it = S->queue.erase(it);
          S->done_cv.notify_all();
        } else {
          ++it;
        }
      }
      while (!S->queue.empty() &&
             (S->max_active <= 0 || (int)S->active.size() < S->max_active) &&
             S->protein_bytes + S->bytes_in_use + S->queue.front()->bytes <= S->budget) {
        Req *r = S->queue.front();
        S->queue.pop_front();
        S->bytes_in_use += r->bytes;
        r->state = RQ_ACTIVE;
        r->t_start = Clock::now();
        S->active.push_back(r);
        admitted.push_back(r);
      }
      bool any = !S->active.empty();
      if (!any && admitted.empty()) {
        if (was_busy) {
          S->busy_s += std::chrono::duration<double>(Clock::now() - t_busy).count();
          was_busy = false;
        }
        S->cv.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
      if (!was_busy) {
        t_busy = Clock::now();
        was_busy = true;
      }
    }
    // uploads and state of the admitted requests (outside the lock)
    std::vector<std::pair<Req *, gd_status>> failed;
    for (Req *r : admitted) {
      gd_status st = admit(S, r);
      if (st == GD_OK)
        r->lane->fresh.push_back(r);
      else
        failed.emplace_back(r, st);
    }
    bool progressed = !admitted.empty();
    std::vector<Req *> finished;
    std::vector<std::pair<Req *, gd_status>> lane_failed;
    for (auto &kv : S->lanes) {
      Lane &L = *kv.second;
      if (L.busy) {
        const cudaError_t q = cudaEventQuery(L.done);
        if (q == cudaErrorNotReady) continue;
        L.busy = false;
        progressed = true;
        gd_status st = GD_OK;
        if (q != cudaSuccess) {
          st = fail(GD_ECUDA, "server launch: %s", cudaGetErrorString(q));
        } else if (*(volatile int *)L.h_err != 0) {
          st = kernel_error(*L.h_err);
          *(volatile int *)L.h_err = 0;  // the lane's next launch starts after this
        }
        for (Req *r : L.in_flight) {
          if (st != GD_OK) {
            lane_failed.emplace_back(r, st);
            continue;
          }
          r->step += r->n_run;
          if (r->step >= r->mc.steps_total) {
            const gd_status cs = copy_out(r);
            if (cs == GD_OK)
              finished.push_back(r);
            else
              lane_failed.emplace_back(r, cs);
          }
        }
        std::vector<Req *> keep;
        for (Req *r : L.members) {
          bool gone = std::find(finished.begin(), finished.end(), r) != finished.end();
          for (auto &f : lane_failed) gone = gone || f.first == r;
          if (!gone) keep.push_back(r);
        }
        L.members.swap(keep);
        L.in_flight.clear();
      }
    }
    // cancelled members leave while their lane is idle
    std::vector<Req *> cancelled;
    {
      std::lock_guard<std::mutex> g(S->mu);
      for (auto &kv : S->lanes) {
        Lane &L = *kv.second;
        if (L.busy) continue;
        std::vector<Req *> keep;
        for (Req *r : L.members) (r->cancel ? cancelled : keep).push_back(r);
        L.members.swap(keep);
      }
    }
    // relaunch every idle lane
    for (auto &kv : S->lanes) {
      Lane &L = *kv.second;
      if (L.busy || (L.members.empty() && L.fresh.empty())) continue;
      const auto t_issue = Clock::now();
      gd_status st = GD_OK;
      if (!L.fresh.empty()) {
        st = launch_lane(S, L, L.fresh, KMODE_INIT);
        for (Req *r : L.fresh) L.members.push_back(r);
        L.fresh.clear();
      }
      if (st == GD_OK) {
        plan_steps(S, L.members);
        st = launch_lane(S, L, L.members, KMODE_REMC);
      }
      if (st == GD_OK && cudaEventRecord(L.done, L.stream) != cudaSuccess)
        st = fail(GD_ECUDA, "server: event record");
      if (st != GD_OK) {
        cudaStreamSynchronize(L.stream);
        for (Req *r : L.members) lane_failed.emplace_back(r, st);
        L.members.clear();
        continue;
      }
      S->host_launch_s.store(S->host_launch_s.load() +
                             std::chrono::duration<double>(Clock::now() - t_issue).count());
      L.in_flight = L.members;
      L.busy = true;
      S->n_iter += 1;
      progressed = true;
    }
    {
      std::lock_guard<std::mutex> g(S->mu);
      for (auto &f : failed) finish(S, f.first, RQ_FAILED, f.second);
      for (auto &f : lane_failed) finish(S, f.first, RQ_FAILED, f.second);
      for (Req *r : cancelled) finish(S, r, RQ_CANCELLED, GD_ECANCELLED);
      for (Req *r : finished) finish(S, r, RQ_DONE, GD_OK);
      if (!failed.empty() || !lane_failed.empty() || !cancelled.empty() || !finished.empty())
        S->done_cv.notify_all();
    }
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  // stopping: wait for the lanes' launches to end
  for (auto &kv : S->lanes)
    if (kv.second->busy) cudaEventSynchronize(kv.second->done);
}

gd_status copy_request(gd_server *S, int protein_id, const gd_complex *cx,
                       const gd_mc_params *mc, Req *r) {
  const SrvProtein &P = *S->proteins[protein_id];
  const gd_ligand &L = cx->lig;
  const size_t nl = (size_t)L.n_conf * L.lna;
  r->lx = vcopy(L.x, nl);
  r->ly = vcopy(L.y, nl);
  r->lz = vcopy(L.z, nl);
  r->lt = vcopy(L.t, (size_t)L.lna);
  r->lc = vcopy(L.c, (size_t)L.lna);
  r->ln = vcopy(L.n, (size_t)L.lna);
  r->psp = vcopy(cx->psp.psp, (size_t)GD_NLT * cx->psp.n_col);
  r->kx = vcopy(cx->kde.x, (size_t)cx->kde.pnk);
  r->ky = vcopy(cx->kde.y, (size_t)cx->kde.pnk);
  r->kz = vcopy(cx->kde.z, (size_t)cx->kde.pnk);
  r->kt = vcopy(cx->kde.t, (size_t)cx->kde.pnk);
  const size_t nm = (size_t)cx->mcs.pos * cx->mcs.n_field;
  r->mx = vcopy(cx->mcs.x, nm);
  r->my = vcopy(cx->mcs.y, nm);
  r->mz = vcopy(cx->mcs.z, nm);
  r->tcc = vcopy(cx->mcs.tcc, (size_t)cx->mcs.pos);
  r->ff = *cx->ff;
  r->mb = vcopy(mc->minus_beta, (size_t)mc->n_tmp);
  r->cx = *cx;
  r->cx.lig.x = r->lx.data();
  r->cx.lig.y = r->ly.data();
  r->cx.lig.z = r->lz.data();
  r->cx.lig.t = r->lt.data();
  r->cx.lig.c = r->lc.data();
  r->cx.lig.n = r->ln.data();
  r->cx.psp.psp = r->psp.data();
  r->cx.kde.x = r->kx.data();
  r->cx.kde.y = r->ky.data();
  r->cx.kde.z = r->kz.data();
  r->cx.kde.t = r->kt.data();
  r->cx.mcs.x = r->mx.data();
  r->cx.mcs.y = r->my.data();
  r->cx.mcs.z = r->mz.data();
  r->cx.mcs.tcc = r->tcc.data();
  r->cx.ff = &r->ff;
  r->cx.prt = P.prt;  // the resident protein
  r->mc = *mc;
  r->mc.minus_beta = r->mb.data();
  r->protein = protein_id;
  r->n_rep = P.prt.n_conf * L.n_conf * mc->n_tmp;
  r->bytes = request_bytes(&r->cx, &r->mc, r->n_rep);
  return GD_OK;
}

}  // namespace

extern "C" gd_status gd_server_create(int device, size_t hbm_budget_bytes, int max_active,
                                      int steps_per_launch, gd_server **out) {
  if (!out) return fail(GD_EINVAL, "gd_server_create: out is NULL");
  *out = nullptr;
  if (steps_per_launch < 1) return fail(GD_EINVAL, "steps_per_launch=%d", steps_per_launch);
  gd_ctx *ctx = nullptr;
  GD_TRY(gd_ctx_create(device, nullptr, &ctx));
  gd_server *S = new (std::nothrow) gd_server;
  if (!S) {
    ctx_release(ctx);
    return fail(GD_ENOMEM, "host allocation");
  }
  S->ctx = ctx;
  S->budget = hbm_budget_bytes;
  S->max_active = max_active > 0 ? max_active : 2 * ctx->n_sm;
  S->steps_per_launch = steps_per_launch;
  if (cudaMalloc(&S->d_busy_ns, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(S->d_busy_ns, 0, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost(&S->h_err_pool, kMaxLanes * sizeof(int)) != cudaSuccess) {
    if (S->d_busy_ns) cudaFree(S->d_busy_ns);
    ctx_release(ctx);
    delete S;
    return fail(GD_ENOMEM, "server error words");
  }
  std::memset(S->h_err_pool, 0, kMaxLanes * sizeof(int));
  S->th = std::thread(scheduler, S);
  *out = S;
  return GD_OK;
}

extern "C" gd_status gd_server_add_protein(gd_server *S, const gd_complex *cx, int *protein_id) {
  if (!S || !cx || !protein_id) return fail(GD_EINVAL, "gd_server_add_protein: NULL argument");
  GD_TRY(gd_complex_validate(cx));
  auto P = std::make_unique<SrvProtein>();
  const gd_protein &src = cx->prt;
  const size_t np = (size_t)src.pnp, nc = (size_t)src.n_conf * src.pnp;
  P->x = vcopy(src.x, nc);
  P->y = vcopy(src.y, nc);
  P->z = vcopy(src.z, nc);
  P->t = vcopy(src.t, np);
  P->c = vcopy(src.c, np);
  P->ele = vcopy(src.ele, np);
  P->seq3r = vcopy(src.seq3r, np);
  P->hflag = vcopy(src.c0_and_d12_or_c2, np);
  P->hpp = vcopy(src.hpp, np);
  P->prt = src;
  P->prt.x = P->x.data();
  P->prt.y = P->y.data();
  P->prt.z = P->z.data();
  P->prt.t = P->t.data();
  P->prt.c = P->c.data();
  P->prt.ele = P->ele.data();
  P->prt.seq3r = P->seq3r.data();
  P->prt.c0_and_d12_or_c2 = P->hflag.data();
  P->prt.hpp = P->hpp.data();
  std::lock_guard<std::mutex> g(S->mu);
  cudaSetDevice(S->ctx->device);
  GD_TRY(gd_complex_upload(S->ctx, cx, &P->dcx));
  P->bytes = gd_complex_device_bytes(P->dcx);
  if (S->protein_bytes + P->bytes > S->budget) {
    dcx_release(P->dcx);
    return fail(GD_EBUDGET, "protein needs %zu bytes, budget %zu already holds %zu", P->bytes,
                S->budget, S->protein_bytes);
  }
  S->protein_bytes += P->bytes;
  *protein_id = (int)S->proteins.size();
  S->proteins.push_back(std::move(P));
  return GD_OK;
}

extern "C" gd_status gd_server_submit(gd_server *S, int protein_id, const gd_complex *cx,
                                      const gd_mc_params *mc, uint64_t *req_id) {
  if (!S || !cx || !mc || !req_id) return fail(GD_EINVAL, "gd_server_submit: NULL argument");
  {
    std::lock_guard<std::mutex> g(S->mu);
    if (protein_id < 0 || protein_id >= (int)S->proteins.size())
      return fail(GD_EINVAL, "unknown protein %d", protein_id);
  }
  if (mc->n_tmp < 1 || mc->n_tmp > MAX_TMP || !mc->minus_beta)
    return fail(GD_EINVAL, "n_tmp=%d", mc->n_tmp);
  if (mc->steps_per_exchange < 1)
    return fail(GD_EINVAL, "steps_per_exchange=%d", mc->steps_per_exchange);
  if (mc->steps_total < mc->steps_per_exchange || mc->steps_total % mc->steps_per_exchange != 0)
    return fail(GD_EINVAL, "steps_total %d is not a positive multiple of steps_per_exchange %d",
                mc->steps_total, mc->steps_per_exchange);
  auto r = std::make_unique<Req>();
  try {
    GD_TRY(copy_request(S, protein_id, cx, mc, r.get()));
  } catch (const std::bad_alloc &) {
    return fail(GD_ENOMEM, "host allocation");
  }
  GD_TRY(gd_complex_validate(&r->cx));
  std::lock_guard<std::mutex> g(S->mu);
  if (S->protein_bytes + r->bytes > S->budget)
    return fail(GD_EBUDGET, "request needs %zu bytes; budget %zu, proteins hold %zu", r->bytes,
                S->budget, S->protein_bytes);
  r->id = S->next_id++;
  r->t_submit = Clock::now();
  *req_id = r->id;
  S->queue.push_back(r.get());
  S->reqs[r->id] = std::move(r);
  S->cv.notify_all();
  return GD_OK;
}

static gd_status take_result(gd_server *S, std::unordered_map<uint64_t, std::unique_ptr<Req>>::iterator it,
                             gd_mc_log *log) {
  Req *r = it->second.get();
  gd_status st = GD_OK;
  if (r->state == RQ_DONE) {
    if (log) {
      const size_t n = (size_t)r->n_rep;
      if (log->energy) std::memcpy(log->energy, r->energy.data(), n * GD_NTERM * 4);
      if (log->movematrix) std::memcpy(log->movematrix, r->movematrix.data(), n * 24);
      if (log->acs_mc) std::memcpy(log->acs_mc, r->acs.data(), n * 4);
      if (log->idx_tmp) std::memcpy(log->idx_tmp, r->idx.data(), n * 4);
      if (log->acs_temp_exchg) std::memcpy(log->acs_temp_exchg, r->acx.data(), r->acx.size() * 4);
      if (log->record && !r->rec.empty())
        std::memcpy(log->record, r->rec.data(), r->rec.size() * sizeof(gd_record));
      log->ac_mc = 0;
      for (int v : r->acs) log->ac_mc += v;
      log->ac_temp_exchg = 0;
      for (int v : r->acx) log->ac_temp_exchg += v;
      log->t_wall = std::chrono::duration<double>(r->t_done - r->t_submit).count();
      log->t_compute = std::chrono::duration<double>(r->t_done - r->t_start).count();
    }
  } else if (r->state == RQ_CANCELLED) {
    st = fail(GD_ECANCELLED, "request %llu was cancelled", (unsigned long long)r->id);
  } else {
    st = r->err != GD_OK ? r->err : GD_ECUDA;
  }
  S->reqs.erase(it);
  return st;
}

extern "C" gd_status gd_server_poll(gd_server *S, uint64_t req_id, gd_mc_log *log) {
  if (!S) return fail(GD_EINVAL, "server NULL");
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->reqs.find(req_id);
  if (it == S->reqs.end()) return fail(GD_ENOTFOUND, "no request %llu", (unsigned long long)req_id);
  const ReqState st = it->second->state;
  if (st == RQ_QUEUED || st == RQ_ACTIVE) return GD_EAGAIN;
  return take_result(S, it, log);
}

extern "C" gd_status gd_server_wait(gd_server *S, uint64_t req_id, int timeout_ms,
                                    gd_mc_log *log) {
  if (!S) return fail(GD_EINVAL, "server NULL");
  std::unique_lock<std::mutex> lk(S->mu);
  const auto deadline = Clock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
  for (;;) {
    auto it = S->reqs.find(req_id);
    if (it == S->reqs.end())
      return fail(GD_ENOTFOUND, "no request %llu", (unsigned long long)req_id);
    const ReqState st = it->second->state;
    if (st != RQ_QUEUED && st != RQ_ACTIVE) return take_result(S, it, log);
    if (S->done_cv.wait_until(lk, deadline) == std::cv_status::timeout) {
      auto it2 = S->reqs.find(req_id);
      if (it2 != S->reqs.end() &&
          (it2->second->state == RQ_QUEUED || it2->second->state == RQ_ACTIVE))
        return fail(GD_ETIMEDOUT, "request %llu not finished after %d ms",
                    (unsigned long long)req_id, timeout_ms);
    }
  }
}

extern "C" gd_status gd_server_cancel(gd_server *S, uint64_t req_id) {
  if (!S) return fail(GD_EINVAL, "server NULL");
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->reqs.find(req_id);
  if (it == S->reqs.end()) return fail(GD_ENOTFOUND, "no request %llu", (unsigned long long)req_id);
  it->second->cancel = true;
  S->cv.notify_all();
  return GD_OK;
}

extern "C" gd_ctx *gd_server_context(gd_server *S) { return S ? S->ctx : nullptr; }

extern "C" gd_status gd_server_get_stats(gd_server *S, gd_server_stats *out) {
  if (!S || !out) return fail(GD_EINVAL, "gd_server_get_stats: NULL argument");
  std::lock_guard<std::mutex> g(S->mu);
  out->queued = (int)S->queue.size();
  out->active = (int)S->active.size();
  out->completed = S->n_done;
  out->iterations = S->n_iter;
  out->launches = S->n_launch;
  out->bytes_in_use = S->bytes_in_use + S->protein_bytes;
  out->busy_s = S->busy_s;
  unsigned long long ns = 0;
  cudaSetDevice(S->ctx->device);
  GD_CUDA(cudaMemcpy(&ns, S->d_busy_ns, sizeof ns, cudaMemcpyDeviceToHost));
  out->cta_busy_s = (double)ns * 1e-9;
  out->host_launch_s = S->host_launch_s.load();
  return GD_OK;
}

extern "C" gd_status gd_server_destroy(gd_server *S) {
  if (!S) return GD_OK;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
    S->cv.notify_all();
  }
  if (S->th.joinable()) S->th.join();
  cudaSetDevice(S->ctx->device);
  for (Req *r : S->active)
    if (r->stream) release_device(r);
  cudaStreamSynchronize(S->ctx->stream);
  for (auto &p : S->proteins) dcx_release(p->dcx);
  for (auto &kv : S->lanes) {
    Lane &L = *kv.second;
    cudaStreamSynchronize(L.stream);
    for (Lane::Desc &D : L.desc) {
      if (D.items) cudaFreeHost(D.items);
      if (D.cta) cudaFreeHost(D.cta);
      if (D.groups) cudaFreeHost(D.groups);
    }
    cudaEventDestroy(L.done);
    cudaStreamDestroy(L.stream);
  }
  if (S->d_busy_ns) cudaFree(S->d_busy_ns);
  if (S->h_err_pool) cudaFreeHost(S->h_err_pool);
  ctx_release(S->ctx);
  delete S;
  return GD_OK;
}
