// gd_ensemble.cu -- replica-exchange Monte Carlo runs: the plain per-complex
// form (gd_remc, one complex) and the batched form (gd_batch, many complexes
// of uneven sizes advanced together), both built on one launch planner.
//
// Reference path replaced: the Run() loop of gpudocksm-rem-1.2/src/run.cu and
// gpusingle.cu:5-37 (MonteCarlo_d launches of steps_per_exchange steps, each
// followed by a single-thread ExchangeReplicas_d, all synchronous).
//
// Planning: every complex gets a launch shape (A x P warps, NA atoms per
// warp; from the context's autotuned table or the default), complexes with
// the same shape share one launch.  When the temperature count divides 32 a
// CTA holds whole exchange groups (32 / n_tmp ligand conformations x all
// temperatures) and the exchange runs inside the kernel, so a run of any
// length is one launch per shape; otherwise an exchange kernel follows every
// interval.  The per-interval launch sequence reads its first MC step from a
// device counter, so it is captured once into a CUDA graph and replayed.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <atomic>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "gd_common.h"

using namespace gd;

namespace {

struct Plan {
  Tile tile;
  double cost = 0.0;  // sum over its CTAs of ligand atoms x protein points
  int n_stages = 0, resident = 0, group_major = 0, fused = 0, grid = 0;
  int hb_pairs = 0;  // largest hb_pairs_of over its items
  int split = 1;     // CTAs (a cluster) per unit (split_for)
  int *d_cta_item = nullptr, *d_cta_rep0 = nullptr, *d_cta_nrep = nullptr;
  // persistent schedules (KRun.pieces) of this plan's units, by launch length
  std::vector<double> unit_cost;  // [grid] cost of one MC step of each unit
  int *d_progress = nullptr;      // [grid] MC steps done by each unit
  int auto_machines = 0;          // SMs x resident CTAs per SM (0: not asked yet)
  struct Sched {
    int n_steps = 0, machines = 0, grid = 0, tail = 0;
    int n_queue = 0, queue_first = 0;  // the shared queue (KRun.n_queue)
    int4 *d_pieces = nullptr;
    int *d_off = nullptr, *d_ticket = nullptr;
    int *d_queue_ctl = nullptr;  // [3]: next queue piece, CTAs done, CTAs started
  };
  std::vector<Sched> scheds;
};

// Trajectory dumps of a run (gd_remc_set_trajectory): a two-dump device
// ring the kernel writes records into, two pinned host slots, and a copy
// stream on which each completed dump is copied and then written to disk by
// a host function (so the compute stream never waits for the disk, only,
// two dumps later, for the copy out of the ring half it is about to reuse).
struct Traj {
  std::string dir, stem;
  int spd = 0;                 // MC steps per dump
  int n_rep = 0;
  int seq = 0;                 // number of the next file
  gd_record *ring = nullptr;   // device [n_rep][2 spd]
  gd_record *host[2] = {nullptr, nullptr};  // pinned [n_rep][spd]
  cudaStream_t copy = nullptr;
  cudaEvent_t done = nullptr;  // end of a dump on the compute stream
  cudaEvent_t copied[2] = {nullptr, nullptr};
  bool pending[2] = {false, false};  // copied[h] not yet waited on
  std::atomic<int> err{0};     // a file could not be written
};

// LigRecordSingleStep (dock.h:487-493) is the first 88 bytes of gd_record.
constexpr size_t kLigRecordBytes = 88;
static_assert(offsetof(gd_record, e_prop_total) == kLigRecordBytes,
              "gd_record must start with the LigRecordSingleStep fields");

struct Ens {
  gd_ctx *ctx = nullptr;
  std::vector<gd_dcomplex *> dcx;
  std::vector<gd_mc_params> mc;
  std::vector<KItem> items;
  KItem *d_items = nullptr;
  int n_rep_total = 0, spe = 0, step = 0;
  float *m_old = nullptr, *e_old = nullptr, *minus_beta = nullptr, *cmcc = nullptr;
  int *idx_tmp = nullptr, *acs_mc = nullptr, *acs_exchg = nullptr, *d_step = nullptr;
  std::vector<Plan> plans;
  KGroup *d_groups = nullptr;
  int n_groups = 0;  // groups exchanged by the separate kernel
  bool all_fused = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  // fused runs (exchange inside the kernel): one captured graph per run
  // length, holding every launch shape's kernel (side by side) and the step
  // counter's advance
  std::map<int, std::pair<cudaGraph_t, cudaGraphExec_t>> fused_graphs;
  std::map<int, int> fused_seen;  // run lengths enqueued so far (capture on the second)
  bool profile = false;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_kind;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timing = false;
  double t_compute = 0.0;
  std::vector<void *> allocs;
  std::unique_ptr<Traj> traj;
};

// Stream-ordered (cudaMallocAsync / cudaFreeAsync on the context stream):
// creating and freeing a run never synchronises the device.
template <typename T>
gd_status dalloc(Ens &E, T **out, size_t n) {
  void *p = nullptr;
  if (injected_alloc_failure(E.ctx))
    return fail(GD_ENOMEM, "cudaMallocAsync of %zu bytes: out of memory (injected)",
                std::max<size_t>(n, 1) * sizeof(T));
  GD_CUDA(cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), E.ctx->stream));
  E.allocs.push_back(p);
  GD_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), E.ctx->stream));
  *out = (T *)p;
  return GD_OK;
}

template <typename T>
gd_status dcopy(Ens &E, T **out, const std::vector<T> &h) {
  GD_TRY(dalloc(E, out, h.size()));
  if (!h.empty())
    GD_CUDA(cudaMemcpyAsync(*out, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice,
                            E.ctx->stream));
  return GD_OK;
}

gd_status validate_mc(const gd_mc_params *mc) {
  if (!mc) return fail(GD_EINVAL, "mc params NULL");
  if (mc->n_tmp < 1 || mc->n_tmp > MAX_TMP)
    return fail(GD_EINVAL, "n_tmp=%d outside [1, %d]", mc->n_tmp, MAX_TMP);
  if (!mc->minus_beta) return fail(GD_EINVAL, "minus_beta NULL");
  if (mc->steps_total < 0) return fail(GD_EINVAL, "steps_total=%d", mc->steps_total);
  if (mc->steps_per_exchange < 1)
    return fail(GD_EINVAL, "steps_per_exchange=%d", mc->steps_per_exchange);
  if (mc->steps_total % mc->steps_per_exchange != 0)
    return fail(GD_EINVAL, "steps_total %d is not a multiple of steps_per_exchange %d",
                mc->steps_total, mc->steps_per_exchange);
  for (int i = 0; i < mc->n_tmp; ++i)
    if (!std::isfinite(mc->minus_beta[i])) return fail(GD_EINVAL, "minus_beta[%d] not finite", i);
  return GD_OK;
}

void ens_free(Ens &E) {
  if (E.ctx) {
    cudaSetDevice(E.ctx->device);
    cudaStreamSynchronize(E.ctx->stream);
  }
  if (E.traj) {
    Traj &t = *E.traj;
    if (t.copy) cudaStreamSynchronize(t.copy);  // copies and file writes
    for (cudaEvent_t e : {t.done, t.copied[0], t.copied[1]})
      if (e) cudaEventDestroy(e);
    if (t.copy) cudaStreamDestroy(t.copy);
    for (gd_record *h : t.host)
      if (h) cudaFreeHost(h);
    E.traj.reset();
  }
  if (E.gexec) cudaGraphExecDestroy(E.gexec);
  if (E.graph) cudaGraphDestroy(E.graph);
  for (auto &kv : E.fused_graphs) {
    if (kv.second.second) cudaGraphExecDestroy(kv.second.second);
    if (kv.second.first) cudaGraphDestroy(kv.second.first);
  }
  E.fused_graphs.clear();
  if (E.ctx)
    for (void *p : E.allocs) cudaFreeAsync(p, E.ctx->stream);
  E.allocs.clear();
  for (cudaEvent_t e : E.prof_ev) cudaEventDestroy(e);
  if (E.ev0) cudaEventDestroy(E.ev0);
  if (E.ev1) cudaEventDestroy(E.ev1);
  for (gd_dcomplex *d : E.dcx) dcx_release(d);
  E.dcx.clear();
  ctx_release(E.ctx);
  E.ctx = nullptr;
}

gd_status ens_build(Ens &E, gd_ctx *ctx, int n, const gd_dcomplex *const *dcx,
                    const gd_mc_params *mc) {
  E.ctx = ctx;
  ctx_retain(ctx);
  if (n < 1) return fail(GD_EINVAL, "no complexes");
  E.spe = mc[0].steps_per_exchange;
  for (int i = 0; i < n; ++i) {
    if (!dcx[i]) return fail(GD_EINVAL, "complex %d is NULL", i);
    if (dcx[i]->ctx != ctx) return fail(GD_EINVAL, "complex %d belongs to another context", i);
    GD_TRY(validate_mc(&mc[i]));
    if (mc[i].steps_per_exchange != E.spe)
      return fail(GD_EINVAL, "complex %d: steps_per_exchange %d differs from %d", i,
                  mc[i].steps_per_exchange, E.spe);
    E.dcx.push_back(const_cast<gd_dcomplex *>(dcx[i]));
    dcx_retain(E.dcx.back());
    E.mc.push_back(mc[i]);
  }
  // replica layout and per-item state
  E.items.resize(n);
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    const KTables &T = E.dcx[i]->T;
    KItem &I = E.items[i];
    I.T = T;
    I.n_tmp = mc[i].n_tmp;
    I.n_lig_conf = T.n_lig;
    I.n_prt = T.n_prt;
    I.n_rep = T.n_prt * T.n_lig * mc[i].n_tmp;
    I.rep_base = (int)total;
    I.steps_per_dump = mc[i].steps_per_dump;
    I.rec_steps = 0;
    for (int k = 0; k < 6; ++k) I.move_scale[k] = mc[i].move_scale[k];
    I.seed = mc[i].seed;
    I.stream_id = mc[i].stream_id;
    I.flags = mc[i].flags;
    I.spe = mc[i].steps_per_exchange;
    total += I.n_rep;
  }
  if (total > (1LL << 30)) return fail(GD_EINVAL, "too many replicas: %lld", total);
  E.n_rep_total = (int)total;
  GD_TRY(dalloc(E, &E.m_old, (size_t)total * 6));
  GD_TRY(dalloc(E, &E.e_old, (size_t)total * GD_NTERM));
  GD_TRY(dalloc(E, &E.cmcc, (size_t)total));
  GD_TRY(dalloc(E, &E.idx_tmp, (size_t)total));
  GD_TRY(dalloc(E, &E.acs_mc, (size_t)total));
  GD_TRY(dalloc(E, &E.acs_exchg, (size_t)n * MAX_TMP));
  GD_TRY(dalloc(E, &E.d_step, 1));
  {
    std::vector<float> mb((size_t)n * MAX_TMP, 0.f);
    for (int i = 0; i < n; ++i)
      std::copy(mc[i].minus_beta, mc[i].minus_beta + mc[i].n_tmp, mb.begin() + (size_t)i * MAX_TMP);
    GD_TRY(dcopy(E, &E.minus_beta, mb));
  }
  for (int i = 0; i < n; ++i) {
    KItem &I = E.items[i];
    I.minus_beta = E.minus_beta + (size_t)i * MAX_TMP;
    I.acs_exchg = E.acs_exchg + (size_t)i * MAX_TMP;
    I.m_old = E.m_old + (size_t)I.rep_base * 6;
    I.e_old = E.e_old + (size_t)I.rep_base * GD_NTERM;
    I.cmcc = E.cmcc + I.rep_base;
    I.idx_tmp = E.idx_tmp + I.rep_base;
    I.acs_mc = E.acs_mc + I.rep_base;
    I.record = nullptr;
    if (mc[i].flags & GD_MC_RECORD) {
      gd_record *rec = nullptr;
      GD_TRY(dalloc(E, &rec, (size_t)I.n_rep * std::max(1, mc[i].steps_total)));
      I.record = rec;
      I.rec_steps = mc[i].steps_total;
    }
  }
  GD_TRY(dcopy(E, &E.d_items, E.items));

  // launch plans: one per (shape, staging, layout); CTAs in decreasing cost
  using Key = std::tuple<int, int, int, int, int, int, int>;
  std::map<Key, std::vector<std::tuple<double, int, int, int>>> ctas;  // cost, item, rep0, n
  std::map<Key, Plan> plans;
  std::vector<KGroup> groups;
  int run_units = 0;  // units of the whole run (the split rule's bound)
  for (const KItem &I : E.items) run_units += units_of(I.n_prt, I.n_lig_conf, I.n_tmp);
  for (int i = 0; i < n; ++i) {
    const KItem &I = E.items[i];
    Tile t = tile_for(ctx, I.T);
    const int split = split_for(ctx, I.T, run_units, kRunSplitCost);
    int ns, res;
    pick_stages(I.T, t, &ns, &res, split);
    const int nt = I.n_tmp, nl = I.n_lig_conf;
    const bool gm = (32 % nt) == 0;
    const bool exch = (I.flags & GD_MC_EXCHANGE) != 0;
    const Key key{t.A, t.P, t.NA, ns, res, gm ? 1 : 0, split};
    Plan &pl = plans[key];
    pl.tile = t;
    pl.split = split;
    pl.n_stages = ns;
    pl.resident = res;
    pl.group_major = gm ? 1 : 0;
    pl.fused = gm ? 1 : 0;
    pl.hb_pairs = std::max(pl.hb_pairs, hb_pairs_of(I.T, t.A));
    const double cost = (double)I.T.lna * I.T.pnp;
    auto &list = ctas[key];
    if (gm) {
      const int G = 32 / nt;
      for (int p = 0; p < I.n_prt; ++p)
        for (int l0 = 0; l0 < nl; l0 += G)
          list.emplace_back(cost, i, p * nl + l0, std::min(G, nl - l0) * nt);
    } else {
      const int per_p = nt * nl;
      for (int p = 0; p < I.n_prt; ++p)
        for (int j = 0; j < per_p; j += 32)
          list.emplace_back(cost, i, p * per_p + j, std::min(32, per_p - j));
      if (exch) {
        E.all_fused = false;
        for (int p = 0; p < I.n_prt; ++p)
          for (int l = 0; l < nl; ++l) groups.push_back(KGroup{i, p, l, 0});
      }
    }
  }
  for (auto &kv : plans) {
    Plan pl = kv.second;
    auto &list = ctas[kv.first];
    std::stable_sort(list.begin(), list.end(),
                     [](const auto &a, const auto &b) { return std::get<0>(a) > std::get<0>(b); });
    std::vector<int> ci, c0, cn;
    for (auto &c : list) {
      ci.push_back(std::get<1>(c));
      c0.push_back(std::get<2>(c));
      cn.push_back(std::get<3>(c));
      pl.cost += std::get<0>(c);
      pl.unit_cost.push_back(std::get<0>(c));
    }
    pl.grid = (int)ci.size();
    GD_TRY(dcopy(E, &pl.d_cta_item, ci));
    GD_TRY(dcopy(E, &pl.d_cta_rep0, c0));
    GD_TRY(dcopy(E, &pl.d_cta_nrep, cn));
    GD_TRY(dalloc(E, &pl.d_progress, ci.size()));
    E.plans.push_back(pl);
  }
  // costliest plans are issued first, so they start first on the SMs
  std::stable_sort(E.plans.begin(), E.plans.end(),
                   [](const Plan &a, const Plan &b) { return a.cost > b.cost; });
  E.n_groups = (int)groups.size();
  if (E.n_groups) GD_TRY(dcopy(E, &E.d_groups, groups));
  {
    // create the side streams now, outside any later stream capture
    cudaStream_t ss[kMaxSide];
    const int ns = std::min((int)E.plans.size(), kMaxSide);
    GD_TRY(fork_streams(ctx, ns, ss));
    GD_TRY(join_streams(ctx, ns));
  }
  GD_CUDA(cudaEventCreate(&E.ev0));
  GD_CUDA(cudaEventCreate(&E.ev1));
  GD_CUDA(cudaStreamSynchronize(ctx->stream));
  return GD_OK;
}

KRun run_desc(const Ens &E, const Plan &pl, int mode) {
  KRun R{};
  R.mode = mode;
  R.A = pl.tile.A;
  R.P = pl.tile.P;
  R.n_stages = pl.n_stages;
  R.resident = pl.resident;
  R.items = E.d_items;
  R.cta_item = pl.d_cta_item;
  R.cta_rep0 = pl.d_cta_rep0;
  R.cta_nrep = pl.d_cta_nrep;
  R.group_major = pl.group_major;
  R.fused_exchange = pl.fused;
  R.spe = E.spe;
  R.err = E.ctx->d_err;
  R.wait_limit = E.ctx->wait_limit;
  R.wait_bias = E.ctx->wait_bias;
  R.hb_pairs = pl.hb_pairs;
  R.split = pl.split;
  return R;
}

// MC steps per unit left to a persistent launch's shared queue: only for a
// run of one launch plan, whose CTAs then normally all fit on the GPU at once
// (CTAs take queue pieces only once all of them have started).
int sched_tail(const Ens &E, int n_steps) {
  if (E.plans.size() != 1) return 0;
  return std::min(E.ctx->sched_tail, n_steps);
}

// Makes (once per launch length) the persistent schedule of every plan that
// the context's schedule mode gives one; called outside stream capture.
gd_status ens_prepare(Ens &E, int n_steps) {
  const int mode = E.ctx->sched_mode;
  if (mode == GD_SCHED_WAVES || n_steps < 2) return GD_OK;
  for (Plan &pl : E.plans) {
    // each plan as if it had the GPU to itself: plans that run side by side
    // are balanced better by the hardware's dynamic CTA placement than by
    // static shares of the SMs (measured on the batched form)
    if (pl.auto_machines == 0) {
      KRun R = run_desc(E, pl, KMODE_REMC);
      int occ = 0;
      GD_CUDA(dock_ctas_per_sm(R, pl.tile.NA, &occ));
      pl.auto_machines = std::max(1, occ) * E.ctx->n_sm;
    }
    const int machines = E.ctx->sched_machines ? E.ctx->sched_machines : pl.auto_machines;
    if (pl.split > 1 || (mode == GD_SCHED_AUTO && pl.grid <= machines)) continue;
    const int tail = sched_tail(E, n_steps);
    bool have = false;
    for (const Plan::Sched &s : pl.scheds)
      have = have || (s.n_steps == n_steps && s.machines == machines && s.tail == tail);
    if (have) continue;
    Plan::Sched s;
    s.n_steps = n_steps;
    s.machines = machines;
    s.tail = tail;
    std::vector<int4> pieces;
    std::vector<int> off;
    if (tail > 0) {
      // a plan alone on the GPU (all its CTAs resident): each unit's last
      // steps go to the shared queue
      s.grid = schedule_queue(pl.unit_cost, std::vector<int>(pl.grid, n_steps), machines, tail,
                              &pieces, &off, &s.n_queue);
      s.queue_first = off[machines];
      GD_TRY(dalloc(E, &s.d_queue_ctl, 3));
    } else {
      s.grid = schedule_pieces(pl.unit_cost, std::vector<int>(pl.grid, n_steps), machines,
                               &pieces, &off);
    }
    GD_TRY(dcopy(E, &s.d_pieces, pieces));
    GD_TRY(dcopy(E, &s.d_off, off));
    GD_TRY(dalloc(E, &s.d_ticket, 1));
    pl.scheds.push_back(s);
  }
  return GD_OK;
}

// The schedule ens_prepare made for this plan and launch length, if any.
const Plan::Sched *find_sched(const Ens &E, const Plan &pl, int n_steps) {
  const int mode = E.ctx->sched_mode;
  if (mode == GD_SCHED_WAVES) return nullptr;
  if (pl.split > 1) return nullptr;  // split plans' staging is per rank: never a schedule
  const int machines = E.ctx->sched_machines ? E.ctx->sched_machines : pl.auto_machines;
  if (mode == GD_SCHED_AUTO && pl.grid <= machines) return nullptr;
  const int tail = sched_tail(E, n_steps);
  for (const Plan::Sched &s : pl.scheds)
    if (s.n_steps == n_steps && s.machines == machines && s.tail == tail) return &s;
  return nullptr;
}

gd_status mark(Ens &E, int kind) {
  cudaEvent_t e;
  GD_CUDA(cudaEventCreate(&e));
  E.prof_ev.push_back(e);
  E.prof_kind.push_back(kind);
  GD_CUDA(cudaEventRecord(e, E.ctx->stream));
  return GD_OK;
}

// One launch per plan, the plans side by side on the context's side streams
// (joined back into ctx->stream).  Profiling brackets the whole group.
gd_status launch_plans(Ens &E, int mode, int step0, int n_steps, bool device_step) {
  const int n = std::min((int)E.plans.size(), kMaxSide);
  cudaStream_t ss[kMaxSide];
  if (E.profile && mode == KMODE_REMC) GD_TRY(mark(E, 0));
  GD_TRY(fork_streams(E.ctx, n, ss));
  for (size_t k = 0; k < E.plans.size(); ++k) {
    const Plan &pl = E.plans[k];
    KRun R = run_desc(E, pl, mode);
    R.step0 = step0;
    R.n_steps = n_steps;
    R.step_ptr = device_step ? E.d_step : nullptr;
    int grid = pl.grid * pl.split;
    if (mode == KMODE_REMC) {
      if (const Plan::Sched *sc = find_sched(E, pl, n_steps)) {
        R.pieces = sc->d_pieces;
        R.n_queue = sc->n_queue;
        R.queue_first = sc->queue_first;
        R.queue_ctl = sc->d_queue_ctl;
        R.piece_off = sc->d_off;
        R.ticket = sc->d_ticket;
        R.progress = pl.d_progress;
        R.split = 1;
        grid = sc->grid;
      }
    }
    GD_CUDA(launch_dock(R, pl.tile.NA, grid, ss[k % n]));
    E.ctx->launches += 1;
  }
  GD_TRY(join_streams(E.ctx, n));
  if (E.profile && mode == KMODE_REMC) GD_TRY(mark(E, 0));
  return GD_OK;
}

gd_status ens_init(Ens &E) {
  GD_CUDA(cudaSetDevice(E.ctx->device));
  cudaStream_t s = E.ctx->stream;
  GD_CUDA(cudaMemsetAsync(E.acs_exchg, 0, sizeof(int) * MAX_TMP * E.items.size(), s));
  GD_CUDA(cudaMemsetAsync(E.d_step, 0, sizeof(int), s));
  for (const Plan &pl : E.plans) {  // progress counts steps from 0 again
    GD_CUDA(cudaMemsetAsync(pl.d_progress, 0, sizeof(int) * std::max(pl.grid, 1), s));
    for (const Plan::Sched &sc : pl.scheds)
      if (sc.d_queue_ctl) GD_CUDA(cudaMemsetAsync(sc.d_queue_ctl, 0, 3 * sizeof(int), s));
  }
  GD_TRY(launch_plans(E, KMODE_INIT, 0, 1, false));
  E.step = 0;
  E.t_compute = 0.0;
  if (E.traj) E.traj->seq = 0;  // a run's files are numbered from 0000
  return GD_OK;
}

// The launches of `k` intervals.  With a device step counter (graph mode)
// every launch reads its first step from it and the last node advances it.
gd_status ens_enqueue(Ens &E, int n_steps, bool device_step) {
  cudaStream_t s = E.ctx->stream;
  if (E.all_fused) {
    // exchanges happen inside the kernel: one launch per plan for the run
    GD_TRY(launch_plans(E, KMODE_REMC, E.step, n_steps, device_step));
    if (device_step) {
      GD_CUDA(launch_advance(E.d_step, n_steps, s));
      E.ctx->launches += 1;
    }
    return GD_OK;
  }
  for (int s0 = E.step; s0 < E.step + n_steps; s0 += E.spe) {
    GD_TRY(launch_plans(E, KMODE_REMC, s0, E.spe, device_step));
    if (E.n_groups) {
      if (E.profile) GD_TRY(mark(E, 1));
      GD_CUDA(launch_exchange(E.d_items, E.d_groups, E.n_groups, E.spe, s0,
                              device_step ? E.d_step : nullptr, s));
      if (E.profile) GD_TRY(mark(E, 1));
      E.ctx->launches += 1;
    }
    if (device_step) {
      GD_CUDA(launch_advance(E.d_step, E.spe, s));
      E.ctx->launches += 1;
    }
  }
  return GD_OK;
}

// n_steps (a multiple of spe) MC steps of every replica, enqueued.
gd_status ens_run_steps(Ens &E, int n_steps) {
  cudaStream_t s = E.ctx->stream;
  // launch length: the whole run when the exchange is inside the kernel,
  // else one interval (per launch, or in the captured graph)
  GD_TRY(ens_prepare(E, E.all_fused ? n_steps : E.spe));
  // keep the device step counter in step with the host's
  GD_CUDA(cudaMemcpyAsync(E.d_step, &E.step, sizeof(int), cudaMemcpyHostToDevice, s));
  if (E.profile || (E.all_fused && E.fused_seen[n_steps]++ == 0)) {
    // profiling brackets each launch; a run length seen for the first time
    // (a one-shot run) is not worth a capture
    GD_TRY(ens_enqueue(E, n_steps, false));
  } else if (E.all_fused) {
    // the whole run is one launch per shape: captured once per run length
    // (on its second use) and replayed as one graph launch (the kernels read
    // the first step from the device counter)
    auto it = E.fused_graphs.find(n_steps);
    if (it == E.fused_graphs.end()) {
      GD_CUDA(cudaStreamSynchronize(s));
      GD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const uint64_t l0 = E.ctx->launches;
      gd_status st = ens_enqueue(E, n_steps, true);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      E.ctx->launches = l0;  // counted when replayed
      if (st != GD_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      if (ce != cudaSuccess) return fail(GD_ECUDA, "graph capture: %s", cudaGetErrorString(ce));
      cudaGraphExec_t ge = nullptr;
      ce = cudaGraphInstantiate(&ge, g, 0);
      if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(GD_ECUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      }
      it = E.fused_graphs.emplace(n_steps, std::make_pair(g, ge)).first;
    }
    GD_CUDA(cudaGraphLaunch(it->second.second, s));
    E.ctx->launches += (int)E.plans.size() + 1;
  } else {
    // one captured interval, replayed n_steps / spe times
    if (!E.gexec) {
      GD_CUDA(cudaStreamSynchronize(s));
      GD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int saved = E.step;
      const uint64_t l0 = E.ctx->launches;
      gd_status st = ens_enqueue(E, E.spe, true);
      E.step = saved;
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (st != GD_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      if (ce != cudaSuccess) return fail(GD_ECUDA, "graph capture: %s", cudaGetErrorString(ce));
      E.graph = g;
      GD_CUDA(cudaGraphInstantiate(&E.gexec, g, 0));
      E.ctx->launches = l0;  // counted when replayed
    }
    const int per_graph = (int)E.plans.size() + (E.n_groups ? 1 : 0) + 1;
    for (int k = 0; k < n_steps / E.spe; ++k) {
      GD_CUDA(cudaGraphLaunch(E.gexec, s));
      E.ctx->launches += per_graph;
    }
  }
  E.step += n_steps;
  return GD_OK;
}

// Writes the file of a dump after its records are copied out of ring half h.
void CUDART_CB write_dump(void *arg);

struct DumpJob {
  Traj *t;
  int slot, seq;
};

void CUDART_CB write_dump(void *arg) {
  DumpJob *j = static_cast<DumpJob *>(arg);
  Traj &t = *j->t;
  char num[16];
  std::snprintf(num, sizeof num, "%04d", j->seq);
  const std::string path = t.dir + "/" + t.stem + "_" + num + ".bin";
  FILE *f = std::fopen(path.c_str(), "wb");
  bool ok = f != nullptr;
  // pack the records to their 88-byte LigRecordSingleStep form in chunks
  const gd_record *r = t.host[j->slot];
  const size_t n = (size_t)t.n_rep * t.spd, chunk = 8192;
  std::vector<unsigned char> buf;
  for (size_t k0 = 0; ok && k0 < n; k0 += chunk) {
    const size_t m = std::min(chunk, n - k0);
    buf.resize(m * kLigRecordBytes);
    for (size_t k = 0; k < m; ++k)
      std::memcpy(buf.data() + k * kLigRecordBytes, &r[k0 + k], kLigRecordBytes);
    ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  }
  if (f && std::fclose(f) != 0) ok = false;
  if (!ok) t.err.store(1);
  delete j;
}

// Copies the completed dump in ring half h out and queues its file.
gd_status traj_dump(Ens &E, int h) {
  Traj &t = *E.traj;
  const size_t w = sizeof(gd_record) * t.spd;
  GD_CUDA(cudaEventRecord(t.done, E.ctx->stream));
  GD_CUDA(cudaStreamWaitEvent(t.copy, t.done, 0));
  GD_CUDA(cudaMemcpy2DAsync(t.host[h], w, t.ring + (size_t)h * t.spd, 2 * w, w, t.n_rep,
                            cudaMemcpyDeviceToHost, t.copy));
  GD_CUDA(cudaEventRecord(t.copied[h], t.copy));
  t.pending[h] = true;
  DumpJob *j = new (std::nothrow) DumpJob{&t, h, t.seq};
  if (!j) return fail(GD_ENOMEM, "host allocation");
  const cudaError_t e = cudaLaunchHostFunc(t.copy, write_dump, j);
  if (e != cudaSuccess) {
    delete j;
    return fail(GD_ECUDA, "cudaLaunchHostFunc: %s", cudaGetErrorString(e));
  }
  t.seq += 1;
  return GD_OK;
}

gd_status ens_run(Ens &E, int n_steps) {
  if (n_steps < 0 || n_steps % E.spe != 0)
    return fail(GD_EINVAL, "n_steps %d is not a multiple of steps_per_exchange %d", n_steps,
                E.spe);
  if (E.traj && E.traj->err.load())
    return fail(GD_EIO, "a trajectory file under %s could not be written", E.traj->dir.c_str());
  if (n_steps == 0) return GD_OK;
  GD_CUDA(cudaSetDevice(E.ctx->device));
  cudaStream_t s = E.ctx->stream;
  GD_CUDA(cudaEventRecord(E.ev0, s));
  if (!E.traj) {
    GD_TRY(ens_run_steps(E, n_steps));
  } else {
    // segments end at dump boundaries, where the completed dump is copied out
    Traj &t = *E.traj;
    for (int left = n_steps; left > 0;) {
      const int in_dump = E.step % t.spd;
      const int h = (E.step / t.spd) % 2;
      const int seg = std::min(left, t.spd - in_dump);
      if (in_dump == 0 && t.pending[h]) {  // the copy of two dumps ago
        GD_CUDA(cudaStreamWaitEvent(s, t.copied[h], 0));
        t.pending[h] = false;
      }
      GD_TRY(ens_run_steps(E, seg));
      left -= seg;
      if (E.step % t.spd == 0) GD_TRY(traj_dump(E, h));
    }
  }
  GD_CUDA(cudaEventRecord(E.ev1, s));
  E.timing = true;
  return GD_OK;
}

// Layout descriptor of the dump files (JSON).
bool write_layout(const Traj &t, const KItem &I) {
  const std::string path = t.dir + "/" + t.stem + ".layout.json";
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  std::fprintf(f,
               "{\n"
               "  \"format\": \"LigRecord dumps: the contents of dataset 'dset' written by "
               "DumpLigRecord (hdf5io.C), one file per dump, native little-endian\",\n"
               "  \"files\": \"%s_%%04d.bin\",\n"
               "  \"dataset\": \"dset\",\n"
               "  \"shape\": [%d],\n"
               "  \"element\": {\"name\": \"LigRecord\", \"field\": \"step\", "
               "\"count\": %d, \"bytes\": %zu},\n"
               "  \"record\": {\"name\": \"LigRecordSingleStep\", \"bytes\": %zu, "
               "\"fields\": [\n"
               "    {\"name\": \"replica.idx_rep\", \"offset\": 0, \"type\": \"int32\"},\n"
               "    {\"name\": \"replica.idx_prt\", \"offset\": 4, \"type\": \"int32\"},\n"
               "    {\"name\": \"replica.idx_tmp\", \"offset\": 8, \"type\": \"int32\"},\n"
               "    {\"name\": \"replica.idx_lig\", \"offset\": 12, \"type\": \"int32\"},\n"
               "    {\"name\": \"energy.e\", \"offset\": 16, \"type\": \"float32\", "
               "\"shape\": [%d]},\n"
               "    {\"name\": \"energy.cmcc\", \"offset\": 56, \"type\": \"float32\"},\n"
               "    {\"name\": \"movematrix\", \"offset\": 60, \"type\": \"float32\", "
               "\"shape\": [6]},\n"
               "    {\"name\": \"step\", \"offset\": 84, \"type\": \"int32\"}]},\n"
               "  \"steps_per_dump\": %d,\n"
               "  \"n_rep\": %d, \"n_prt\": %d, \"n_tmp\": %d, \"n_lig\": %d\n"
               "}\n",
               t.stem.c_str(), t.n_rep, t.spd, kLigRecordBytes * t.spd, kLigRecordBytes,
               GD_NTERM, t.spd, t.n_rep, I.n_prt, I.n_tmp, I.n_lig_conf);
  return std::fclose(f) == 0;
}

gd_status ens_set_trajectory(Ens &E, const char *dir, const char *stem) {
  if (!dir || !*dir || !stem || !*stem || std::strchr(stem, '/'))
    return fail(GD_EINVAL, "trajectory: directory and a file stem without '/' are required");
  if (E.items.size() != 1) return fail(GD_EINVAL, "trajectory: one complex per run");
  if (E.traj) return fail(GD_EINVAL, "trajectory: already set");
  const int spd = E.mc[0].steps_per_dump;
  if (spd <= 0 || spd % E.spe != 0)
    return fail(GD_EINVAL, "trajectory: steps_per_dump %d must be a positive multiple of "
                "steps_per_exchange %d", spd, E.spe);
  KItem &I = E.items[0];
  std::unique_ptr<Traj> t(new (std::nothrow) Traj);
  if (!t) return fail(GD_ENOMEM, "host allocation");
  t->dir = dir;
  t->stem = stem;
  t->spd = spd;
  t->n_rep = I.n_rep;
  if (!write_layout(*t, I))
    return fail(GD_EIO, "trajectory: cannot write %s/%s.layout.json", dir, stem);
  GD_CUDA(cudaSetDevice(E.ctx->device));
  GD_TRY(dalloc(E, &t->ring, (size_t)I.n_rep * 2 * spd));
  E.traj = std::move(t);  // freed by ens_free from here on
  Traj &T = *E.traj;
  for (gd_record *&h : T.host)
    GD_CUDA(cudaMallocHost(&h, sizeof(gd_record) * (size_t)I.n_rep * spd));
  GD_CUDA(cudaStreamCreateWithFlags(&T.copy, cudaStreamNonBlocking));
  GD_CUDA(cudaEventCreateWithFlags(&T.done, cudaEventDisableTiming));
  for (cudaEvent_t &e : T.copied) GD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  I.record = T.ring;
  I.rec_steps = 2 * spd;
  I.rec_ring = 1;
  GD_CUDA(cudaMemcpyAsync(E.d_items, E.items.data(), sizeof(KItem) * E.items.size(),
                          cudaMemcpyHostToDevice, E.ctx->stream));
  GD_CUDA(cudaStreamSynchronize(E.ctx->stream));
  return GD_OK;
}

gd_status ens_read(Ens &E, int i, gd_mc_log *log) {
  if (i < 0 || i >= (int)E.items.size()) return fail(GD_EINVAL, "item %d out of range", i);
  GD_CUDA(cudaSetDevice(E.ctx->device));
  GD_TRY(ctx_check(E.ctx));
  if (E.traj) {  // every queued dump is on disk
    GD_CUDA(cudaStreamSynchronize(E.traj->copy));
    if (E.traj->err.load())
      return fail(GD_EIO, "a trajectory file under %s could not be written",
                  E.traj->dir.c_str());
  }
  if (E.timing) {
    float ms = 0.f;
    GD_CUDA(cudaEventElapsedTime(&ms, E.ev0, E.ev1));
    E.t_compute += ms * 1e-3;
    E.timing = false;
  }
  const KItem &I = E.items[i];
  const size_t n = (size_t)I.n_rep, b = (size_t)I.rep_base;
  std::vector<int> acs(n), acx(I.n_tmp);
  cudaStream_t s = E.ctx->stream;
  GD_CUDA(cudaMemcpyAsync(acs.data(), E.acs_mc + b, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaMemcpyAsync(acx.data(), I.acs_exchg, sizeof(int) * I.n_tmp, cudaMemcpyDeviceToHost,
                          s));
  if (log->energy)
    GD_CUDA(cudaMemcpyAsync(log->energy, E.e_old + b * GD_NTERM, sizeof(float) * GD_NTERM * n,
                            cudaMemcpyDeviceToHost, s));
  if (log->movematrix)
    GD_CUDA(cudaMemcpyAsync(log->movematrix, E.m_old + b * 6, sizeof(float) * 6 * n,
                            cudaMemcpyDeviceToHost, s));
  if (log->idx_tmp)
    GD_CUDA(cudaMemcpyAsync(log->idx_tmp, E.idx_tmp + b, sizeof(int) * n, cudaMemcpyDeviceToHost,
                            s));
  if (log->record && I.record && !I.rec_ring)
    GD_CUDA(cudaMemcpyAsync(log->record, I.record, sizeof(gd_record) * n * std::max(1, I.rec_steps),
                            cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaStreamSynchronize(s));
  log->ac_mc = 0;
  for (size_t k = 0; k < n; ++k) log->ac_mc += acs[k];
  log->ac_temp_exchg = 0;
  for (int t = 0; t < I.n_tmp; ++t) log->ac_temp_exchg += acx[t];
  if (log->acs_mc) std::memcpy(log->acs_mc, acs.data(), sizeof(int) * n);
  if (log->acs_temp_exchg) std::memcpy(log->acs_temp_exchg, acx.data(), sizeof(int) * I.n_tmp);
  log->t_compute = E.t_compute;
  return GD_OK;
}

// Snapshot of a run's state (gd_remc_snapshot / gd_batch_snapshot): a header
// that identifies the run's shape, then the replica state and counters as
// the kernels keep them.  The random stream needs no state: Philox is keyed
// by (seed, stream id) and counted by (replica, step), so restoring the
// state and the step counter continues the run bit for bit.
struct SnapHeader {
  char magic[8];
  int32_t version, n_items, n_rep_total, step, spe, pad;
};
constexpr char kSnapMagic[8] = {'G', 'D', 'S', 'N', 'A', 'P', '1', 0};
struct SnapItem {
  int32_t n_rep, n_tmp, lna, pnp;
  uint64_t seed;
  uint32_t stream_id, flags;
};

size_t snap_bytes(const Ens &E) {
  const size_t n = (size_t)E.n_rep_total;
  return sizeof(SnapHeader) + sizeof(SnapItem) * E.items.size() +
         n * sizeof(float) * (6 + GD_NTERM + 1) + n * sizeof(int) * 2 +
         E.items.size() * MAX_TMP * sizeof(int);
}

// The state arrays in blob order: {device pointer, bytes}.
std::vector<std::pair<void *, size_t>> snap_arrays(const Ens &E) {
  const size_t n = (size_t)E.n_rep_total;
  return {{E.m_old, n * 6 * sizeof(float)},
          {E.e_old, n * GD_NTERM * sizeof(float)},
          {E.cmcc, n * sizeof(float)},
          {E.idx_tmp, n * sizeof(int)},
          {E.acs_mc, n * sizeof(int)},
          {E.acs_exchg, E.items.size() * MAX_TMP * sizeof(int)}};
}

SnapItem snap_item(const Ens &E, size_t i) {
  const KItem &I = E.items[i];
  return SnapItem{I.n_rep, I.n_tmp, I.T.lna, I.T.pnp, E.mc[i].seed, E.mc[i].stream_id,
                  E.mc[i].flags};
}

gd_status ens_snapshot(Ens &E, void *buf, size_t cap, size_t *size) {
  const size_t need = snap_bytes(E);
  if (size) *size = need;
  if (!buf) return GD_OK;  // size query
  if (cap < need) return fail(GD_EINVAL, "snapshot needs %zu bytes, buffer holds %zu", need, cap);
  GD_CUDA(cudaSetDevice(E.ctx->device));
  GD_TRY(ctx_check(E.ctx));  // the state is complete and no kernel reported an error
  unsigned char *p = static_cast<unsigned char *>(buf);
  SnapHeader h{};
  std::memcpy(h.magic, kSnapMagic, sizeof h.magic);
  h.version = 1;
  h.n_items = (int32_t)E.items.size();
  h.n_rep_total = E.n_rep_total;
  h.step = E.step;
  h.spe = E.spe;
  std::memcpy(p, &h, sizeof h);
  p += sizeof h;
  for (size_t i = 0; i < E.items.size(); ++i) {
    const SnapItem it = snap_item(E, i);
    std::memcpy(p, &it, sizeof it);
    p += sizeof it;
  }
  for (const auto &a : snap_arrays(E)) {
    GD_CUDA(cudaMemcpyAsync(p, a.first, a.second, cudaMemcpyDeviceToHost, E.ctx->stream));
    p += a.second;
  }
  GD_CUDA(cudaStreamSynchronize(E.ctx->stream));
  return GD_OK;
}

gd_status ens_restore(Ens &E, const void *buf, size_t size) {
  if (!buf) return fail(GD_EINVAL, "snapshot buffer NULL");
  if (size != snap_bytes(E))
    return fail(GD_EINVAL, "snapshot of %zu bytes does not fit this run (%zu bytes)", size,
                snap_bytes(E));
  const unsigned char *p = static_cast<const unsigned char *>(buf);
  SnapHeader h;
  std::memcpy(&h, p, sizeof h);
  p += sizeof h;
  if (std::memcmp(h.magic, kSnapMagic, sizeof h.magic) != 0 || h.version != 1)
    return fail(GD_EINVAL, "not a run snapshot of this library");
  if (h.n_items != (int32_t)E.items.size() || h.n_rep_total != E.n_rep_total ||
      h.spe != E.spe || h.step < 0 || h.step % E.spe != 0)
    return fail(GD_EINVAL, "snapshot of a run of another shape (items %d, replicas %d, "
                           "steps per exchange %d, step %d)",
                h.n_items, h.n_rep_total, h.spe, h.step);
  for (size_t i = 0; i < E.items.size(); ++i) {
    SnapItem it;
    std::memcpy(&it, p, sizeof it);
    p += sizeof it;
    const SnapItem mine = snap_item(E, i);
    if (std::memcmp(&it, &mine, sizeof it) != 0)
      return fail(GD_EINVAL, "snapshot item %zu has another complex size or random stream", i);
  }
  GD_CUDA(cudaSetDevice(E.ctx->device));
  cudaStream_t s = E.ctx->stream;
  for (const auto &a : snap_arrays(E)) {
    GD_CUDA(cudaMemcpyAsync(a.first, p, a.second, cudaMemcpyHostToDevice, s));
    p += a.second;
  }
  // progress words count absolute steps and only ever grow within a run:
  // start them again below the restored step
  for (const Plan &pl : E.plans) {
    GD_CUDA(cudaMemsetAsync(pl.d_progress, 0, sizeof(int) * std::max(pl.grid, 1), s));
    for (const Plan::Sched &sc : pl.scheds)
      if (sc.d_queue_ctl) GD_CUDA(cudaMemsetAsync(sc.d_queue_ctl, 0, 3 * sizeof(int), s));
  }
  GD_CUDA(cudaStreamSynchronize(s));  // the host buffer may be reused on return
  E.step = h.step;
  if (E.traj) E.traj->seq = E.traj->spd > 0 ? h.step / E.traj->spd : 0;
  return GD_OK;
}

gd_status ens_kernel_times(Ens &E, double *mc_ms, int *mc_n, double *ex_ms, int *ex_n) {
  GD_CUDA(cudaSetDevice(E.ctx->device));
  GD_CUDA(cudaStreamSynchronize(E.ctx->stream));
  *mc_ms = *ex_ms = 0.0;
  *mc_n = *ex_n = 0;
  for (size_t i = 0; i + 1 < E.prof_ev.size(); i += 2) {
    float ms = 0.f;
    GD_CUDA(cudaEventElapsedTime(&ms, E.prof_ev[i], E.prof_ev[i + 1]));
    if (E.prof_kind[i] == 0) {
      *mc_ms += ms;
      *mc_n += 1;
    } else {
      *ex_ms += ms;
      *ex_n += 1;
    }
  }
  for (cudaEvent_t e : E.prof_ev) cudaEventDestroy(e);
  E.prof_ev.clear();
  E.prof_kind.clear();
  return GD_OK;
}

}  // namespace

struct gd_remc {
  Ens e;
};
struct gd_batch {
  Ens e;
};

// ---------------------------------------------------------------------------
// Plain form: one complex
// ---------------------------------------------------------------------------
extern "C" gd_status gd_remc_create(gd_ctx *ctx, const gd_dcomplex *d, const gd_mc_params *mc,
                                    gd_remc **out) {
  if (!ctx || !d || !out) return fail(GD_EINVAL, "gd_remc_create: NULL argument");
  *out = nullptr;
  GD_TRY(validate_mc(mc));
  GD_CUDA(cudaSetDevice(ctx->device));
  gd_remc *r = new (std::nothrow) gd_remc;
  if (!r) return fail(GD_ENOMEM, "host allocation");
  gd_status st;
  try {
    st = ens_build(r->e, ctx, 1, &d, mc);
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation");
  }
  if (st != GD_OK) {
    ens_free(r->e);
    delete r;
    return st;
  }
  *out = r;
  return GD_OK;
}

extern "C" gd_status gd_remc_destroy(gd_remc *r) {
  if (!r) return GD_OK;
  ens_free(r->e);
  delete r;
  return GD_OK;
}

extern "C" int gd_remc_n_rep(const gd_remc *r) { return r ? r->e.n_rep_total : 0; }

extern "C" gd_status gd_remc_init(gd_remc *r) {
  NvtxRange nvtx("gd_remc_init");
  if (!r) return fail(GD_EINVAL, "remc NULL");
  return ens_init(r->e);
}

extern "C" gd_status gd_remc_run(gd_remc *r, int n_steps) {
  NvtxRange nvtx("gd_remc_run");
  if (!r) return fail(GD_EINVAL, "remc NULL");
  return ens_run(r->e, n_steps);
}

extern "C" gd_status gd_remc_read(gd_remc *r, gd_mc_log *log) {
  if (!r || !log) return fail(GD_EINVAL, "gd_remc_read: NULL argument");
  return ens_read(r->e, 0, log);
}

extern "C" gd_status gd_remc_snapshot(gd_remc *r, void *buf, size_t cap, size_t *size) {
  if (!r) return fail(GD_EINVAL, "remc is NULL");
  return ens_snapshot(r->e, buf, cap, size);
}

extern "C" gd_status gd_remc_restore(gd_remc *r, const void *buf, size_t size) {
  if (!r) return fail(GD_EINVAL, "remc is NULL");
  return ens_restore(r->e, buf, size);
}

extern "C" gd_status gd_remc_set_trajectory(gd_remc *r, const char *dir, const char *stem) {
  if (!r) return fail(GD_EINVAL, "remc NULL");
  return ens_set_trajectory(r->e, dir, stem);
}

extern "C" gd_status gd_remc_set_profiling(gd_remc *r, int on) {
  if (!r) return fail(GD_EINVAL, "remc NULL");
  r->e.profile = on != 0;
  return GD_OK;
}

extern "C" gd_status gd_remc_kernel_times(gd_remc *r, double *mc_ms, int *mc_launches,
                                          double *exch_ms, int *exch_launches) {
  if (!r || !mc_ms || !mc_launches || !exch_ms || !exch_launches)
    return fail(GD_EINVAL, "gd_remc_kernel_times: NULL argument");
  return ens_kernel_times(r->e, mc_ms, mc_launches, exch_ms, exch_launches);
}

extern "C" gd_status gd_run(const gd_complex *cx, const gd_mc_params *mc, gd_mc_log *log) {
  NvtxRange nvtx("gd_run");
  const auto t0 = std::chrono::steady_clock::now();
  GD_TRY(validate_mc(mc));
  // one context per calling thread, kept between calls (its stream, side
  // streams and launch-shape cache); everything of the run itself is
  // stream-ordered and released at the end of the call
  thread_local gd_ctx *ctx = nullptr;
  if (!ctx) GD_TRY(gd_ctx_create(0, nullptr, &ctx));
  GD_CUDA(cudaSetDevice(ctx->device));
  gd_dcomplex *d = nullptr;
  gd_remc *r = nullptr;
  gd_status st = gd_complex_upload(ctx, cx, &d);
  if (st == GD_OK) st = gd_remc_create(ctx, d, mc, &r);
  if (st == GD_OK) st = gd_remc_init(r);
  if (st == GD_OK) st = gd_remc_run(r, mc->steps_total);
  if (st == GD_OK && log) st = gd_remc_read(r, log);
  gd_remc_destroy(r);
  gd_complex_free(d);
  if (st == GD_OK && log)
    log->t_wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return st;
}

// ---------------------------------------------------------------------------
// Batched form: many complexes (uneven sizes) advanced together
// ---------------------------------------------------------------------------
extern "C" gd_status gd_batch_create(gd_ctx *ctx, int n, const gd_dcomplex *const *items,
                                     const gd_mc_params *params, gd_batch **out) {
  if (!ctx || !items || !params || !out) return fail(GD_EINVAL, "gd_batch_create: NULL argument");
  *out = nullptr;
  GD_CUDA(cudaSetDevice(ctx->device));
  gd_batch *b = new (std::nothrow) gd_batch;
  if (!b) return fail(GD_ENOMEM, "host allocation");
  gd_status st;
  try {
    st = ens_build(b->e, ctx, n, items, params);
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation");
  }
  if (st != GD_OK) {
    ens_free(b->e);
    delete b;
    return st;
  }
  *out = b;
  return GD_OK;
}

extern "C" gd_status gd_batch_destroy(gd_batch *b) {
  if (!b) return GD_OK;
  ens_free(b->e);
  delete b;
  return GD_OK;
}

extern "C" int gd_batch_n_rep(const gd_batch *b) { return b ? b->e.n_rep_total : 0; }
extern "C" int gd_batch_n_launch_shapes(const gd_batch *b) {
  return b ? (int)b->e.plans.size() : 0;
}

extern "C" gd_status gd_batch_init(gd_batch *b) {
  NvtxRange nvtx("gd_batch_init");
  if (!b) return fail(GD_EINVAL, "batch NULL");
  return ens_init(b->e);
}

extern "C" gd_status gd_batch_run(gd_batch *b, int n_steps) {
  NvtxRange nvtx("gd_batch_run");
  if (!b) return fail(GD_EINVAL, "batch NULL");
  return ens_run(b->e, n_steps);
}

extern "C" gd_status gd_batch_read(gd_batch *b, int item, gd_mc_log *log) {
  if (!b || !log) return fail(GD_EINVAL, "gd_batch_read: NULL argument");
  return ens_read(b->e, item, log);
}

extern "C" gd_status gd_batch_snapshot(gd_batch *b, void *buf, size_t cap, size_t *size) {
  if (!b) return fail(GD_EINVAL, "batch is NULL");
  return ens_snapshot(b->e, buf, cap, size);
}

extern "C" gd_status gd_batch_restore(gd_batch *b, const void *buf, size_t size) {
  if (!b) return fail(GD_EINVAL, "batch is NULL");
  return ens_restore(b->e, buf, size);
}

extern "C" gd_status gd_batch_set_profiling(gd_batch *b, int on) {
  if (!b) return fail(GD_EINVAL, "batch NULL");
  b->e.profile = on != 0;
  return GD_OK;
}

extern "C" gd_status gd_batch_kernel_times(gd_batch *b, double *mc_ms, int *mc_launches,
                                           double *exch_ms, int *exch_launches) {
  if (!b || !mc_ms || !mc_launches || !exch_ms || !exch_launches)
    return fail(GD_EINVAL, "gd_batch_kernel_times: NULL argument");
  return ens_kernel_times(b->e, mc_ms, mc_launches, exch_ms, exch_launches);
}

// ---------------------------------------------------------------------------
// Launch-shape autotuner.  Every compiled shape that covers the complex's
// ligand-size bucket is timed on the REMC kernel itself: a temporary batch of
// copies of the complex, 32 temperatures per exchange group (one group per
// CTA, exchange inside the kernel), at least one CTA per SM, a few MC steps
// per sample.  The fastest shape is cached in the context for the size class
// (bucket, protein tiles) and used by every later launch of that class.
// ---------------------------------------------------------------------------
namespace {

gd_status time_shape(gd_ctx *ctx, const gd_dcomplex *d, const std::vector<gd_mc_params> &mc,
                     int n_items, int steps, float *ms) {
  std::vector<const gd_dcomplex *> ds(n_items, d);
  Ens E;
  gd_status st = ens_build(E, ctx, n_items, ds.data(), mc.data());
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (st == GD_OK) st = ens_init(E);
  if (st == GD_OK) st = ens_run(E, steps);  // warm-up
  if (st == GD_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    st = fail(GD_ECUDA, "autotune: event creation");
  float best = 1e30f;
  for (int rep = 0; rep < 2 && st == GD_OK; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    st = ens_run(E, steps);
    cudaEventRecord(e1, ctx->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(GD_ECUDA, "autotune: sync");
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    best = std::min(best, t);
  }
  if (st == GD_OK) st = ctx_check(ctx);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  ens_free(E);
  *ms = best;
  return st;
}

}  // namespace

extern "C" gd_status gd_autotune(gd_ctx *ctx, const gd_dcomplex *d, gd_tile *best,
                                 double *best_ms) {
  if (!ctx || !d) return fail(GD_EINVAL, "gd_autotune: NULL handle");
  if (d->ctx != ctx) return fail(GD_EINVAL, "gd_autotune: complex belongs to another context");
  GD_CUDA(cudaSetDevice(ctx->device));
  const KTables &T = d->T;
  const int hi = lna_bucket(T.lna);  // the shape must cover the whole bucket
  const std::pair<int, int> key{hi, (T.pnp + TILE_PTS - 1) / TILE_PTS};
  // 32 temperatures: one exchange group fills a CTA whatever the complex's
  // conformation counts; enough copies for one CTA per SM
  constexpr int kTmp = 32, kSpe = 2, kSteps = 4;
  std::vector<float> mb(kTmp);
  for (int t = 0; t < kTmp; ++t) mb[t] = -1.0f / (0.004f * powf(10.0f, t / (float)(kTmp - 1)));
  const int groups = T.n_prt * T.n_lig;
  const int n_items = std::max(1, std::min(256, (ctx->n_sm + groups - 1) / groups));
  gd_mc_params p{};
  p.steps_total = 1 << 20;
  p.steps_per_exchange = kSpe;
  p.steps_per_dump = 0;
  p.n_tmp = kTmp;
  for (int i = 0; i < 6; ++i) p.move_scale[i] = i < 3 ? 0.02f : 0.08f;
  p.minus_beta = mb.data();
  p.seed = 12345;
  p.flags = GD_MC_EXCHANGE;
  std::vector<gd_mc_params> mc(n_items, p);
  for (int i = 0; i < n_items; ++i) mc[i].stream_id = (uint32_t)i;

  bool had = false;
  Tile prev;
  {
    std::lock_guard<std::mutex> g(ctx->tile_mu);
    auto it = ctx->tiles.find(key);
    if (it != ctx->tiles.end()) {
      had = true;
      prev = it->second;
    }
  }
  Tile best_t;
  float best_time = 1e30f;
  gd_status st = GD_OK;
  for (int na : kNAValues) {
    const int A = (hi + na - 1) / na;
    if (A > MAX_WARPS || (A > 1 && round_na((hi + A - 1) / A) != na)) continue;
    for (int P = 1; A * P <= MAX_WARPS && st == GD_OK; ++P) {
      Tile t;
      t.A = A;
      t.P = P;
      t.NA = na;
      if (A * P < 4 && A * P * 2 <= MAX_WARPS) continue;  // too few warps per SM
      {
        std::lock_guard<std::mutex> g(ctx->tile_mu);
        ctx->tiles[key] = t;
      }
      float ms = 1e30f;
      st = time_shape(ctx, d, mc, n_items, kSteps, &ms);
      if (st == GD_OK && ms < best_time) {
        best_time = ms;
        best_t = t;
      }
    }
    if (st != GD_OK) break;
  }
  {
    std::lock_guard<std::mutex> g(ctx->tile_mu);
    if (st == GD_OK && best_t.valid())
      ctx->tiles[key] = best_t;
    else if (had)
      ctx->tiles[key] = prev;
    else
      ctx->tiles.erase(key);
  }
  GD_TRY(st);
  if (!best_t.valid()) return fail(GD_EINVAL, "no launch shape fits lna=%d", T.lna);
  if (best) {
    best->atom_groups = best_t.A;
    best->tile_groups = best_t.P;
    best->atoms_per_warp = best_t.NA;
  }
  if (best_ms) *best_ms = best_time;
  return GD_OK;
}
