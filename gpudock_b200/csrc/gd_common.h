// gd_common.h -- host-side internals shared by gd_api.cu and gd_ensemble.cu:
// the opaque handle types, error reporting and launch-shape selection.
#pragma once

#include <atomic>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "gd_internal.h"

namespace gd {

gd_status fail(gd_status st, const char *fmt, ...);

#define GD_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return ::gd::fail(e_ == cudaErrorMemoryAllocation ? GD_ENOMEM : GD_ECUDA,          \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,      \
                        __LINE__);                                                      \
  } while (0)

#define GD_TRY(call)            \
  do {                          \
    gd_status s_ = (call);      \
    if (s_ != GD_OK) return s_; \
  } while (0)

constexpr float kPI = 3.1415926535f;  // size.h:86

// NVTX range over a host call (shown by profilers that attach a tool; free
// otherwise).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// Launch shape of the energy kernel: A atom groups x P tile groups of warps,
// NA ligand atoms per warp.
struct Tile {
  int A = 0, P = 0, NA = 0;
  bool valid() const { return A > 0 && P > 0 && NA > 0; }
};

// Candidate atoms-per-warp values compiled into the kernel.
// Even: the pair loop handles two atoms per packed f32x2 instruction.
constexpr int kNAValues[] = {2, 4, 6, 8, 10};

Tile default_tile(int lna);
int round_na(int na);  // smallest compiled NA >= na (0 if none)
// Resident staging when the tiles of one CTA (of a split's busiest CTA) fit
// in shared memory, else the streaming ring.
void pick_stages(const KTables &T, const Tile &t, int *n_stages, int *resident, int split = 1);

}  // namespace gd

// Handles are reference counted: a complex keeps its context (and a shared
// protein's owner) alive, a REMC run or batch keeps its complexes alive, so
// callers may destroy them in any order.
struct gd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int *d_err = nullptr;
  uint64_t launches = 0;
  int n_sm = 148;
  int sched_mode = 0;      // GD_SCHED_*
  int sched_machines = 0;  // persistent CTAs (0: SMs x occupancy)
  int sched_tail = 2;      // last MC steps of every unit left to the shared queue
  int split_mode = 0;      // CTAs per unit of MC launches (0: split_for's rule)
  uint32_t wait_limit = 0; // polls of a dependency wait before it gives up (0: default)
  int wait_bias = 0;       // added to every dependency wait's target (test hook)
  std::atomic<int> alloc_fail_in{0};  // > 0: that many device allocations from now,
                                      // the last one fails (test hook)
  std::atomic<int> refs{1};
  // autotuned launch shapes keyed by (ligand-size bucket, protein tiles)
  std::mutex tile_mu;
  std::map<std::pair<int, int>, gd::Tile> tiles;
  // side streams: launches of different shapes run side by side on them
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_done;
  cudaEvent_t forked = nullptr;
  // address of the library's fixed pose-scratch array in the CUDA context
  // that was current when this gd_ctx was created (gd_energy_poses_noalloc)
  unsigned char *noalloc_scratch = nullptr;
};

struct gd_dcomplex {
  gd_ctx *ctx = nullptr;
  gd::KTables T{};
  std::vector<void *> allocs;
  size_t bytes = 0;
  std::atomic<int> refs{1};
  gd_dcomplex *protein_owner = nullptr;  // when the protein arrays are shared
  // device position -> caller's point index: points whose type can form an
  // H-bond come first, so a 32-point chunk rarely mixes the two kinds
  std::vector<int> point_order;
};

namespace gd {
void ctx_retain(gd_ctx *c);
void ctx_release(gd_ctx *c);
void dcx_retain(gd_dcomplex *d);
void dcx_release(gd_dcomplex *d);
gd_status ctx_check(gd_ctx *c);
// Status for a nonzero kernel error word (KRun.err).
gd_status kernel_error(int code);
// Loads the module that holds the fixed pose-scratch array of
// gd_energy_poses_noalloc on c's device (current) and stores the array's
// address in c->noalloc_scratch (gd_noalloc.cu).  Called by gd_ctx_create.
gd_status noalloc_attach(gd_ctx *c);
// Test hook of gd_ctx_set_alloc_fail: true (and the hook off again) when
// this device allocation through c is the one set to fail.
inline bool injected_alloc_failure(gd_ctx *c) {
  int n = c->alloc_fail_in.load();
  while (n > 0 && !c->alloc_fail_in.compare_exchange_weak(n, n - 1)) {
  }
  return n == 1;
}
// Ligand-size bucket: sizes are rounded up to a multiple of 8 atoms; launch
// shapes are chosen (and autotuned) per bucket and cover its largest size.
int lna_bucket(int lna);
Tile tile_for(gd_ctx *ctx, const KTables &T);
// CTAs (a thread-block cluster) that share each 32-replica unit of a complex
// in MC launches: a function of the complex (ligand-size bucket x protein
// points) and of the units of its own run, never of what else runs, so
// results are the same in any mix.  The largest power of two <= cost /
// min_cost and <= SMs / units, at most 8.  Runs (gd_remc, gd_batch) have the
// GPU to themselves and split down to kRunSplitCost pairs per CTA; a server
// request is a run of its own among others and splits only from
// kServeSplitCost, so that splitting under load costs little throughput.
constexpr double kRunSplitCost = 4500.0;
constexpr double kServeSplitCost = 42500.0;
int split_for(gd_ctx *ctx, const KTables &T, int run_units, double min_cost);
// 32-replica units of a complex's replicas (n_prt x n_lig x n_tmp): whole
// exchange groups per unit when n_tmp divides 32.
int units_of(int n_prt, int n_lig, int n_tmp);

// Launches of different shapes (one per launch plan) are independent; each
// kernel holds one CTA per SM, so a plan with fewer CTAs than SMs leaves the
// rest idle unless the next plan runs beside it.  fork_streams returns n
// streams (n <= kMaxSide; the first is ctx->stream) that start after the work
// already queued on ctx->stream; join_streams makes ctx->stream wait for all
// of them.  Both work inside a stream capture, which turns the plans into
// parallel graph branches.  Plans beyond kMaxSide share streams (and run
// after the plan they share one with), so it covers every launch-shape class
// a batch can have in practice.
constexpr int kMaxSide = 32;
gd_status fork_streams(gd_ctx *c, int n, cudaStream_t *out);
gd_status join_streams(gd_ctx *c, int n);
}  // namespace gd
