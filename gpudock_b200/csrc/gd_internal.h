// gd_internal.h -- device data layout and kernel launch descriptors shared by
// the host API (gd_api.cu, gd_batch.cu) and the kernels (gd_kernels.cu).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/gpudock.h"

namespace gd {

// Protein points are staged through shared memory in tiles of TILE_PTS
// points: a 16-byte record {x, y, z, ele} and an 8-byte record {hpp, meta}.
constexpr int TILE_PTS = 128;
constexpr int STREAM_STAGES = 8;       // ring depth when the protein streams
constexpr int MAX_RESIDENT_TILES = 56; // 7168 points kept in smem for a launch
#ifndef GD_MAX_WARPS
#define GD_MAX_WARPS 12
#endif
constexpr int MAX_WARPS = GD_MAX_WARPS; // warps per CTA (all compute)
constexpr int MAX_NA = 10;             // ligand atoms per warp (template bound)
constexpr int MAX_LNA = 128;           // ligand atoms per complex
constexpr int NRED = 10;               // partial sums per replica per warp
constexpr int MAX_TMP = 64;            // temperatures per exchange group
constexpr int TAB_ROWS = GD_NLT + 1;   // + one all-zero row for padding atoms

// meta word of a protein point: type | class << 5 | hpc flag << 8 |
// seq3r << 12 (seq3r < 2^20)
constexpr uint32_t META_TYPE_MASK = 31u;
constexpr uint32_t META_CLASS_SHIFT = 5u;
constexpr uint32_t META_HPC_BIT = 1u << 8;
constexpr uint32_t META_SEQ_SHIFT = 12u;
constexpr int MAX_SEQ3R = (1 << 20) - 1;
// Points past the protein's last point (up to the tile boundary) are padding:
// type PAD_POINT_TYPE, whose kernel table rows are all zero, no charge, and
// far from everything (on the opposite side from the padding ligand atoms,
// with d^9 to any atom still finite in FP32), so the pair loop may run over
// them and add exactly zero.
constexpr int PAD_POINT_TYPE = 31;
constexpr float PAD_POINT_COORD = -3.0e3f;

enum KMode : int { KMODE_POSES = 0, KMODE_REMC = 1, KMODE_INIT = 2 };

// Tables of one complex (device pointers + scalars).
struct KTables {
  const float4 *pt_a;   // [n_prt][pnp_pad] {x, y, z, ele}
  const float2 *pt_b;   // [pnp_pad] {hpp, meta bits}
  const float4 *tab_a;  // [TAB_ROWS*NPT] {p1a, p2a, pmf0, pmf1}
  const float2 *tab_b;  // [TAB_ROWS*NPT] {hdb0, hdb1}
  const float4 *lig;    // [n_lig][lna] {x, y, z, 0} relative to the centre
  const int *lig_order; // [lna] atom of each kernel slot: atoms with an H-bond
                        // term first, so they share atom pairs and warps
  const int *lig_t;     // [lna]
  const float *lig_q;   // [lna]
  const float *psp;     // [NLT][psp_ncol]
  const uint32_t *psp_mask;  // [(psp_ncol + 31) / 32] bit r: some atom type of
                             // this ligand has a nonzero psp[type][r]
  const float4 *kde;    // [pnk] sorted by type {x, y, z, 0}
  const int *kde_off;   // [NLT + 1]
  const float4 *mcs;    // [pos][lna] {x, y, z, valid}
  const float *mcs_tcc; // [pos]
  const float *mcs_cnt; // [pos] number of valid atoms (float)
  const uint32_t *mcc_ref;  // [lna][mcc_words] reference contact map (bits)
  int lna, n_lig, pnp, pnp_pad, n_prt, pos, psp_ncol, mcc_words;
  int n_hb;             // atoms with an H-bond term (the first n_hb slots)
  int pad1;
  float mcc_nref;      // contacts in the reference map
  float near_mcc2;      // squared distance within which a contact can occur
                        // (max pmf0^2, with margin)
  float near_ele2;      // squared distance of the near-field electrostatics
                        // switch (1/el1)^2, with margin
  float lj0, lj0lj1, el0, el1, inv_el1, a1, b1, kde2, kde3;
  float s2pi;           // sqrtf(2 * 3.1415926535f), the reference's float
  float near4[4];       // squared distance below which a close-range term can
                        // fire, by point kind (hpc flag | class 2 << 1)
  float hpl0[GD_NLT], hpl1[GD_NLT], hpl2[GD_NLT];
  float a_para[GD_NTERM], b_para[GD_NTERM], w[GD_NTERM];
  float lig_center[3], pocket[3];
};

// One complex of a launch with its Monte Carlo parameters and the location
// of its replicas in the launch-wide state arrays.
struct KItem {
  KTables T;
  int rep_base;          // first replica of this item in the state arrays
  int n_rep, n_tmp, n_lig_conf, n_prt;
  int steps_per_dump;    // exchange parity restarts every dump (<= 0: never)
  int rec_steps;
  int step0;             // first MC step of the launch when KRun.item_step
  int n_run;             // MC steps of the launch when KRun.item_step
  int spe;               // steps per exchange (exchange kernel, per-item mode)
  int rec_ring;          // record is a ring of rec_steps steps (slot step %
  int pad2;              // rec_steps), else steps 0 .. rec_steps-1
  float move_scale[6];
  uint64_t seed;
  uint32_t stream_id, flags;
  const float *minus_beta;  // [n_tmp]
  int *acs_exchg;           // [n_tmp] by slot
  gd_record *record;        // [n_rep][rec_steps] or nullptr (see rec_ring)
  // replica state of this item, indexed by its local replica number
  float *m_old;             // [n_rep][6]
  float *e_old;             // [n_rep][GD_NTERM]
  float *cmcc;              // [n_rep] contact MCC of the state (GD_MC_MCC)
  int *idx_tmp;             // [n_rep]
  int *acs_mc;              // [n_rep]
};

// Launch descriptor of one dock_kernel launch (by value).
struct KRun {
  int mode;              // KMode
  int A, P;              // warp grid: A atom groups x P protein-tile groups
  int n_stages;          // smem tile stages (== n_tiles when resident)
  int resident;          // 1: whole protein conformation kept in smem
  const KItem *items;
  const int *cta_item;   // [grid] item of each CTA (REMC / INIT)
  const int *cta_rep0;   // [grid] first local replica of each CTA, or with
                         // group_major the first exchange group p*n_lig + l
  const int *cta_nrep;   // [grid] replicas of each CTA (<= 32, one protein conf)
  int group_major;       // lane = (group g0 + lane / n_tmp, temperature slot
                         // lane % n_tmp): whole exchange groups per CTA
  int fused_exchange;    // group_major only: exchange inside the kernel after
                         // every spe MC steps
  int spe;               // MC steps per exchange
  // poses (item 0)
  int prt_conf, lig_conf, n_pose;
  const float *poses;    // [n_pose][6]
  float *terms;          // [n_pose][GD_NTERM]
  double *raw;           // [n_pose][GD_NRAW] or nullptr
  // REMC: the first MC step and the step count are KItem.step0 / n_run with
  // item_step (complexes at different steps in one launch), else the first
  // step is *step_ptr when step_ptr is set (graph replay), else step0
  int step0, n_steps;
  const int *step_ptr;
  int item_step;
  int split;             // REMC / INIT without a schedule: clusters of `split`
                         // CTAs (<= 8) share each unit, CTA rank r taking the
                         // protein tiles r, r + split, ... (grid = units x split);
                         // 0 or 1: one CTA per unit
  int hb_pairs;          // most atom pairs with an H-bond term in any warp of
                         // any item (hb_pairs_of); selects the kernel variant
  // Persistent schedule (REMC; nullptr: CTA b runs every step of unit b,
  // where a unit is one entry of cta_item / cta_rep0 / cta_nrep).  CTA m, in
  // the order the CTAs start, runs pieces piece_off[m] .. piece_off[m+1]-1,
  // each {unit, first step, end step, wait}: MC steps [first, end) of the
  // launch for that unit, after waiting (wait != 0) until progress[unit]
  // reaches the launch's first step + first.
  // With n_queue > 0 a CTA that has run its own pieces takes pieces
  // queue_first, queue_first + 1, ... (one at a time, in order) from a shared
  // counter (queue_ctl[0]), once every CTA of the launch has started
  // (queue_ctl[2] counts them); the last CTA to leave (counted in
  // queue_ctl[1]) sets all three back to 0 for the next launch.
  const int4 *pieces;
  const int *piece_off;  // [grid + 1]
  int n_queue, queue_first;
  int *queue_ctl;
  int *ticket;           // start-order counter, 0 before the launch (wraps)
  int *progress;         // [units] MC steps done (absolute step count)
  int *err;              // error word: 2 bounded wait ran out, 3 hb_pairs too
                         // low, 4 a piece's predecessor never finished
  unsigned long long *busy_ns;  // nullptr, or: each CTA adds the nanoseconds
                                // from its start to its end (SM occupancy)
  uint32_t wait_limit;   // polls of a piece's dependency wait (0: 2^24, ~4 s)
  int wait_bias;         // added to the wait's target: 0, or (test hook) a step
                         // the predecessor never reaches, so the wait runs out
};

// McNaughton's wrap-around rule, for MC steps that must run in order: units
// of `cost[u]` per step and `steps[u]` steps each are laid end to end and cut
// into `m` machines of equal length C = max(max_u cost[u] steps[u],
// sum / m), each cut at a step boundary.  A unit cut at a machine boundary
// runs its first steps at the start of the lower machine and the rest at the
// end of the next one (after a wait that therefore rarely blocks), so each
// machine waits only on the one before it.  Returns the pieces grouped by
// machine (piece_off[m] .. piece_off[m+1]-1, in run order) and the number of
// machines that got work.
int schedule_pieces(const std::vector<double> &cost, const std::vector<int> &steps, int m,
                    std::vector<int4> *pieces, std::vector<int> *piece_off);
// The same for each unit's first steps[u] - tail steps, plus a shared queue:
// the last `tail` steps of every unit as one-step pieces, appended after the
// m machines' pieces (piece_off has m + 1 entries, empty machines included),
// first every unit's first tail step, then its second, ..., units in the
// order their first part is expected to end.  CTAs that have run their own
// pieces take queue pieces in order, so the launch ends within about one
// unit-step of the balanced length whatever the machines' actual speeds.
// Returns m, the queue length in *n_queue.
int schedule_queue(const std::vector<double> &cost, const std::vector<int> &steps, int m, int tail,
                   std::vector<int4> *pieces, std::vector<int> *piece_off, int *n_queue);

// Atom pairs of warp 0 (the most) holding a slot below n_hb: a warp's pair h
// holds slots ag + 2hA and ag + (2h+1)A.
inline int hb_pairs_of(const KTables &T, int A) {
  const int k = (T.n_hb + A - 1) / A;
  return (k + 1) / 2;
}

// Exchange groups: one (item, protein conf, ligand conf) each.
struct KGroup {
  int item, p, l, pad;
};

size_t dock_smem_bytes(int A, int P, int NA, int n_stages, int split = 1);

// Kernel launchers (gd_kernels.cu); return the launch status.
cudaError_t launch_dock(const KRun &R, int NA, int grid, cudaStream_t s);
// CTAs of the launch's kernel variant resident per SM (occupancy).
cudaError_t dock_ctas_per_sm(const KRun &R, int NA, int *n);
cudaError_t launch_exchange(const KItem *items, const KGroup *groups, int n_groups, int spe,
                            int step0, const int *step_ptr, cudaStream_t s);
cudaError_t launch_advance(int *step_ptr, int spe, cudaStream_t s);
cudaError_t launch_metropolis(int n, const float *e_new, const float *e_old,
                              const float *mbeta, const int *rep, const int *step,
                              uint64_t seed, uint32_t stream_id, int *acc, cudaStream_t s);
cudaError_t launch_philox(int n, const uint32_t *ctr, const uint32_t *key, uint32_t *out,
                          cudaStream_t s);
cudaError_t launch_expf(int n, const float *x, float *y, cudaStream_t s);
cudaError_t launch_fma_peak(float *out, int n_blocks, int iters, cudaStream_t s);

}  // namespace gd
