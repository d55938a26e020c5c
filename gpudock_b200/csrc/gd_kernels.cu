// gd_kernels.cu -- sm_100a kernels of the REMC docking path.
//
// dock_kernel: one CTA owns up to 32 replicas (or poses) of one complex that
// share one protein conformation; lane i of every compute warp is replica i,
// so protein-point and type-table reads are warp-uniform shared-memory
// broadcasts.  The compute warps form an A x P grid: warp (ag, pg) (warp
// number pg + P ag) keeps NA ligand atoms a = ag + A k in registers and
// sweeps the protein tiles t = pg, pg + P, ...  The protein conformation is staged in shared memory in
// 128-point tiles by the TMA engine (cp.async.bulk + mbarrier), once per
// launch when it fits (resident) or through an 8-stage ring that the last
// warp to finish a stage refills (then P = 1).  Per step every warp writes
// FP64 partial sums
// per replica; warp 0 reduces them in a fixed order, normalises the terms
// and takes the Metropolis decision with the counter-based RNG.
//
// Per ligand-protein pair the fast path evaluates the terms every pair
// contributes to (soft LJ, far-field electrostatics, contact PMF) with one
// rsqrt, two reciprocals and one exp2.  The terms that only fire close in
// (hydrophobic contact d <= 9 A, near-field electrostatics d < 1/el1,
// pocket-specific potential d <= pmf0) run only when some lane has an atom
// within near_d2 of the point; the H-bond term runs for the type pairs that
// define one.
//
// Reference semantics (gpudocksm-rem-1.2/src):
//   pair terms          calcenergy_d.cu:56-138
//   hydrophobic         calcenergy_d.cu:142-149
//   KDE                 calcenergy_d.cu:175-213
//   LHM restraint       calcenergy_d.cu:229-271
//   finalisation        calcenergy_d.cu:276-371
//   move / move-away    move_d.cu:11-133
//   accept              accept_d.cu:12-52
//   MC step loop        montecarlo_d.cu:12-104
//   exchange            exchangereplicas_d.cu:26-79
#include <cstdint>
#include <cuda_runtime.h>

#include "gd_device.cuh"
#include "gd_internal.h"

namespace gd {

constexpr int STAGE_BYTES = TILE_PTS * (16 + 8);
constexpr int CHUNK = 32;  // points per FP32 partial before the FP64 flush
constexpr int kPointUnroll = 2;  // protein points per iteration of the fast path
constexpr float LOG2E = 1.4426950408889634f;
// coordinate of the padding atoms: far from every point, and close enough
// that d^9 to any point stays finite in FP32
constexpr float FAR = 1.0e3f;
// Point types of the kernel's pair tables: the force field's GD_NPT plus
// all-zero rows, one of which (PAD_POINT_TYPE) marks the padding points that
// fill a tile past the protein's last point, so they add exactly zero.
constexpr int PT_ROWS = 32;
static_assert(PAD_POINT_TYPE >= GD_NPT && PAD_POINT_TYPE < PT_ROWS, "padding type row");

// Per-replica state in shared memory, written by warp 0 only.
struct LaneState {
  float m_old[6];
  float m_new[6];
  float rot[9];
  float e_old[GD_NTERM];
  float mbeta;       // -1/T of the replica's current temperature
  int idx_tmp;       // its temperature index
  int acs;           // accepted moves in this launch
  uint32_t u_bits;   // random word of this step's Metropolis test
  float cmcc_old;    // contact MCC of the accepted state (GD_MC_MCC)
  float cmcc_new;    // and of the proposal
  float pad;
};
static_assert(sizeof(LaneState) == 152, "LaneState layout");
static_assert(sizeof(KItem) % 8 == 0, "KItem must keep the barriers 8-byte aligned");

// Shared-memory carve-up of one CTA.  The pair tables hold, for every
// (atom group, atom pair h, point type), the parameters of the warp's two
// atoms of pair h side by side, so one 16-byte load yields the operand pairs
// of the packed (f32x2) arithmetic:
//   ptab[.][0] = {p1a a, p1a b, -p2a a, -p2a b}
//   ptab[.][1] = {-pmf0 a, -pmf0 b, pmf1 a, pmf1 b}
//   htab[.]    = {-hdb0 a, -hdb0 b, w a, w b}  (w = hdb1 where the H-bond
//                                               term is defined, else 0)
// hmask[ag][pt] has bit h set when pair h of group ag has an H-bond term with
// point type pt.  Slot s = ag + A k holds ligand atom order[s].
struct SmemLayout {
  size_t ptab, htab, hmask, slot_q, slot_t, slot_a, tiles, red, hpc, lane, item, bars, ctl,
      xch, xch_step, total;
};

// Piece bookkeeping of a CTA, in shared memory so that none of it holds a
// register across the pair loop.  A piece is a range of MC steps of one
// unit (a CTA's worth of replicas); without a schedule a CTA runs one piece,
// all steps of unit blockIdx.x.
struct PieceCtl {
  int pc, pc_end;   // next piece, end of this CTA's pieces
  int item;         // item whose tables are in shared memory (-1: none)
  int tiles_key;    // item * MAX_PRT_KEY + protein conformation of the
                    // resident tiles (-1: none)
  int gen;          // resident tile loads so far (mbarrier phase parity)
  int it;           // streaming ring position (continues across pieces)
  int first_it;     // ring position of the current piece's first tile
  int sig_unit;     // unit of the current piece, and the step count its
  int sig_step;     // progress word holds once the piece has ended
  int pad;
};
constexpr int MAX_PRT_KEY = 1 << 16;
static_assert(sizeof(PieceCtl) <= 64, "PieceCtl fits its slot");

// split > 1: the launch runs as clusters of `split` CTAs that share a unit;
// each CTA then also holds two (step parity) exchange buffers of its
// per-replica partial sums: NRED FP64 terms and one FP32 hydrophobic sum per
// atom slot, 32 lanes each.
__host__ __device__ inline SmemLayout smem_layout(int A, int P, int NA, int NS, int split = 1) {
  SmemLayout L;
  const size_t NH = NA / 2, MAXA = (size_t)A * NA, W = (size_t)A * P;
  size_t o = 0;
  L.ctl = o;  // first, at a fixed address
  o += 64;
  L.ptab = o;
  o += (size_t)A * NH * PT_ROWS * 32;
  L.htab = o;
  o += (size_t)A * NH * PT_ROWS * 16;
  L.hmask = o;
  o += (size_t)A * PT_ROWS * 4;
  L.slot_q = o;
  o += MAXA * 4;
  L.slot_t = o;
  o += MAXA * 4;
  L.slot_a = o;
  o += MAXA * 4;
  o = (o + 127) & ~size_t(127);
  L.tiles = o;
  o += (size_t)NS * STAGE_BYTES;
  L.red = o;
  o += W * NRED * 32 * sizeof(double);
  L.hpc = o;
  o += (size_t)P * MAXA * 32 * sizeof(float);
  L.lane = o;
  o += 32 * sizeof(LaneState);
  o = (o + 15) & ~size_t(15);
  L.item = o;
  o += sizeof(KItem);
  o = (o + 7) & ~size_t(7);
  L.bars = o;
  o += 2 * (size_t)NS * sizeof(uint64_t);
  o = (o + 15) & ~size_t(15);
  L.xch = o;
  L.xch_step = (size_t)NRED * 32 * sizeof(double) + MAXA * 32 * sizeof(float);
  if (split > 1) o += 2 * L.xch_step;
  L.total = o;
  return L;
}

size_t dock_smem_bytes(int A, int P, int NA, int n_stages, int split) {
  return smem_layout(A, P, NA, n_stages, split).total;
}

// Hardware approximations (PTX rsqrt / rcp / ex2, flush-to-zero).
__device__ __forceinline__ float frsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float frcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float fex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Packed FP32 pairs (Blackwell f32x2 FMA-pipe instructions).
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// ZYX Euler rotation of move_d.cu:90-105 (row-major 3x3).
__device__ __forceinline__ void make_rot(float a3, float a4, float a5, float *R) {
  float s1, c1, s2, c2, s3, c3;
  sincosf(a3, &s1, &c1);
  sincosf(a4, &s2, &c2);
  sincosf(a5, &s3, &c3);
  R[0] = c1 * c2;
  R[1] = c1 * s2 * s3 - c3 * s1;
  R[2] = s1 * s3 + c1 * c3 * s2;
  R[3] = c2 * s1;
  R[4] = c1 * c3 + s1 * s2 * s3;
  R[5] = c3 * s1 * s2 - c1 * s3;
  R[6] = -1.0f * s2;
  R[7] = c2 * s3;
  R[8] = c2 * c3;
}

// Per-atom hydrophobic sums in shared memory: for tile group g, the float2
// of atom pair h (slots ag + 2hA, ag + (2h+1)A) of atom group ag and lane
// `lane` sits at float2 index ((g A + ag) NH + h) 32 + lane (a warp reads
// a pair's sums as one conflict-free 64-bit access).
__device__ __forceinline__ int hpc_pair_at(int g, int ag, int h, int lane, int A, int NH) {
  return ((g * A + ag) * NH + h) * 32 + lane;
}

// Hydrophobic restraint (calcenergy_d.cu:143-149) of atom pair hp of atom
// group ag: the P tile groups' sums of the pair's two slots added in group
// order, then 0.5 hh^2 - hpl2 with hh = (sum - hpl0) / hpl1 for each slot
// that holds an atom (0 for a slot past the ligand).
__device__ __forceinline__ float2 hpc_transform(const KTables &T, const int *s_lt, int A, int ag,
                                                int hp, float2 v) {
  float r[2] = {0.f, 0.f};
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int a = ag + A * (2 * hp + j);
    if (a < T.lna) {
      const int lt = s_lt[a];
      const float hh = __fdiv_rn(__fsub_rn(j ? v.y : v.x, T.hpl0[lt]), T.hpl1[lt]);
      r[j] = __fsub_rn(__fmul_rn(__fmul_rn(0.5f, hh), hh), T.hpl2[lt]);
    }
  }
  return make_float2(r[0], r[1]);
}
__device__ __forceinline__ float2 hpc_restraint(const KTables &T, const float2 *s_hpc2,
                                                const int *s_lt, int P, int A, int NH, int ag,
                                                int hp, int lane) {
  float2 v = make_float2(0.f, 0.f);
  for (int g = 0; g < P; ++g) {
    const float2 x = s_hpc2[hpc_pair_at(g, ag, hp, lane, A, NH)];
    v.x += x.x;
    v.y += x.y;
  }
  return hpc_transform(T, s_lt, A, ag, hp, v);
}

// Warp 0 after the step's partial sums: cross-warp reduction in a fixed
// order, hydrophobic restraint per atom (hpc_done: already transformed by the
// warps into tile group 0's slots), normalisation and total in the
// reference's order, then the pose output, or the Metropolis decision (with
// the trajectory record) and, at the end of an interval, the in-CTA
// temperature exchange.  Kept out of line so its registers do not burden the
// pair loop.
template <int MODE>
__device__ __noinline__ void finish_step(const KRun &R, const KItem &I, LaneState &me,
                                         double *s_red, const float *s_hpc, const int *s_lt,
                                         int W, int P, int A, int NH, int lane, int rep,
                                         bool active, int prt_conf, int lig_conf, int step,
                                         bool primary, bool hpc_done) {
  const KTables &T = I.T;
  const int lna = T.lna;
  const float lcx = T.lig_center[0], lcy = T.lig_center[1], lcz = T.lig_center[2];
    double S[NRED];
#pragma unroll
    for (int i = 0; i < NRED; ++i) S[i] = 0.0;
    for (int w = 0; w < W; ++w) {
      const double *red = s_red + (size_t)w * NRED * 32;
#pragma unroll
      for (int i = 0; i < NRED; ++i) S[i] += red[i * 32 + lane];
    }
    // hydrophobic restraint per ligand atom, by slot (slot a = ag + A k holds
    // one atom, s_lt its type), an atom pair's two slots at a time, in slot
    // order
    const float2 *s_hpc2 = reinterpret_cast<const float2 *>(s_hpc);
    for (int ag = 0; ag < A; ++ag)
      for (int hp = 0; hp < NH; ++hp) {
        if (ag + 2 * hp * A >= lna) break;
        const float2 r = hpc_done ? s_hpc2[hpc_pair_at(0, ag, hp, lane, A, NH)]
                                  : hpc_restraint(T, s_hpc2, s_lt, P, A, NH, ag, hp, lane);
        S[5] += (double)r.x;
        if (ag + A * (2 * hp + 1) < lna) S[5] += (double)r.y;
      }
    const double n = (double)lna;
    double raw[GD_NRAW];
    raw[0] = S[0] / n;
    raw[1] = S[1] / n;
    raw[2] = S[2] / n;
    raw[3] = S[3] / n;
    raw[4] = -(S[4] / n / (double)T.s2pi);
    raw[5] = S[5] / n;
    raw[6] = S[6] / (double)T.kde3 / n;
    raw[7] = log(S[7] / (double)T.pos);
    {
      // distance to the pocket (calcenergy_d.cu:278-283); centre = c + m
      const float cx = __fadd_rn(lcx, me.m_new[0]);
      const float cy = __fadd_rn(lcy, me.m_new[1]);
      const float cz = __fadd_rn(lcz, me.m_new[2]);
      const float dx = __fsub_rn(cx, T.pocket[0]);
      const float dy = __fsub_rn(cy, T.pocket[1]);
      const float dz = __fsub_rn(cz, T.pocket[2]);
      raw[8] = (double)__fsqrt_rn(
          __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
    }
    float e[GD_NTERM];
#pragma unroll
    for (int i = 0; i < 9; ++i)
      e[i] = __fadd_rn(__fmul_rn(T.a_para[i], (float)raw[i]), T.b_para[i]);
    float tot = __fmul_rn(T.w[0], e[0]);
#pragma unroll
    for (int i = 1; i < 9; ++i) tot = __fadd_rn(tot, __fmul_rn(T.w[i], e[i]));
    if (MODE != KMODE_POSES && (I.flags & GD_MC_BAYES)) tot = bayes_total(e);
    e[9] = tot;
    if (MODE != KMODE_POSES && (I.flags & GD_MC_MCC)) {
      // confusion counts against the reference map (calcmcc_d.cu:189-206);
      // the counts are exact integers in FP32 below 2^24 pairs
      const float tp = (float)S[9];
      const float fp = __fsub_rn((float)S[8], tp);
      const float fn = __fsub_rn(T.mcc_nref, tp);
      const float n = __fmul_rn((float)T.lna, (float)T.pnp);
      const float tn = __fsub_rn(__fsub_rn(__fsub_rn(n, tp), fn), fp);
      const float dividend = __fsqrt_rn(
          __fmul_rn(__fmul_rn(__fmul_rn(__fadd_rn(tp, fp), __fadd_rn(tp, fn)), __fadd_rn(tn, fp)),
                    __fadd_rn(tn, fn)));
      me.cmcc_new = dividend != 0.0f
                        ? __fdiv_rn(__fsub_rn(__fmul_rn(tp, tn), __fmul_rn(fp, fn)), dividend)
                        : GD_CMCC_INVALID;
    }

    if (MODE == KMODE_POSES) {
      if (active) {
#pragma unroll
        for (int i = 0; i < GD_NTERM; ++i) R.terms[(size_t)rep * GD_NTERM + i] = e[i];
        if (R.raw) {
#pragma unroll
          for (int i = 0; i < GD_NRAW; ++i) R.raw[(size_t)rep * GD_NRAW + i] = raw[i];
        }
      }
    } else {
      int acc;
      if (MODE == KMODE_INIT) {
        acc = 1;  // forced accept with beta = 0 (montecarlo_d.cu:236-239)
      } else {
        acc = metropolis(e[9], me.e_old[9], me.mbeta, u01(me.u_bits));
        if (primary && active && I.record && (I.rec_ring || step < I.rec_steps)) {
          const int slot = I.rec_ring ? step % I.rec_steps : step;
          gd_record *rc = I.record + (size_t)rep * I.rec_steps + slot;
          rc->idx_rep = rep;
          rc->idx_prt = prt_conf;
          rc->idx_tmp = me.idx_tmp;
          rc->idx_lig = lig_conf;
#pragma unroll
          for (int i = 0; i < GD_NTERM; ++i) rc->e[i] = me.e_old[i];
          rc->cmcc = (I.flags & GD_MC_MCC) ? me.cmcc_old : 0.f;
#pragma unroll
          for (int i = 0; i < 6; ++i) rc->movematrix[i] = me.m_old[i];
          rc->step = step;
          rc->e_prop_total = e[9];
          rc->accepted = acc;
        }
      }
      if (acc) {
        me.acs += 1;
#pragma unroll
        for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = e[i];
#pragma unroll
        for (int i = 0; i < 6; ++i) me.m_old[i] = me.m_new[i];
        me.cmcc_old = me.cmcc_new;
      }
      // temperature exchange of the CTA's own groups at the end of every
      // interval (exchangereplicas_d.cu:26-79); slot t of group gi is lane
      // gi * n_tmp + t, so the groups never leave the CTA
      if (MODE == KMODE_REMC && R.fused_exchange && ((step + 1) % R.spe) == 0 &&
          (I.flags & GD_MC_EXCHANGE)) {
        const int nt = I.n_tmp;
        int *s_tmp = reinterpret_cast<int *>(s_red);          // 32 ints
        float *s_en = reinterpret_cast<float *>(s_red) + 32;  // 32 floats
        s_tmp[lane] = me.idx_tmp;
        s_en[lane] = me.e_old[GD_E_TOTAL];
        __syncwarp();
        const int s0 = step + 1 - R.spe;
        const int within = I.steps_per_dump > 0 ? (s0 % I.steps_per_dump) : s0;
        const int mode_t = (within / R.spe) % 2;
        if (active && (lane % nt) == 0) {
          const int b = lane;  // first slot of this group
          const uint32_t gid = (uint32_t)(prt_conf * I.n_lig_conf + (rep % I.n_lig_conf));
          uint32_t k0, k1;
          rng_key(I.seed, I.stream_id, k0, k1);
          int orders[MAX_TMP];
          for (int t = 0; t < nt; ++t) orders[s_tmp[b + t]] = t;
          const int maxpair = nt / 2 - (nt % 2 == 0) * (mode_t == 1);
          for (int pair = 0; pair < maxpair; ++pair) {
            const int i1 = (pair << 1) + mode_t;
            const int o1 = orders[i1], o2 = orders[i1 + 1];
            const int tt = s_tmp[b + o1];
            const float mb1 = I.minus_beta[s_tmp[b + o1]];
            const float mb2 = I.minus_beta[s_tmp[b + o2]];
            const float delta =
                __fmul_rn(__fsub_rn(mb1, mb2), __fsub_rn(s_en[b + o2], s_en[b + o1]));
            const float prob = decision_expf(delta);
            const U4 o =
                philox4x32_10(U4{gid, (uint32_t)(s0 / R.spe), 2u, (uint32_t)pair}, k0, k1);
            if (prob > u01(o.x)) {
              s_tmp[b + o1] = s_tmp[b + o2];
              s_tmp[b + o2] = tt;
              if (primary) {  // once per cluster
                atomicAdd(&I.acs_exchg[o1], 1);
                atomicAdd(&I.acs_exchg[o2], 1);
              }
            }
          }
        }
        __syncwarp();
        me.idx_tmp = s_tmp[lane];
        me.mbeta = I.minus_beta[me.idx_tmp];
      }
    }
  }

struct PairConst {
  float2 one, lj1, lj0, ca, cb;
};

// One protein point (A0) against this lane's NA atoms, two atoms per packed
// instruction (atom pair h): soft LJ, far-field electrostatics (per-atom
// sums of ele/d), contact PMF and, for the first NHB atom pairs, the H-bond
// term (H-bond-capable atoms come first in the slot order, so the later
// pairs of a warp have none; weight 0 and hdb0 = 0 for an atom of a pair
// without it).  pp / hp point at the point type's entry of atom pair 0 of
// this warp's pair tables.
//
// The soft LJ of calcenergy_d.cu:96-100, (p1 - p2) / p4 with p1 = p1a / d^9,
// p2 = p2a / d^6, p4 = 1 + p1 L and L = lj0 (1 + lj1 d^2), is evaluated
// multiplied through by d^9: (p1a - p2a d^3) / (d^9 + p1a L).  That takes
// two multiplies fewer than the powers of 1/d, and its denominator D1 stays
// between p1a L and d^9, so it cannot overflow at short range.  The LJ and
// PMF quotients share one reciprocal: with D2 = 1 + exp(.),
// num1/D1 = num1 D2 / (D1 D2) and pmf1/D2 = pmf1 D1 / (D1 D2).
// Branch-free and written in stages over all atom pairs -- distances and
// rsqrt, then powers, PMF argument and exp, then the shared reciprocals and
// sums, then the H-bond Gaussians -- so that the MUFU operations of one
// stage overlap the FMA work of the others; each accumulator still adds its
// atom pairs in order h = 0, 1, ...
template <int NH, int NHB>
__device__ __forceinline__ void pair_block1(const float2 (&nx)[NH], const float2 (&ny)[NH],
                                            const float2 (&nz)[NH], const float4 &A0,
                                            const float4 *pp, const float4 *hp,
                                            const PairConst &K, float2 &fvdw, float2 &fpmf,
                                            float2 &fhdb, float2 (&fek)[NH], float &mn) {
  float2 d2[NH], r[NH];
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    const float2 dx = add2(dup2(A0.x), nx[h]);
    const float2 dy = add2(dup2(A0.y), ny[h]);
    const float2 dz = add2(dup2(A0.z), nz[h]);
    d2[h] = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    r[h] = make_float2(frsqrt(d2[h].x), frsqrt(d2[h].y));
  }
  float2 ex[NH], den1[NH], num1[NH], pm[NH];
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    const float4 T0 = pp[h * 2 * PT_ROWS];      // p1a, -p2a
    const float4 T1 = pp[h * 2 * PT_ROWS + 1];  // -pmf0, pmf1
    const float2 d = mul2(d2[h], r[h]);
    const float2 g = mul2(d2[h], d);            // d^3
    const float2 g3 = mul2(mul2(g, g), g);      // d^9
    den1[h] = fma2(lo2(T0), fma2(K.lj1, d2[h], K.lj0), g3);  // d^9 + p1a L
    num1[h] = fma2(hi2(T0), g, lo2(T0));                      // p1a - p2a d^3
    pm[h] = mul2(hi2(T1), den1[h]);
    const float2 arg = mul2(fma2(K.ca, d, K.cb), add2(d, lo2(T1)));
    ex[h] = make_float2(fex2(arg.x), fex2(arg.y));
  }
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    // D1 D2 and num1 D2 as single FMAs: D1 (1 + ex) = D1 ex + D1
    const float2 den = fma2(den1[h], ex[h], den1[h]);
    const float2 inv = make_float2(frcp(den.x), frcp(den.y));
    fvdw = fma2(fma2(num1[h], ex[h], num1[h]), inv, fvdw);
    fpmf = fma2(pm[h], inv, fpmf);
    fek[h] = fma2(dup2(A0.w), r[h], fek[h]);
    mn = fminf(mn, fminf(d2[h].x, d2[h].y));
  }
#pragma unroll
  for (int h = 0; h < (NHB < NH ? NHB : NH); ++h) {
    const float2 d = mul2(d2[h], r[h]);
    const float4 H = hp[h * PT_ROWS];  // -hdb0, w
    const float2 h3 = mul2(add2(d, lo2(H)), hi2(H));
    const float2 ha = mul2(mul2(h3, h3), K.ca);  // -0.5 log2(e) h3^2
    fhdb = fma2(hi2(H), make_float2(fex2(ha.x), fex2(ha.y)), fhdb);
  }
}

template <int NH, int NHB>
__device__ __forceinline__ uint32_t chunk_fast(const float2 (&nx)[NH], const float2 (&ny)[NH],
                                               const float2 (&nz)[NH], const float4 *ta,
                                               const float2 *tb, int j0, int j1,
                                               const float4 *my_ptab, const float4 *my_htab,
                                               const PairConst &K, float thr_l, float2 &fvdw,
                                               float2 &fpmf, float2 &fhdb, float2 (&fek)[NH]) {
  uint32_t close = 0u;
  // the next point's record is read one iteration ahead
  float4 Ap = ta[j0];
  int pt = (int)(__float_as_uint(tb[j0].y) & META_TYPE_MASK);
#pragma unroll kPointUnroll
  for (int j = j0; j < j1; ++j) {
    const int jn = min(j + 1, j1 - 1);
    const float4 An = ta[jn];
    const int ptn = (int)(__float_as_uint(tb[jn].y) & META_TYPE_MASK);
    float mn = 3.0e38f;
    pair_block1<NH, NHB>(nx, ny, nz, Ap, my_ptab + pt * 2, my_htab + pt, K, fvdw, fpmf, fhdb,
                         fek, mn);
    const float thr = __shfl_sync(0xffffffffu, thr_l, j - j0);
    close |= (__any_sync(0xffffffffu, mn <= thr) ? 1u : 0u) << (j - j0);
    Ap = An;
    pt = ptn;
  }
  return close;
}

// Close-range terms of one protein point (calcenergy_d.cu:80-138): the
// hydrophobic contact per atom (points with the hpc flag, d <= 9 A), the
// near-field electrostatics (el1 d < 1) and the pocket-specific potential
// (class-2 points, d <= pmf0); with the MCC score on, the contacts d <= pmf0
// of every point, counted (with those also in the reference map,
// calcmcc_d.cu:148-213) straight into the lane's FP64 slots 8 and 9 of
// my_red, so the rare counts hold no registers in the pair loop.  Distances
// are recomputed per atom pair; p is the point's index in the protein.
// The hydrophobic polynomial runs packed over an atom pair, branch-free
// (zero beyond 9 A and for padding slots), into the pair's float2 of
// per-atom sums of the chunk (hacc[h], added to the shared-memory sums once
// per chunk).  The contact test d <= pmf0 (a distance and a table read per
// atom) runs only with the MCC score on or on residues where some atom type
// of this ligand has a nonzero PSP entry (T.psp_mask): elsewhere the PSP
// term adds exactly zero.
template <int NA>
__device__ __forceinline__ void close_range(const float2 (&nx)[NA / 2], const float2 (&ny)[NA / 2],
                                            const float2 (&nz)[NA / 2], const float4 &Ap,
                                            float hpp, uint32_t meta, const float4 *pp,
                                            const KTables &T, const float *s_q, const int *s_lt,
                                            const int *s_atom, float2 (&hacc)[NA / 2], int A, int ag,
                                            int n_my, float inv_el1, float &fnear, float &fpsp,
                                            bool mcc_on, int p, double *my_red) {
  const bool is_c2 = ((meta >> META_CLASS_SHIFT) & 3u) == 2u;
  const bool hflag = (meta & META_HPC_BIT) != 0u;
  const uint32_t res = meta >> META_SEQ_SHIFT;
  // the d <= pmf0 block below: the contact count of the MCC score, or a PSP
  // entry of this residue for some atom type of the ligand
  const bool psp_on = is_c2 && ((__ldg(&T.psp_mask[res >> 5]) >> (res & 31)) & 1u) != 0u;
  const bool thr_pm = is_c2 || mcc_on;  // the threshold stays the point kind's
  // the largest squared distance at which a term below can fire for this
  // point: atom pairs that no lane has within it are skipped (warp-uniform)
  const float thr = fmaxf(T.near_ele2, fmaxf(hflag ? 81.0f : 0.0f, thr_pm ? T.near_mcc2 : 0.0f));
  const float c1 = 3.5f / 81.0f;
  const float c2 = -4.5f / 81.0f / 81.0f;
  const float c3 = 2.5f / 81.0f / 81.0f / 81.0f;
  const float c4 = -0.5f / 81.0f / 81.0f / 81.0f / 81.0f;
#pragma unroll
  for (int h = 0; h < NA / 2; ++h) {
    const float2 dx2 = add2(nx[h], dup2(Ap.x));
    const float2 dy2 = add2(ny[h], dup2(Ap.y));
    const float2 dz2 = add2(nz[h], dup2(Ap.z));
    const float2 d2p = fma2(dx2, dx2, fma2(dy2, dy2, mul2(dz2, dz2)));
    if (!__any_sync(0xffffffffu, fminf(d2p.x, d2p.y) <= thr)) continue;
    if (hflag) {
      // 1 - (c1 d2 + c2 d4 + c3 d6 + c4 d8), Horner in d2
      const float2 q = fma2(fma2(fma2(dup2(c4), d2p, dup2(c3)), d2p, dup2(c2)), d2p, dup2(c1));
      float2 poly = fma2(make_float2(-q.x, -q.y), d2p, dup2(1.0f));
      poly.x = (d2p.x <= 81.0f && 2 * h < n_my) ? poly.x : 0.0f;
      poly.y = (d2p.y <= 81.0f && 2 * h + 1 < n_my) ? poly.y : 0.0f;
      hacc[h] = fma2(dup2(hpp), poly, hacc[h]);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int k = 2 * h + j;
      const float d2 = j ? d2p.y : d2p.x;
      // the distance itself only where a switch can be near (d^2 bounds with
      // margin: the tests below decide on d exactly as before)
      if (d2 <= T.near_ele2) {
        const float rk = frsqrt(d2);
        const float s1 = T.el1 * (d2 * rk);
        if (s1 < 1.0f) {
          const float gnear = fmaf(s1 * s1, fmaf(T.b1, s1, T.a1), T.el0);
          fnear = fmaf(s_q[ag + A * k] * Ap.w, gnear - rk * inv_el1, fnear);
        }
      }
      if ((psp_on || mcc_on) && k < n_my && d2 <= T.near_mcc2) {
        const float d = d2 * frsqrt(d2);
        const float4 T1 = pp[(k >> 1) * 2 * PT_ROWS + 1];
        const float dm = d + ((k & 1) ? T1.y : T1.x);
        if (dm <= 0.0f) {
          if (psp_on) fpsp += __ldg(&T.psp[(size_t)s_lt[ag + A * k] * T.psp_ncol + res]);
          if (mcc_on) {
            const int a = s_atom[ag + A * k];
            my_red[8 * 32] += 1.0;
            if ((__ldg(&T.mcc_ref[(size_t)a * T.mcc_words + (p >> 5)]) >> (p & 31)) & 1u)
              my_red[9 * 32] += 1.0;
          }
        }
      }
    }
  }
}

// HB: atom pairs per warp that evaluate the H-bond term (at least what the
// launch's items need, KRun.hb_pairs).  PIECES: the CTA runs the pieces of a
// persistent schedule (KRun.pieces, REMC only), else all steps of unit
// blockIdx.x.
// No producer warp: sm_100 splits the register file between the four
// schedulers, so a 13th warp would put four warps on one scheduler and cap
// every thread at 128 registers; 12 warps leave room for about 168.
template <int MODE, int NA, int HB, bool PIECES>
__global__ void __launch_bounds__(MAX_WARPS * 32, 1)
    dock_kernel(const __grid_constant__ KRun R) {
  static_assert(NA % 2 == 0, "atoms are processed in pairs");
  constexpr int NH = NA / 2;
  static_assert(HB >= 0 && HB <= NH, "H-bond pair bound");
  extern __shared__ __align__(128) unsigned char smem[];
  const int A = R.A, P = R.P, W = A * P, NS = R.n_stages;
  const int MAXA = A * NA;
  // split launch: clusters of csize CTAs, rank crank, share one unit; CTA
  // crank takes the protein tiles crank, crank + csize, ...
  const int csize = (MODE != KMODE_POSES && !PIECES && R.split > 1) ? R.split : 1;
  const SmemLayout SL = smem_layout(A, P, NA, NS, csize);
  float4 *s_ptab = reinterpret_cast<float4 *>(smem + SL.ptab);
  float4 *s_htab = reinterpret_cast<float4 *>(smem + SL.htab);
  uint32_t *s_hmask = reinterpret_cast<uint32_t *>(smem + SL.hmask);
  float *s_q = reinterpret_cast<float *>(smem + SL.slot_q);
  int *s_lt = reinterpret_cast<int *>(smem + SL.slot_t);
  int *s_atom = reinterpret_cast<int *>(smem + SL.slot_a);
  unsigned char *s_tiles = smem + SL.tiles;
  double *s_red = reinterpret_cast<double *>(smem + SL.red);
  float *s_hpc = reinterpret_cast<float *>(smem + SL.hpc);
  LaneState *s_lane = reinterpret_cast<LaneState *>(smem + SL.lane);
  KItem *s_item = reinterpret_cast<KItem *>(smem + SL.item);
  uint64_t *s_full = reinterpret_cast<uint64_t *>(smem + SL.bars);
  int *s_done = reinterpret_cast<int *>(s_full + NS);  // warps done with a stage
  PieceCtl *s_ctl = reinterpret_cast<PieceCtl *>(smem);  // SmemLayout.ctl == 0

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  // ---- barriers and the pieces of this CTA ----------------------------------
  // With a schedule (PIECES, R.pieces) a CTA's number is a ticket taken when it
  // starts (wrapping back to 0 after the last CTA), so a CTA only ever waits
  // on one that started before it.
  const unsigned long long t_start = R.busy_ns ? global_ns() : 0ull;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&s_full[i], 1);
      s_done[i] = 0;
    }
    fence_barrier_init();
    int pc = 0, pc_end = 1;
    if (PIECES) {
      const int m = (int)atomicInc(reinterpret_cast<unsigned *>(R.ticket), gridDim.x - 1);
      pc = R.piece_off[m];
      pc_end = R.piece_off[m + 1];
      if (R.n_queue > 0) atomicAdd(R.queue_ctl + 2, 1);  // CTAs started
    }
    s_ctl->pc = pc;
    s_ctl->pc_end = pc_end;
    s_ctl->item = -1;
    s_ctl->tiles_key = -1;
    s_ctl->gen = 0;
    s_ctl->it = 0;
  }
  __syncthreads();

  for (;;) {
  if (PIECES && R.n_queue > 0 && s_ctl->pc >= s_ctl->pc_end) {
    // this CTA's own pieces are done: the next piece of the shared queue
    __syncthreads();  // every thread has read s_ctl
    if (threadIdx.x == 0) {
      // queue pieces may wait on any CTA's pieces: take them only once every
      // CTA of the launch has started (else this CTA leaves the queue to the
      // later ones), so that every wait is on a running CTA
      const bool all_started = ld_acquire(R.queue_ctl + 2) >= (int)gridDim.x;
      const int q = all_started ? atomicAdd(R.queue_ctl, 1) : R.n_queue;
      if (q < R.n_queue) {
        s_ctl->pc = R.queue_first + q;
        s_ctl->pc_end = s_ctl->pc + 1;
      } else {
        s_ctl->pc = 1;  // none left: the CTA ends
        s_ctl->pc_end = 0;
        // the last CTA out sets the queue back for the next launch (every
        // CTA's last claim is ordered before its count)
        __threadfence();
        if (atomicAdd(R.queue_ctl + 1, 1) == (int)gridDim.x - 1) {
          R.queue_ctl[0] = 0;
          R.queue_ctl[1] = 0;
          R.queue_ctl[2] = 0;
        }
      }
    }
    __syncthreads();
  }
  const int pc = s_ctl->pc;
  if (pc >= s_ctl->pc_end) break;
  int unit = blockIdx.x / csize, lo = 0, hi = -1;  // hi < 0: every step of the launch
  bool wait_dep = false;
  if (PIECES) {
    const int4 pz = R.pieces[pc];
    unit = pz.x;
    lo = pz.y;
    hi = pz.z;
    wait_dep = pz.w != 0;
  }

  // ---- item of this piece into shared memory, pair tables -----------------
  const int item = (MODE == KMODE_POSES) ? 0 : R.cta_item[unit];
  if (item != s_ctl->item) {
    // one read of the descriptor (it may live in pinned host memory), then
    // the shared-memory copy
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&R.items[item]);
    uint32_t *dst = reinterpret_cast<uint32_t *>(s_item);
    for (int i = threadIdx.x; i < (int)(sizeof(KItem) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    const KTables &TG = s_item->T;
    const int lna = TG.lna;
    // slot s holds atom order[s]; slots past the ligand are padding atoms
    // (all-zero table row, no charge, far from everything)
    for (int s = threadIdx.x; s < MAXA; s += blockDim.x) {
      const int a = s < lna ? TG.lig_order[s] : -1;
      s_atom[s] = a;
      s_lt[s] = a >= 0 ? TG.lig_t[a] : GD_NLT;
      s_q[s] = a >= 0 ? TG.lig_q[a] : 0.f;
    }
    // point types GD_NPT..PT_ROWS-1 (the padding points) get all-zero entries
    for (int i = threadIdx.x; i < A * NH * PT_ROWS; i += blockDim.x) {
      const int pt = i % PT_ROWS, h = (i / PT_ROWS) % NH, ag = i / (PT_ROWS * NH);
      const int s0 = ag + A * (2 * h), s1 = s0 + A;
      const int ptc = pt < GD_NPT ? pt : 0;
      const int r0 = (s0 < lna && pt < GD_NPT ? TG.lig_t[TG.lig_order[s0]] : GD_NLT) * GD_NPT + ptc;
      const int r1 = (s1 < lna && pt < GD_NPT ? TG.lig_t[TG.lig_order[s1]] : GD_NLT) * GD_NPT + ptc;
      const float4 a0 = TG.tab_a[r0], a1 = TG.tab_a[r1];
      s_ptab[2 * i] = make_float4(a0.x, a1.x, -a0.y, -a1.y);
      s_ptab[2 * i + 1] = make_float4(-a0.z, -a1.z, a0.w, a1.w);
      // H-bond term where hdb0 > 0.1 (calcenergy_d.cu:115-126)
      const float2 b0 = TG.tab_b[r0], b1 = TG.tab_b[r1];
      const bool h0 = b0.x > 0.1f, h1 = b1.x > 0.1f;
      s_htab[i] = make_float4(h0 ? -b0.x : 0.f, h1 ? -b1.x : 0.f, h0 ? b0.y : 0.f,
                              h1 ? b1.y : 0.f);
    }
    for (int i = threadIdx.x; i < A * PT_ROWS; i += blockDim.x) {
      const int pt = i % PT_ROWS, ag = i / PT_ROWS;
      uint32_t m = 0;
      for (int h = 0; h < NH && pt < GD_NPT; ++h) {
        const int s0 = ag + A * (2 * h), s1 = s0 + A;
        const int r0 = (s0 < lna ? TG.lig_t[TG.lig_order[s0]] : GD_NLT) * GD_NPT + pt;
        const int r1 = (s1 < lna ? TG.lig_t[TG.lig_order[s1]] : GD_NLT) * GD_NPT + pt;
        if (TG.tab_b[r0].x > 0.1f || TG.tab_b[r1].x > 0.1f) m |= 1u << h;
      }
      s_hmask[i] = m;
    }
    __syncthreads();  // every thread has read s_ctl->item
    if (threadIdx.x == 0) s_ctl->item = item;
  }
  const KItem &I = *s_item;
  const KTables &T = I.T;

  // ---- work of this piece ---------------------------------------------------
  int rep0, n_act, prt_conf, lane_rep;
  if (MODE == KMODE_POSES) {
    rep0 = blockIdx.x * 32;
    n_act = min(32, R.n_pose - rep0);
    prt_conf = R.prt_conf;
    lane_rep = rep0 + (lane < n_act ? lane : 0);
  } else if (R.group_major) {
    // whole exchange groups: lane = group offset * n_tmp + temperature slot
    const int nt = I.n_tmp, nl = I.n_lig_conf;
    const int g0 = R.cta_rep0[unit];
    n_act = R.cta_nrep[unit];
    rep0 = g0;
    prt_conf = g0 / nl;
    const int ln = lane < n_act ? lane : 0;
    lane_rep = nt * nl * prt_conf + nl * (ln % nt) + (g0 % nl) + ln / nt;
  } else {
    rep0 = R.cta_rep0[unit];
    n_act = R.cta_nrep[unit];
    prt_conf = rep0 / (I.n_tmp * I.n_lig_conf);
    lane_rep = rep0 + (lane < n_act ? lane : 0);
  }
  const int n_tiles = (T.pnp + TILE_PTS - 1) / TILE_PTS;
  const int crank0 = csize > 1 ? cluster_rank() : 0;
  const int n_tl = (n_tiles - crank0 + csize - 1) / csize;  // tiles of this CTA
  const bool resident = R.resident != 0;
  const int launch_steps = (MODE != KMODE_REMC) ? 1 : (R.item_step ? I.n_run : R.n_steps);
  const int launch_base = (MODE == KMODE_REMC && R.item_step)  ? I.step0
                          : (MODE == KMODE_REMC && R.step_ptr) ? *R.step_ptr
                                                               : R.step0;
  // this piece: MC steps lo .. hi-1 of the launch
  const int s_hi = hi < 0 ? launch_steps : hi;
  const int n_steps = s_hi - lo;
  const int step_base = launch_base + lo;
  const int passes = resident ? 1 : n_steps;

  // ---- protein staging: the tile sequence of the piece (every tile once
  // when resident and not already in place, else all tiles once per MC step
  // through the NS-stage ring).  Thread 0 issues the first copies; afterwards
  // the last warp to finish a stage (elected by the s_done counter) refills it.
  const float4 *src_a = T.pt_a + (size_t)prt_conf * T.pnp_pad;
  const float2 *src_b = T.pt_b;
  const int n_seq = passes * n_tl;
  auto issue_tile = [&](int s, int t) {
    unsigned char *dst = s_tiles + (size_t)s * STAGE_BYTES;
    mbar_arrive_expect_tx(&s_full[s], STAGE_BYTES);
    bulk_g2s(dst, src_a + (size_t)t * TILE_PTS, TILE_PTS * 16, &s_full[s]);
    bulk_g2s(dst + TILE_PTS * 16, src_b + (size_t)t * TILE_PTS, TILE_PTS * 8, &s_full[s]);
  };
  int it = s_ctl->it;  // ring position of the piece's first tile
  const int tiles_key = item * MAX_PRT_KEY + prt_conf;
  const bool reload = resident && tiles_key != s_ctl->tiles_key;
  const int gen = s_ctl->gen + (reload ? 1 : 0);
  if (threadIdx.x == 0) {
    // the previous piece's reads of the stages are ordered before the copies
    // by the barrier that ended it
    fence_proxy_async_smem();
    if (resident) {
      if (reload)
        for (int tl = 0; tl < n_tl; ++tl) issue_tile(tl, crank0 + csize * tl);
    } else {
      for (int q = 0; q < min(NS, n_seq); ++q)
        issue_tile((it + q) % NS, crank0 + csize * (q % n_tl));
    }
    // the steps before this piece ran on another CTA: wait until it has
    // written their state back (bounded; code 4 if it never does)
    if (wait_dep)
      wait_progress(R.progress + unit, step_base + R.wait_bias, R.err, 4,
                    R.wait_limit ? R.wait_limit : (1u << 24));
    s_ctl->first_it = it;
    s_ctl->sig_unit = unit;
    s_ctl->sig_step = launch_base + s_hi;
  }
  __syncthreads();  // every thread has read s_ctl; the dependency is met
  if (threadIdx.x == 0) {
    s_ctl->tiles_key = resident ? tiles_key : -1;
    s_ctl->gen = gen;
  }

  // ---- compute warps -----------------------------------------------------
  // warp w = pg + P ag: an atom group's P warps sit on P different schedulers
  // (w mod 4), so the groups whose atoms carry more H-bond pairs (the first
  // ones: capable atoms are dealt round robin from group 0) do not pile onto
  // one scheduler.  lw = pg A + ag numbers the warp's reduction slots and LHM
  // records, which keeps the order of every sum.
  const int ag = warp / P, pg = warp % P;
  const int lw = pg * A + ag;
  const int lna = T.lna;
  const bool active = lane < n_act;
  const int rep = lane_rep;                    // local replica / pose index
  const int lig_conf = (MODE == KMODE_POSES) ? R.lig_conf : rep % I.n_lig_conf;
  const float4 *orig = T.lig + (size_t)lig_conf * lna;
  LaneState &me = s_lane[lane];
  const float lcx = T.lig_center[0], lcy = T.lig_center[1], lcz = T.lig_center[2];
  // slots of this warp: ag + A k, k < n_my hold atoms
  const int n_my = lna > ag ? min(NA, (lna - ag + A - 1) / A) : 0;

  if (warp == 0) {
    me.acs = 0;
    me.idx_tmp = 0;
    me.mbeta = 0.f;
    if (MODE == KMODE_REMC) {
      // through L2: the state may have been written by another CTA
      me.idx_tmp = __ldcg(&I.idx_tmp[rep]);
      me.mbeta = I.minus_beta[me.idx_tmp];
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_old[i] = __ldcg(&I.m_old[(size_t)rep * 6 + i]);
#pragma unroll
      for (int i = 0; i < GD_NTERM; ++i)
        me.e_old[i] = __ldcg(&I.e_old[(size_t)rep * GD_NTERM + i]);
      me.cmcc_old = I.cmcc ? __ldcg(&I.cmcc[rep]) : 0.f;
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_old[i] = 0.f;
#pragma unroll
      for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = 0.f;
      me.cmcc_old = 0.f;
    }
    me.cmcc_new = 0.f;
  }
  const float inv_el1 = T.inv_el1;
  PairConst K;
  K.one = dup2(1.0f);
  K.lj1 = dup2(T.lj0lj1);
  K.lj0 = dup2(T.lj0);
  K.ca = dup2(-0.5f * LOG2E);
  K.cb = dup2(6.0f * LOG2E);
  const float4 *my_ptab = s_ptab + (size_t)ag * NH * PT_ROWS * 2;
  const float4 *my_htab = s_htab + (size_t)ag * NH * PT_ROWS;
  const uint32_t *my_hmask = s_hmask + (size_t)ag * PT_ROWS;
  const bool mcc_on = MODE != KMODE_POSES && (I.flags & GD_MC_MCC) != 0u;
  // atom pairs of this warp with an H-bond term for some point type: the
  // first my_nhb pairs (capable atoms come first in the slot order)
  const int my_nhb =
      32 - __clz(__reduce_or_sync(0xffffffffu, lane < PT_ROWS ? my_hmask[lane] : 0u));
  // the host's bound must cover this warp; report it if not (code 3)
  if (my_nhb > HB && lane == 0) atomicExch(R.err, 3);
  // warps whose atoms need fewer H-bond pairs than the launch's HB take a
  // variant with one pair less (most warps of a ligand: the capable atoms
  // come first in the slot order, dealt round robin over the atom groups)
  constexpr int kHB1 = HB > 1 ? HB - 1 : HB;

  for (int si = 0; si < n_steps; ++si) {
    const int step = step_base + si;

    // ---- warp 0 proposes the move and publishes it -------------------------
    if (warp == 0) {
      float m_new[6];
      if (MODE == KMODE_REMC) {
        uint32_t k0, k1;
        rng_key(I.seed, I.stream_id, k0, k1);
        const U4 a = philox4x32_10(U4{(uint32_t)rep, (uint32_t)step, 0u, 0u}, k0, k1);
        const U4 b = philox4x32_10(U4{(uint32_t)rep, (uint32_t)step, 1u, 0u}, k0, k1);
        const uint32_t bits[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
        me.u_bits = b.z;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const float pert = __fadd_rn(__fmul_rn(2.0f, u01(bits[i])), -1.0f);
          m_new[i] = __fadd_rn(__fmul_rn(I.move_scale[i], pert), me.m_old[i]);
        }
      } else if (MODE == KMODE_INIT) {
        const bool away = (I.flags & GD_MC_MOVE_AWAY) != 0;
#pragma unroll
        for (int i = 0; i < 6; ++i)
          m_new[i] = away ? __fadd_rn(__fmul_rn(I.move_scale[i], 44.5f), 0.0f) : 0.0f;
      } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) m_new[i] = active ? R.poses[(size_t)rep * 6 + i] : 0.f;
      }
      float rot[9];
      make_rot(m_new[3], m_new[4], m_new[5], rot);
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_new[i] = m_new[i];
#pragma unroll
      for (int i = 0; i < 9; ++i) me.rot[i] = rot[i];
    }
    named_sync(1, W * 32);

    // ---- place this warp's atoms (negated: d = atom - point = (-point)... ---
    const float q00 = me.rot[0], q01 = me.rot[1], q02 = me.rot[2];
    const float q10 = me.rot[3], q11 = me.rot[4], q12 = me.rot[5];
    const float q20 = me.rot[6], q21 = me.rot[7], q22 = me.rot[8];
    const float t0 = me.m_new[0], t1 = me.m_new[1], t2 = me.m_new[2];
    // nx[h] = {-x of slot 2h, -x of slot 2h+1}: point - atom = px + nx
    float2 nx[NH], ny[NH], nz[NH];
    // per-atom hydrophobic sums of this warp's tiles live in shared memory
    // (touched only on the close-range path)
    float2 *my_hpc2 = reinterpret_cast<float2 *>(s_hpc) + (size_t)(pg * A + ag) * NH * 32 + lane;
#pragma unroll
    for (int k = 0; k < NA; ++k) {
      const float4 o =
          (k < n_my) ? orig[s_atom[ag + A * k]] : make_float4(FAR, FAR, FAR, 0.f);
      const float x = q00 * o.x + q01 * o.y + q02 * o.z + t0 + lcx;
      const float y = q10 * o.x + q11 * o.y + q12 * o.z + t1 + lcy;
      const float z = q20 * o.x + q21 * o.y + q22 * o.z + t2 + lcz;
      if (k & 1) {
        nx[k >> 1].y = -x;
        ny[k >> 1].y = -y;
        nz[k >> 1].y = -z;
      } else {
        nx[k >> 1].x = -x;
        ny[k >> 1].x = -y;
        nz[k >> 1].x = -z;
      }
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) my_hpc2[h * 32] = make_float2(0.f, 0.f);

    // ---- pair terms over the protein tiles -----------------------------------
    // FP64 sums of this lane live in the warp's own reduction slots (read by
    // warp 0 after the barrier), which keeps registers for the pair loop
    double *my_red = s_red + (size_t)lw * NRED * 32 + lane;
#pragma unroll
    for (int i = 0; i < NRED; ++i) my_red[i * 32] = 0.0;
    // resident: the tile groups take the 32-point chunks round robin
    // (chunk c to group c mod P), which balances them to within one chunk.
    // Streaming: the same split of every tile of the ring, and every warp
    // waits for every stage and reports it done, chunk or not
    constexpr int CPT = TILE_PTS / CHUNK;  // chunks per tile
    for (int tl = 0; tl < n_tl; ++tl, ++it) {
      const int t = crank0 + csize * tl;  // protein tile
      const int nvalid = min(TILE_PTS, T.pnp - t * TILE_PTS);
      const int nvalid2 = nvalid;
      const int k0 = ((pg - (t * CPT) % P) % P + P) % P;
      const int kstep = P;
      if (resident && k0 * CHUNK >= nvalid2) continue;  // no chunk of this tile here
      const int s = resident ? tl : (it % NS);
      // resident tiles: the phase of their latest load (s_ctl->gen loads so far)
      const uint32_t ph = resident ? (uint32_t)((s_ctl->gen - 1) & 1) : (uint32_t)((it / NS) & 1);
      mbar_wait(&s_full[s], ph, R.err, 2);
      const float4 *ta = reinterpret_cast<const float4 *>(s_tiles + (size_t)s * STAGE_BYTES);
      const float2 *tb =
          reinterpret_cast<const float2 *>(s_tiles + (size_t)s * STAGE_BYTES + TILE_PTS * 16);
      for (int j0 = k0 * CHUNK; j0 < nvalid2; j0 += kstep * CHUNK) {
        const int j1 = min(nvalid2, j0 + CHUNK);
        float2 fvdw = dup2(0.f), fpmf = dup2(0.f), fhdb = dup2(0.f);
        float fnear = 0.f, fpsp = 0.f;
        float2 fek[NH];  // sum of ele_p / d per atom (far-field electrostatics)
#pragma unroll
        for (int h = 0; h < NH; ++h) fek[h] = dup2(0.f);
        // the chunk's variant of the fast path: with the H-bond term when one
        // of its points has a type that forms one with an atom of this warp
        // (points are ordered so that chunks rarely mix the two kinds); the
        // close-range votes are collected in a mask and served after the
        // branch-free pass, so consecutive points' chains overlap
        const int jl = j0 + lane;
        const uint32_t meta_l = jl < j1 ? __float_as_uint(tb[jl].y) : (uint32_t)PAD_POINT_TYPE;
        const bool chunk_hdb = __any_sync(0xffffffffu, my_hmask[meta_l & META_TYPE_MASK] != 0u);
        float thr_l = T.near4[((meta_l & META_HPC_BIT) ? 1 : 0) |
                              ((((meta_l >> META_CLASS_SHIFT) & 3u) == 2u) ? 2 : 0)];
        if (mcc_on) thr_l = fmaxf(thr_l, T.near_mcc2);
        // three variants per kernel: no H-bond term, HB - 1 pairs (warps that
        // need no more) and HB pairs; each is a long unrolled body, so more
        // of them would cost more in instruction fetch than they save
        const uint32_t close =
            (chunk_hdb && my_nhb > 0)
                ? (my_nhb <= kHB1
                       ? chunk_fast<NH, kHB1>(nx, ny, nz, ta, tb, j0, j1, my_ptab, my_htab, K,
                                              thr_l, fvdw, fpmf, fhdb, fek)
                       : chunk_fast<NH, HB>(nx, ny, nz, ta, tb, j0, j1, my_ptab, my_htab, K,
                                            thr_l, fvdw, fpmf, fhdb, fek))
                : chunk_fast<NH, 0>(nx, ny, nz, ta, tb, j0, j1, my_ptab, my_htab, K, thr_l,
                                    fvdw, fpmf, fhdb, fek);
        if (close) {
          // the chunk's hydrophobic sums in registers, added to the per-atom
          // sums once per chunk
          float2 hacc[NH];
#pragma unroll
          for (int h = 0; h < NH; ++h) hacc[h] = make_float2(0.f, 0.f);
          for (uint32_t m = close; m != 0u; m &= m - 1u) {
            const int j = j0 + __ffs(m) - 1;
            const uint32_t meta = __float_as_uint(tb[j].y);
            close_range<NA>(nx, ny, nz, ta[j], tb[j].x, meta,
                            my_ptab + (int)(meta & META_TYPE_MASK) * 2, T, s_q, s_lt, s_atom,
                            hacc, A, ag, n_my, inv_el1, fnear, fpsp, mcc_on, t * TILE_PTS + j,
                            my_red);
          }
#pragma unroll
          for (int h = 0; h < NH; ++h) my_hpc2[h * 32] = add2(my_hpc2[h * 32], hacc[h]);
        }
        float fele = 0.f;
#pragma unroll
        for (int h = 0; h < NH; ++h) {
          fele = fmaf(s_q[ag + A * (2 * h)], fek[h].x, fele);
          fele = fmaf(s_q[ag + A * (2 * h + 1)], fek[h].y, fele);
        }
        my_red[0 * 32] += (double)fvdw.x + (double)fvdw.y;
        my_red[1 * 32] += (double)fele * (double)inv_el1 + (double)fnear;
        my_red[2 * 32] += (double)fpmf.x + (double)fpmf.y;
        my_red[3 * 32] += (double)fpsp;
        my_red[4 * 32] += (double)fhdb.x + (double)fhdb.y;
      }
      if (!resident) {
        // the last of the W warps to finish this stage refills it with the
        // tile NS positions later in the sequence
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          if (atomicAdd(&s_done[s], 1) == W - 1) {
            s_done[s] = 0;
            __threadfence_block();
            const int q = it - s_ctl->first_it;  // position within the piece
            if (q + NS < n_seq) {
              fence_proxy_async_smem();
              issue_tile(s, crank0 + csize * ((q + NS) % n_tl));
            }
          }
        }
      }
    }

    // ---- KDE ------------------------------------------------------------------
    double dkde = 0.0, dlhm = 0.0;
#pragma unroll
    for (int k = 0; k < NA; ++k) {
      if (k < n_my && k % P == pg && crank0 == 0) {  // rank 0 of a split
        const int lt = s_lt[ag + A * k];
        const int kb = T.kde_off[lt], ke = T.kde_off[lt + 1];
        if (ke > kb) {
          const float2 ax = nx[k >> 1], ay = ny[k >> 1], az = nz[k >> 1];
          const float x = -((k & 1) ? ax.y : ax.x);
          const float y = -((k & 1) ? ay.y : ay.x);
          const float z = -((k & 1) ? az.y : az.x);
          float kv = 0.f;
          for (int q = kb; q < ke; ++q) {
            const float4 K = T.kde[q];
            const float dx = x - K.x, dy = y - K.y, dz = z - K.z;
            kv += fex2(T.kde2 * LOG2E * fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
          }
          dkde += (double)kv / (double)(ke - kb);
        }
      }
    }
    // ---- LHM position restraints: MCS records m = lw, lw + W, ... -----------
    for (int m = crank0 == 0 ? lw : T.pos; m < T.pos; m += W) {
      float sv = 0.f;
      const float4 *Mm = T.mcs + (size_t)m * lna;
      for (int l = 0; l < lna; ++l) {
        const float4 M = Mm[l];
        if (M.w != 0.0f) {
          const float4 o = orig[l];
          const float x = q00 * o.x + q01 * o.y + q02 * o.z + t0 + lcx;
          const float y = q10 * o.x + q11 * o.y + q12 * o.z + t1 + lcy;
          const float z = q20 * o.x + q21 * o.y + q22 * o.z + t2 + lcz;
          const float dx = x - M.x, dy = y - M.y, dz = z - M.z;
          sv += fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        }
      }
      dlhm += (double)T.mcs_tcc[m] * sqrt((double)sv / (double)T.mcs_cnt[m]);
    }

    // ---- cross-warp reduction and finalisation (warp 0) ----------------------
    {
      my_red[6 * 32] = dkde;
      my_red[7 * 32] = dlhm;
    }
    named_sync(1, W * 32);
    if (csize > 1) {
      // split: this CTA's partial sums go to the exchange buffer of the step's
      // parity; after the cluster barrier every CTA adds all ranks' buffers in
      // rank order (the same totals in every CTA) and takes the same decision.
      // A buffer is rewritten two steps later, after the next barrier, which
      // no CTA passes before it has read this step's buffers.
      unsigned char *xb = smem + SL.xch + (size_t)(si & 1) * SL.xch_step;
      double *xs = reinterpret_cast<double *>(xb);
      float2 *xh2 = reinterpret_cast<float2 *>(xb + (size_t)NRED * 32 * sizeof(double));
      float2 *s_hpc2 = reinterpret_cast<float2 *>(s_hpc);
      // both halves spread over the warps (tasks i = lw, lw + W, ... of the
      // NRED terms and the A x NH atom pairs, each summed in a fixed order):
      // this CTA's sums over its warp slots and tile groups into the buffer
      for (int i = lw; i < NRED + A * NH; i += W) {
        if (i < NRED) {
          double acc = 0.0;
          for (int w = 0; w < W; ++w) acc += s_red[((size_t)w * NRED + i) * 32 + lane];
          xs[i * 32 + lane] = acc;
        } else {
          const int j = i - NRED;  // atom pair (ag, h) = (j / NH, j % NH)
          float2 v = make_float2(0.f, 0.f);
          for (int g = 0; g < P; ++g) {
            const float2 x = s_hpc2[hpc_pair_at(g, j / NH, j % NH, lane, A, NH)];
            v.x += x.x;
            v.y += x.y;
          }
          xh2[j * 32 + lane] = v;
        }
      }
      cluster_sync_all();
      // then all ranks' buffers in rank order into slot 0 (terms) and tile
      // group 0's slots (the atom pairs' hydrophobic restraints)
      for (int i = lw; i < NRED + A * NH; i += W) {
        if (i < NRED) {
          double acc = 0.0;
          for (int r = 0; r < csize; ++r) acc += cluster_map(xs, r)[i * 32 + lane];
          s_red[(size_t)i * 32 + lane] = acc;
        } else {
          const int j = i - NRED, ai = j / NH, hp = j % NH;
          float2 v = make_float2(0.f, 0.f);
          for (int r = 0; r < csize; ++r) {
            const float2 x = cluster_map(xh2, r)[j * 32 + lane];
            v.x += x.x;
            v.y += x.y;
          }
          if (ai + 2 * hp * A < lna)
            s_hpc2[hpc_pair_at(0, ai, hp, lane, A, NH)] = hpc_transform(T, s_lt, A, ai, hp, v);
        }
      }
      named_sync(1, W * 32);
      if (warp == 0)
        finish_step<MODE>(R, I, me, s_red, s_hpc, s_lt, 1, 1, A, NH, lane, rep, active, prt_conf,
                          lig_conf, step, crank0 == 0, true);
    } else {
      // spread over the warps (tasks i = lw, lw + W, ...): the cross-warp sum
      // of each of the NRED terms (in warp-slot order, into slot 0) and the
      // hydrophobic restraint of each of the A x NH atom pairs (into tile
      // group 0's slot of the pair); warp 0 then finishes from slot 0 alone
      float2 *s_hpc2 = reinterpret_cast<float2 *>(s_hpc);
      for (int i = lw; i < NRED + A * NH; i += W) {
        if (i < NRED) {
          double acc = 0.0;
          for (int w = 0; w < W; ++w) acc += s_red[((size_t)w * NRED + i) * 32 + lane];
          s_red[(size_t)i * 32 + lane] = acc;
        } else {
          const int ai = (i - NRED) / NH, hp = (i - NRED) % NH;
          if (ai + 2 * hp * A >= lna) continue;
          const float2 r = hpc_restraint(T, s_hpc2, s_lt, P, A, NH, ai, hp, lane);
          s_hpc2[hpc_pair_at(0, ai, hp, lane, A, NH)] = r;
        }
      }
      named_sync(1, W * 32);
      if (warp == 0)
        finish_step<MODE>(R, I, me, s_red, s_hpc, s_lt, 1, P, A, NH, lane, rep, active, prt_conf,
                          lig_conf, step, true, true);
    }
    // the next step's first barrier orders warp 0's updates (and its use of
    // s_red for the exchange) before any other warp touches them again
  }

  // ---- write the replica state back (rank 0 of a split) ---------------------
  if (MODE != KMODE_POSES && warp == 0 && active && crank0 == 0) {
#pragma unroll
    for (int i = 0; i < 6; ++i) I.m_old[(size_t)rep * 6 + i] = me.m_old[i];
#pragma unroll
    for (int i = 0; i < GD_NTERM; ++i) I.e_old[(size_t)rep * GD_NTERM + i] = me.e_old[i];
    if (I.cmcc) I.cmcc[rep] = me.cmcc_old;
    if (MODE == KMODE_INIT) {
      I.acs_mc[rep] = 0;
      I.idx_tmp[rep] = (rep / I.n_lig_conf) % I.n_tmp;
    } else {
      I.acs_mc[rep] = __ldcg(&I.acs_mc[rep]) + me.acs;
      if (R.fused_exchange) I.idx_tmp[rep] = me.idx_tmp;
    }
  }

  // ---- end of the piece: publish its progress, move to the next ------------
  // (without pieces the loop body runs once: no back edge, so the pair loop
  // is compiled as in a plain kernel; a loop around it costs it registers)
  if (!PIECES) break;
  if (warp == 0) __threadfence();  // the state writes above, device-wide
  __syncthreads();  // every warp is done with the stages, tables and lanes
  if (threadIdx.x == 0) {
    st_release(R.progress + s_ctl->sig_unit, s_ctl->sig_step);
    s_ctl->pc += 1;
    s_ctl->it = it;
  }
  __syncthreads();
  }  // pieces
  // a split CTA leaves only when no other CTA of its cluster can still read
  // its exchange buffers
  if (csize > 1) cluster_sync_all();
  if (R.busy_ns) {  // the CTA's time on its SM, for occupancy statistics
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(R.busy_ns, global_ns() - t_start);
  }
}

// Temperature exchange, one thread per (item, protein conf, ligand conf)
// group (exchangereplicas_d.cu:26-79).  Pairs of adjacent temperature
// indices (2 pair + mode_t, 2 pair + mode_t + 1) swap their slots when
// exp((mb1 - mb2)(E2 - E1)) > u; the counters are kept per slot.
__global__ void exchange_kernel(const KItem *items, const KGroup *groups, int n_groups, int spe,
                                int step0, const int *step_ptr) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups) return;
  const KGroup G = groups[g];
  const KItem &I = items[G.item];
  // interval start: the device counter, the launch's step, or (step0 < 0)
  // each item's own step
  const bool per_item = !step_ptr && step0 < 0;
  const int s0 = step_ptr ? *step_ptr : (per_item ? I.step0 : step0);
  if (per_item) spe = I.spe;
  const int within = I.steps_per_dump > 0 ? (s0 % I.steps_per_dump) : s0;
  const int mode_t = (within / spe) % 2;
  const int round = s0 / spe;
  const int nt = I.n_tmp, nl = I.n_lig_conf;
  int temps[MAX_TMP], orders[MAX_TMP];
  float en[MAX_TMP];
  for (int t = 0; t < nt; ++t) {
    const int r = nt * nl * G.p + nl * t + G.l;
    temps[t] = I.idx_tmp[r];
    en[t] = I.e_old[(size_t)r * GD_NTERM + GD_E_TOTAL];
  }
  for (int t = 0; t < nt; ++t) orders[temps[t]] = t;
  uint32_t k0, k1;
  rng_key(I.seed, I.stream_id, k0, k1);
  const uint32_t gid = (uint32_t)(G.p * nl + G.l);
  const int maxpair = nt / 2 - (nt % 2 == 0) * (mode_t == 1);
  for (int pair = 0; pair < maxpair; ++pair) {
    const int i1 = (pair << 1) + mode_t;
    const int i2 = i1 + 1;
    const int o1 = orders[i1], o2 = orders[i2];
    const int tt = temps[o1];
    const float mb1 = I.minus_beta[temps[o1]];
    const float mb2 = I.minus_beta[temps[o2]];
    const float delta = __fmul_rn(__fsub_rn(mb1, mb2), __fsub_rn(en[o2], en[o1]));
    const float prob = decision_expf(delta);
    const U4 o = philox4x32_10(U4{gid, (uint32_t)round, 2u, (uint32_t)pair}, k0, k1);
    if (prob > u01(o.x)) {
      temps[o1] = temps[o2];
      temps[o2] = tt;
      atomicAdd(&I.acs_exchg[o1], 1);
      atomicAdd(&I.acs_exchg[o2], 1);
    }
  }
  for (int t = 0; t < nt; ++t) I.idx_tmp[nt * nl * G.p + nl * t + G.l] = temps[t];
}

__global__ void advance_kernel(int *step_ptr, int spe) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *step_ptr += spe;
}

__global__ void metropolis_kernel(int n, const float *e_new, const float *e_old,
                                  const float *mbeta, const int *rep, const int *step,
                                  uint64_t seed, uint32_t stream, int *acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k0, k1;
  rng_key(seed, stream, k0, k1);
  const U4 b = philox4x32_10(U4{(uint32_t)rep[i], (uint32_t)step[i], 1u, 0u}, k0, k1);
  acc[i] = metropolis(e_new[i], e_old[i], mbeta[i], u01(b.z));
}

__global__ void philox_kernel(int n, const uint32_t *ctr, const uint32_t *key, uint32_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U4 c{ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]};
  const U4 o = philox4x32_10(c, key[2 * i], key[2 * i + 1]);
  out[4 * i] = o.x;
  out[4 * i + 1] = o.y;
  out[4 * i + 2] = o.z;
  out[4 * i + 3] = o.w;
}

__global__ void expf_kernel(int n, const float *x, float *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = decision_expf(x[i]);
}

// FP32 FMA throughput probe: 8 independent dependent-FMA chains per thread.
__global__ void fma_peak_kernel(float *out, int iters) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  const float b = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fmaf(a0, b, c);
      a1 = fmaf(a1, b, c);
      a2 = fmaf(a2, b, c);
      a3 = fmaf(a3, b, c);
      a4 = fmaf(a4, b, c);
      a5 = fmaf(a5, b, c);
      a6 = fmaf(a6, b, c);
      a7 = fmaf(a7, b, c);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
template <int MODE, int NA, int HB, bool PIECES>
static cudaError_t launch_kernel(const KRun &R, int grid, cudaStream_t s, int *occ) {
  const int split = (MODE != KMODE_POSES && !PIECES && R.split > 1) ? R.split : 1;
  const size_t smem = dock_smem_bytes(R.A, R.P, NA, R.n_stages, split);
  const int threads = R.A * R.P * 32;
  cudaError_t e = cudaFuncSetAttribute(dock_kernel<MODE, NA, HB, PIECES>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (occ)  // occupancy query instead of a launch
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, dock_kernel<MODE, NA, HB, PIECES>,
                                                         threads, smem);
  if (split == 1) {
    dock_kernel<MODE, NA, HB, PIECES><<<grid, threads, smem, s>>>(R);
    return cudaGetLastError();
  }
  // clusters of `split` CTAs (grid = units x split), on SMs of one GPC
  if (split > 8 || grid % split) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = split;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, dock_kernel<MODE, NA, HB, PIECES>, R);
}

template <int MODE, int NA, int HB>
static cudaError_t launch_nahb(const KRun &R, int grid, cudaStream_t s, int *occ) {
  if constexpr (MODE == KMODE_REMC) {
    if (R.pieces) return launch_kernel<MODE, NA, HB, true>(R, grid, s, occ);
  } else {
    if (R.pieces) return cudaErrorInvalidValue;  // schedules are for MC steps
  }
  return launch_kernel<MODE, NA, HB, false>(R, grid, s, occ);
}

// Three H-bond bounds per NA: at most two or three pairs (ligands where up
// to about a third or half of the atoms have the term, the common cases), or
// every pair.
template <int MODE, int NA>
static cudaError_t launch_na(const KRun &R, int grid, cudaStream_t s, int *occ) {
  constexpr int NH = NA / 2;
  constexpr int HB2 = NH < 2 ? NH : 2;
  constexpr int HB3 = NH < 3 ? NH : 3;
  if (R.hb_pairs <= HB2) return launch_nahb<MODE, NA, HB2>(R, grid, s, occ);
  if (R.hb_pairs <= HB3) return launch_nahb<MODE, NA, HB3>(R, grid, s, occ);
  return launch_nahb<MODE, NA, NH>(R, grid, s, occ);
}

template <int MODE>
static cudaError_t launch_mode(const KRun &R, int NA, int grid, cudaStream_t s, int *occ) {
  switch (NA) {
    case 2: return launch_na<MODE, 2>(R, grid, s, occ);
    case 4: return launch_na<MODE, 4>(R, grid, s, occ);
    case 6: return launch_na<MODE, 6>(R, grid, s, occ);
    case 8: return launch_na<MODE, 8>(R, grid, s, occ);
    case 10: return launch_na<MODE, 10>(R, grid, s, occ);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t dock_dispatch(const KRun &R, int NA, int grid, cudaStream_t s, int *occ) {
  switch (R.mode) {
    case KMODE_POSES: return launch_mode<KMODE_POSES>(R, NA, grid, s, occ);
    case KMODE_REMC: return launch_mode<KMODE_REMC>(R, NA, grid, s, occ);
    default: return launch_mode<KMODE_INIT>(R, NA, grid, s, occ);
  }
}

cudaError_t launch_dock(const KRun &R, int NA, int grid, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  return dock_dispatch(R, NA, grid, s, nullptr);
}

cudaError_t dock_ctas_per_sm(const KRun &R, int NA, int *n) {
  *n = 0;
  return dock_dispatch(R, NA, 0, nullptr, n);
}

cudaError_t launch_exchange(const KItem *items, const KGroup *groups, int n_groups, int spe,
                            int step0, const int *step_ptr, cudaStream_t s) {
  if (n_groups <= 0) return cudaSuccess;
  exchange_kernel<<<(n_groups + 127) / 128, 128, 0, s>>>(items, groups, n_groups, spe, step0,
                                                          step_ptr);
  return cudaGetLastError();
}

cudaError_t launch_advance(int *step_ptr, int spe, cudaStream_t s) {
  advance_kernel<<<1, 32, 0, s>>>(step_ptr, spe);
  return cudaGetLastError();
}

cudaError_t launch_metropolis(int n, const float *e_new, const float *e_old, const float *mbeta,
                              const int *rep, const int *step, uint64_t seed, uint32_t stream_id,
                              int *acc, cudaStream_t s) {
  metropolis_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, e_new, e_old, mbeta, rep, step, seed,
                                                    stream_id, acc);
  return cudaGetLastError();
}

cudaError_t launch_philox(int n, const uint32_t *ctr, const uint32_t *key, uint32_t *out,
                          cudaStream_t s) {
  philox_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, ctr, key, out);
  return cudaGetLastError();
}

cudaError_t launch_expf(int n, const float *x, float *y, cudaStream_t s) {
  expf_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, x, y);
  return cudaGetLastError();
}

cudaError_t launch_fma_peak(float *out, int n_blocks, int iters, cudaStream_t s) {
  fma_peak_kernel<<<n_blocks, 256, 0, s>>>(out, iters);
  return cudaGetLastError();
}

}  // namespace gd
