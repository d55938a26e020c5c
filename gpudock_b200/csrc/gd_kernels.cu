// gd_kernels.cu -- sm_100a kernels of the REMC docking path.
//
// dock_kernel: one CTA owns up to 32 replicas (or poses) of one complex that
// share one protein conformation; lane i of every compute warp is replica i,
// so protein-point and type-table reads are warp-uniform shared-memory
// broadcasts.  The compute warps form an A x P grid: warp (ag, pg) keeps NA
// ligand atoms a = ag + A k in registers and sweeps the protein tiles
// t = pg, pg + P, ...  The protein conformation is staged in shared memory in
// 128-point tiles by the TMA engine (cp.async.bulk + mbarrier), once per
// launch when it fits (resident) or through an 8-stage ring fed by a
// producer warp (then P = 1).  Per step every warp writes FP64 partial sums
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

constexpr int TAB_N = TAB_ROWS * GD_NPT;
constexpr int TAB_BYTES = TAB_N * (16 + 8);
constexpr int STAGE_BYTES = TILE_PTS * (16 + 8);
constexpr int CHUNK = 32;  // points per FP32 partial before the FP64 flush
constexpr float LOG2E = 1.4426950408889634f;
constexpr float FAR = 1.0e4f;  // coordinate of the padding atoms

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
  float pad;
};
static_assert(sizeof(LaneState) == 144, "LaneState layout");
static_assert(sizeof(KItem) % 8 == 0, "KItem must keep the barriers 8-byte aligned");
static_assert(TAB_BYTES % 16 == 0, "tile staging must start 16-byte aligned");

size_t dock_smem_bytes(int A, int P, int NA, int n_stages) {
  const int W = A * P;
  return (size_t)TAB_BYTES + (size_t)n_stages * STAGE_BYTES +
         (size_t)W * NRED * 32 * sizeof(double) + (size_t)P * A * NA * 32 * sizeof(float) +
         32 * sizeof(LaneState) + sizeof(KItem) + (size_t)2 * n_stages * sizeof(uint64_t);
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

// Hydrophobic contact polynomial of calcenergy_d.cu:80-86 in Horner form:
// 1 - (3.5/81 d2 - 4.5/81^2 d4 + 2.5/81^3 d6 - 0.5/81^4 d8)
__device__ __forceinline__ float hpc_poly(float d2) {
  const float c1 = 3.5f / 81.0f;
  const float c2 = -4.5f / 81.0f / 81.0f;
  const float c3 = 2.5f / 81.0f / 81.0f / 81.0f;
  const float c4 = -0.5f / 81.0f / 81.0f / 81.0f / 81.0f;
  const float q = fmaf(fmaf(fmaf(c4, d2, c3), d2, c2), d2, c1);
  return 1.0f - q * d2;
}

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

// Warp 0 after the step's partial sums: cross-warp reduction in a fixed
// order, hydrophobic transform per atom, normalisation and total in the
// reference's order, then the pose output, or the Metropolis decision (with
// the trajectory record) and, at the end of an interval, the in-CTA
// temperature exchange.  Kept out of line so its registers do not burden the
// pair loop.
template <int MODE>
__device__ __noinline__ void finish_step(const KRun &R, const KItem &I, LaneState &me,
                                         double *s_red, const float *s_hpc, int W, int P,
                                         int MAXA, int lane, int rep, bool active, int prt_conf,
                                         int lig_conf, int step) {
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
    // hydrophobic restraint per ligand atom (calcenergy_d.cu:143-149)
    for (int a = 0; a < lna; ++a) {
      float h = 0.f;
      for (int g = 0; g < P; ++g) h += s_hpc[((size_t)g * MAXA + a) * 32 + lane];
      const int lt = T.lig_t[a];
      const float hh = __fdiv_rn(__fsub_rn(h, T.hpl0[lt]), T.hpl1[lt]);
      S[5] += (double)__fsub_rn(__fmul_rn(__fmul_rn(0.5f, hh), hh), T.hpl2[lt]);
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
    e[9] = tot;

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
        if (active && I.record && step < I.rec_steps) {
          gd_record *rc = I.record + (size_t)rep * I.rec_steps + step;
          rc->idx_rep = rep;
          rc->idx_prt = prt_conf;
          rc->idx_tmp = me.idx_tmp;
          rc->idx_lig = lig_conf;
#pragma unroll
          for (int i = 0; i < GD_NTERM; ++i) rc->e[i] = me.e_old[i];
          rc->cmcc = 0.f;
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
              atomicAdd(&I.acs_exchg[o1], 1);
              atomicAdd(&I.acs_exchg[o2], 1);
            }
          }
        }
        __syncwarp();
        me.idx_tmp = s_tmp[lane];
        me.mbeta = I.minus_beta[me.idx_tmp];
      }
    }
  }

template <int MODE, int NA>
__global__ void __launch_bounds__((MAX_WARPS + 1) * 32, 1)
    dock_kernel(const __grid_constant__ KRun R) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int A = R.A, P = R.P, W = A * P, NS = R.n_stages;
  const int MAXA = A * NA;
  float4 *s_tab_a = reinterpret_cast<float4 *>(smem);
  float2 *s_tab_b = reinterpret_cast<float2 *>(smem + TAB_N * 16);
  unsigned char *s_tiles = smem + TAB_BYTES;
  double *s_red = reinterpret_cast<double *>(s_tiles + (size_t)NS * STAGE_BYTES);
  float *s_hpc = reinterpret_cast<float *>(s_red + (size_t)W * NRED * 32);
  LaneState *s_lane = reinterpret_cast<LaneState *>(s_hpc + (size_t)P * MAXA * 32);
  KItem *s_item = reinterpret_cast<KItem *>(s_lane + 32);
  uint64_t *s_full = reinterpret_cast<uint64_t *>(s_item + 1);
  uint64_t *s_empty = s_full + NS;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  // ---- item of this CTA into shared memory, type table, barriers ----------
  const int item = (MODE == KMODE_POSES) ? 0 : R.cta_item[blockIdx.x];
  const KItem &G = R.items[item];
  {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&G);
    uint32_t *dst = reinterpret_cast<uint32_t *>(s_item);
    for (int i = threadIdx.x; i < (int)(sizeof(KItem) / 4); i += blockDim.x) dst[i] = src[i];
    const float4 *ta = G.T.tab_a;
    const float2 *tb = G.T.tab_b;
    for (int i = threadIdx.x; i < TAB_N; i += blockDim.x) {
      s_tab_a[i] = ta[i];
      s_tab_b[i] = tb[i];
    }
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], W);
    }
    fence_barrier_init();
  }
  __syncthreads();
  const KItem &I = *s_item;
  const KTables &T = I.T;

  // ---- work of this CTA --------------------------------------------------
  int rep0, n_act, prt_conf, lane_rep;
  if (MODE == KMODE_POSES) {
    rep0 = blockIdx.x * 32;
    n_act = min(32, R.n_pose - rep0);
    prt_conf = R.prt_conf;
    lane_rep = rep0 + (lane < n_act ? lane : 0);
  } else if (R.group_major) {
    // whole exchange groups: lane = group offset * n_tmp + temperature slot
    const int nt = I.n_tmp, nl = I.n_lig_conf;
    const int g0 = R.cta_rep0[blockIdx.x];
    n_act = R.cta_nrep[blockIdx.x];
    rep0 = g0;
    prt_conf = g0 / nl;
    const int ln = lane < n_act ? lane : 0;
    lane_rep = nt * nl * prt_conf + nl * (ln % nt) + (g0 % nl) + ln / nt;
  } else {
    rep0 = R.cta_rep0[blockIdx.x];
    n_act = R.cta_nrep[blockIdx.x];
    prt_conf = rep0 / (I.n_tmp * I.n_lig_conf);
    lane_rep = rep0 + (lane < n_act ? lane : 0);
  }
  const int n_tiles = (T.pnp + TILE_PTS - 1) / TILE_PTS;
  const bool resident = R.resident != 0;
  const int n_steps = (MODE == KMODE_REMC) ? R.n_steps : 1;
  const int passes = resident ? 1 : n_steps;
  const int step_base = (MODE == KMODE_REMC && R.item_step)  ? I.step0
                        : (MODE == KMODE_REMC && R.step_ptr) ? *R.step_ptr
                                                             : R.step0;

  // ---- producer warp: stages the protein conformation -------------------
  if (warp == W) {
    if (lane == 0) {
      const float4 *src_a = T.pt_a + (size_t)prt_conf * T.pnp_pad;
      const float2 *src_b = T.pt_b;
      int it = 0;
      for (int pass = 0; pass < passes; ++pass) {
        for (int t = 0; t < n_tiles; ++t, ++it) {
          const int s = resident ? t : (it % NS);
          if (!resident) {
            const uint32_t ph = (uint32_t)((it / NS) & 1);
            mbar_wait(&s_empty[s], ph ^ 1u, R.err, 1);
          }
          unsigned char *dst = s_tiles + (size_t)s * STAGE_BYTES;
          mbar_arrive_expect_tx(&s_full[s], STAGE_BYTES);
          bulk_g2s(dst, src_a + (size_t)t * TILE_PTS, TILE_PTS * 16, &s_full[s]);
          bulk_g2s(dst + TILE_PTS * 16, src_b + (size_t)t * TILE_PTS, TILE_PTS * 8, &s_full[s]);
        }
      }
    }
    return;
  }

  // ---- compute warps -----------------------------------------------------
  const int ag = warp % A, pg = warp / A;
  const int lna = T.lna;
  const bool active = lane < n_act;
  const int rep = lane_rep;                    // local replica / pose index
  const int lig_conf = (MODE == KMODE_POSES) ? R.lig_conf : rep % I.n_lig_conf;
  const float4 *orig = T.lig + (size_t)lig_conf * lna;
  LaneState &me = s_lane[lane];
  const float lcx = T.lig_center[0], lcy = T.lig_center[1], lcz = T.lig_center[2];

  // this warp's atoms; padding atoms use the all-zero table row, no charge,
  // and sit far from everything
  int lto[NA];
  float lq[NA];  // charge / el1: far-field electrostatics is q ele / (el1 d)
  int n_my = 0;
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    const int a = ag + A * k;
    if (a < lna) {
      n_my = k + 1;
      lto[k] = T.lig_t[a] * GD_NPT;
      lq[k] = T.lig_q[a];
    } else {
      lto[k] = GD_NLT * GD_NPT;
      lq[k] = 0.f;
    }
  }

  if (warp == 0) {
    me.acs = 0;
    me.idx_tmp = 0;
    me.mbeta = 0.f;
    if (MODE == KMODE_REMC) {
      me.idx_tmp = I.idx_tmp[rep];
      me.mbeta = I.minus_beta[me.idx_tmp];
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_old[i] = I.m_old[(size_t)rep * 6 + i];
#pragma unroll
      for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = I.e_old[(size_t)rep * GD_NTERM + i];
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_old[i] = 0.f;
#pragma unroll
      for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = 0.f;
    }
  }
  const float lj0 = T.lj0, lj0lj1 = T.lj0lj1, inv_el1 = T.inv_el1, near_d2 = T.near_d2;

  int it = 0;  // streaming ring position
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

    // ---- place this warp's atoms -------------------------------------------
    const float q00 = me.rot[0], q01 = me.rot[1], q02 = me.rot[2];
    const float q10 = me.rot[3], q11 = me.rot[4], q12 = me.rot[5];
    const float q20 = me.rot[6], q21 = me.rot[7], q22 = me.rot[8];
    const float t0 = me.m_new[0], t1 = me.m_new[1], t2 = me.m_new[2];
    float lx[NA], ly[NA], lz[NA];
    // per-atom hydrophobic sums of this warp's tiles live in shared memory
    // (touched only on the close-range path)
    float *my_hpc = s_hpc + ((size_t)pg * MAXA + ag) * 32 + lane;  // + A*k*32 per atom
#pragma unroll
    for (int k = 0; k < NA; ++k) {
      // padding atoms sit far from everything
      const float4 o = (k < n_my) ? orig[ag + A * k] : make_float4(FAR, FAR, FAR, 0.f);
      lx[k] = q00 * o.x + q01 * o.y + q02 * o.z + t0 + lcx;
      ly[k] = q10 * o.x + q11 * o.y + q12 * o.z + t1 + lcy;
      lz[k] = q20 * o.x + q21 * o.y + q22 * o.z + t2 + lcz;
      if (k < n_my) my_hpc[(size_t)A * k * 32] = 0.f;
    }

    // ---- pair terms over the protein tiles -----------------------------------
    // FP64 sums of this lane live in the warp's own reduction slots (read by
    // warp 0 after the barrier), which keeps registers for the pair loop
    double *my_red = s_red + (size_t)warp * NRED * 32 + lane;
#pragma unroll
    for (int i = 0; i < NRED; ++i) my_red[i * 32] = 0.0;
    const int t_first = resident ? pg : 0;
    const int t_step = resident ? P : 1;
    for (int t = t_first; t < n_tiles; t += t_step, ++it) {
      const int s = resident ? t : (it % NS);
      const uint32_t ph = resident ? 0u : (uint32_t)((it / NS) & 1);
      mbar_wait(&s_full[s], ph, R.err, 2);
      const float4 *ta = reinterpret_cast<const float4 *>(s_tiles + (size_t)s * STAGE_BYTES);
      const float2 *tb =
          reinterpret_cast<const float2 *>(s_tiles + (size_t)s * STAGE_BYTES + TILE_PTS * 16);
      const int nvalid = min(TILE_PTS, T.pnp - t * TILE_PTS);
      for (int j0 = 0; j0 < nvalid; j0 += CHUNK) {
        const int j1 = min(nvalid, j0 + CHUNK);
        float fvdw = 0.f, fnear = 0.f, fpmf = 0.f, fpsp = 0.f, fhdb = 0.f;
        float fek[NA];  // sum of ele_p / d per atom (far-field electrostatics)
#pragma unroll
        for (int k = 0; k < NA; ++k) fek[k] = 0.f;
        for (int j = j0; j < j1; ++j) {
          const float4 Ap = ta[j];
          const float2 Bp = tb[j];
          const uint32_t meta = __float_as_uint(Bp.y);
          const int pt = (int)(meta & META_TYPE_MASK);
          float mn = 3.0e38f;
          // fast path: soft LJ, far-field electrostatics, contact PMF.  The LJ
          // and PMF quotients share one reciprocal: with D1 = p4 and
          // D2 = 1 + exp(.), num1/D1 = num1 D2 / (D1 D2); d2 >= 1e-6 keeps
          // D1 D2 below 1e35.
#pragma unroll
          for (int k = 0; k < NA; ++k) {
            const float4 Pk = s_tab_a[lto[k] + pt];  // p1a p2a pmf0 pmf1
            const float dx = lx[k] - Ap.x;
            const float dy = ly[k] - Ap.y;
            const float dz = lz[k] - Ap.z;
            const float d2 = fmaxf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)), 1.0e-6f);
            const float r = frsqrt(d2);
            const float d = d2 * r;
            const float r2 = r * r;
            const float r3 = r2 * r;
            const float r6 = r3 * r3;
            const float r9 = r6 * r3;
            const float p1 = Pk.x * r9;
            const float p2 = Pk.y * r6;
            const float p4 = fmaf(p1, fmaf(lj0lj1, d2, lj0), 1.0f);
            const float dm = d - Pk.z;
            const float e1 = 1.0f + fex2(fmaf(-0.5f * LOG2E, d, 6.0f * LOG2E) * dm);
            const float inv = frcp(p4 * e1);
            fvdw = fmaf((p1 - p2) * e1, inv, fvdw);
            fpmf = fmaf(Pk.w * p4, inv, fpmf);
            fek[k] = fmaf(Ap.w, r, fek[k]);
            mn = fminf(mn, d2);
            // hydrogen bond, for the type pairs that define one
            const float2 Hk = s_tab_b[lto[k] + pt];  // hdb0 hdb1
            if (Hk.x > 0.1f) {
              const float h3 = (d - Hk.x) * Hk.y;
              fhdb = fmaf(Hk.y, fex2((-0.5f * LOG2E) * h3 * h3), fhdb);
            }
          }
          // close-range terms, only when some lane has an atom within near_d2
          // (distances recomputed: this path is taken for a few % of points)
          if (__any_sync(0xffffffffu, mn <= near_d2)) {
            const bool is_c2 = ((meta >> META_CLASS_SHIFT) & 3u) == 2u;
            const bool hflag = (meta & META_HPC_BIT) != 0u;
#pragma unroll
            for (int k = 0; k < NA; ++k) {
              const float dx = lx[k] - Ap.x;
              const float dy = ly[k] - Ap.y;
              const float dz = lz[k] - Ap.z;
              const float d2 = fmaxf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)), 1.0e-6f);
              const float rk = frsqrt(d2);
              const float d = d2 * rk;
              if (hflag && d2 <= 81.0f && k < n_my) {
                float *h = my_hpc + (size_t)A * k * 32;
                *h = fmaf(Bp.x, hpc_poly(d2), *h);
              }
              const float s1 = T.el1 * d;
              if (s1 < 1.0f) {
                const float gnear = fmaf(s1 * s1, fmaf(T.b1, s1, T.a1), T.el0);
                fnear = fmaf(lq[k] * Ap.w, gnear - rk * inv_el1, fnear);
              }
              if (is_c2 && k < n_my) {
                const float dm = d - s_tab_a[lto[k] + pt].z;
                if (dm <= 0.0f)
                  fpsp += __ldg(&T.psp[(size_t)(lto[k] / GD_NPT) * T.psp_ncol +
                                       (meta >> META_SEQ_SHIFT)]);
              }
            }
          }
        }
        float fele = 0.f;
#pragma unroll
        for (int k = 0; k < NA; ++k) fele = fmaf(lq[k], fek[k], fele);
        my_red[0 * 32] += (double)fvdw;
        my_red[1 * 32] += (double)fele * (double)inv_el1 + (double)fnear;
        my_red[2 * 32] += (double)fpmf;
        my_red[3 * 32] += (double)fpsp;
        my_red[4 * 32] += (double)fhdb;
      }
      if (!resident) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_empty[s]);
      }
    }

    // ---- per-atom hydrophobic sums, KDE --------------------------------------
    double dkde = 0.0, dlhm = 0.0;
#pragma unroll
    for (int k = 0; k < NA; ++k) {
      if (k < n_my) {
        if (k % P == pg) {
          const int lt = lto[k] / GD_NPT;
          const int kb = T.kde_off[lt], ke = T.kde_off[lt + 1];
          if (ke > kb) {
            float kv = 0.f;
            for (int q = kb; q < ke; ++q) {
              const float4 K = T.kde[q];
              const float dx = lx[k] - K.x, dy = ly[k] - K.y, dz = lz[k] - K.z;
              kv += fex2(T.kde2 * LOG2E * fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
            }
            dkde += (double)kv / (double)(ke - kb);
          }
        }
      }
    }
    // ---- LHM position restraints: MCS records m = warp, warp + W, ... -------
    for (int m = warp; m < T.pos; m += W) {
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
    if (warp == 0)
      finish_step<MODE>(R, I, me, s_red, s_hpc, W, P, MAXA, lane, rep, active, prt_conf,
                        lig_conf, step);
    // the next step's first barrier orders warp 0's updates (and its use of
    // s_red for the exchange) before any other warp touches them again
  }

  // ---- write the replica state back ----------------------------------------
  if (MODE != KMODE_POSES && warp == 0 && active) {
#pragma unroll
    for (int i = 0; i < 6; ++i) I.m_old[(size_t)rep * 6 + i] = me.m_old[i];
#pragma unroll
    for (int i = 0; i < GD_NTERM; ++i) I.e_old[(size_t)rep * GD_NTERM + i] = me.e_old[i];
    if (MODE == KMODE_INIT) {
      I.acs_mc[rep] = 0;
      I.idx_tmp[rep] = (rep / I.n_lig_conf) % I.n_tmp;
    } else {
      I.acs_mc[rep] += me.acs;
      if (R.fused_exchange) I.idx_tmp[rep] = me.idx_tmp;
    }
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
  const int s0 = step_ptr ? *step_ptr : (step0 >= 0 ? step0 : I.step0);
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
template <int MODE, int NA>
static cudaError_t launch_na(const KRun &R, int grid, cudaStream_t s) {
  const size_t smem = dock_smem_bytes(R.A, R.P, NA, R.n_stages);
  const int threads = (R.A * R.P + 1) * 32;
  cudaError_t e = cudaFuncSetAttribute(dock_kernel<MODE, NA>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dock_kernel<MODE, NA><<<grid, threads, smem, s>>>(R);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_mode(const KRun &R, int NA, int grid, cudaStream_t s) {
  switch (NA) {
    case 1: return launch_na<MODE, 1>(R, grid, s);
    case 2: return launch_na<MODE, 2>(R, grid, s);
    case 3: return launch_na<MODE, 3>(R, grid, s);
    case 4: return launch_na<MODE, 4>(R, grid, s);
    case 5: return launch_na<MODE, 5>(R, grid, s);
    case 6: return launch_na<MODE, 6>(R, grid, s);
    case 8: return launch_na<MODE, 8>(R, grid, s);
    case 10: return launch_na<MODE, 10>(R, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_dock(const KRun &R, int NA, int grid, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  switch (R.mode) {
    case KMODE_POSES: return launch_mode<KMODE_POSES>(R, NA, grid, s);
    case KMODE_REMC: return launch_mode<KMODE_REMC>(R, NA, grid, s);
    default: return launch_mode<KMODE_INIT>(R, NA, grid, s);
  }
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
