// gd_kernels.cu -- sm_100a kernels of the REMC docking path.
//
// dock_kernel: one CTA owns up to 32 replicas (or poses) that share one
// protein conformation; lane i of every compute warp is replica i, so all
// protein-point and type-table reads are warp-uniform shared-memory
// broadcasts.  The ligand atoms are split across the compute warps (atom
// a = warp + W*k, kept in registers), the protein conformation is staged in
// shared memory in 128-point tiles by the TMA engine (cp.async.bulk +
// mbarrier), either once for the whole launch (resident) or through an
// 8-stage ring fed by a producer warp.  Per step each warp writes FP64 partial
// sums per replica; warp 0 reduces them, normalises the terms, and takes the
// Metropolis decision with the counter-based RNG.
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

constexpr int TAB_N = GD_NLT * GD_NPT;
constexpr int TAB_BYTES = TAB_N * (16 + 8);
constexpr int STAGE_BYTES = TILE_PTS * (16 + 8);
constexpr int CHUNK = 32;  // points per FP32 partial before the FP64 flush

size_t dock_smem_bytes(int n_warps, int n_stages) {
  return (size_t)TAB_BYTES + (size_t)n_stages * STAGE_BYTES +
         (size_t)n_warps * NRED * 32 * sizeof(double) + 32 * 36 * sizeof(float) +
         (size_t)2 * n_stages * sizeof(uint64_t);
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

struct Rot {
  float r00, r01, r02, r10, r11, r12, r20, r21, r22;
};

// Per-replica state in shared memory, written by warp 0 only.
struct LaneState {
  float m_old[6];
  float m_new[6];
  float rot[9];
  float tr[3];
  float e_old[GD_NTERM];
  float pad[2];
};

// ZYX Euler rotation of move_d.cu:90-105.
__device__ __forceinline__ Rot make_rot(float a3, float a4, float a5) {
  float s1, c1, s2, c2, s3, c3;
  sincosf(a3, &s1, &c1);
  sincosf(a4, &s2, &c2);
  sincosf(a5, &s3, &c3);
  Rot R;
  R.r00 = c1 * c2;
  R.r01 = c1 * s2 * s3 - c3 * s1;
  R.r02 = s1 * s3 + c1 * c3 * s2;
  R.r10 = c2 * s1;
  R.r11 = c1 * c3 + s1 * s2 * s3;
  R.r12 = c3 * s1 * s2 - c1 * s3;
  R.r20 = -1.0f * s2;
  R.r21 = c2 * s3;
  R.r22 = c2 * c3;
  return R;
}

template <int MODE>
__global__ void __launch_bounds__((MAX_WARPS + 1) * 32, 1)
    dock_kernel(const __grid_constant__ KTables T, const __grid_constant__ KRun R) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int W = R.n_warps;
  const int NS = R.n_stages;
  float4 *s_tab_a = reinterpret_cast<float4 *>(smem);
  float2 *s_tab_b = reinterpret_cast<float2 *>(smem + TAB_N * 16);
  unsigned char *s_tiles = smem + TAB_BYTES;
  double *s_red = reinterpret_cast<double *>(s_tiles + (size_t)NS * STAGE_BYTES);
  LaneState *s_lane = reinterpret_cast<LaneState *>(s_red + (size_t)W * NRED * 32);
  uint64_t *s_full = reinterpret_cast<uint64_t *>(s_lane + 32);
  uint64_t *s_empty = s_full + NS;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  // ---- work of this CTA --------------------------------------------------
  int rep0, n_act, prt_conf;
  if (MODE == KMODE_POSES) {
    rep0 = blockIdx.x * 32;
    n_act = min(32, R.n_pose - rep0);
    prt_conf = R.prt_conf;
  } else {
    rep0 = R.cta_rep0[blockIdx.x];
    n_act = R.cta_nrep[blockIdx.x];
    prt_conf = rep0 / (R.st.n_tmp * R.st.n_lig_conf);
  }
  const int n_tiles = (T.pnp + TILE_PTS - 1) / TILE_PTS;
  const bool resident = R.resident != 0;
  const int n_steps = (MODE == KMODE_REMC) ? R.n_steps : 1;
  const int passes = resident ? 1 : n_steps;

  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], W);
    }
    fence_barrier_init();
  }
  for (int i = threadIdx.x; i < TAB_N; i += blockDim.x) {
    s_tab_a[i] = T.tab_a[i];
    s_tab_b[i] = T.tab_b[i];
  }
  __syncthreads();

  // ---- producer warp: streams the protein conformation -------------------
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
  const int lna = T.lna;
  const bool active = lane < n_act;
  const int rep = rep0 + (active ? lane : 0);
  const int lig_conf = (MODE == KMODE_POSES) ? R.lig_conf : rep % R.st.n_lig_conf;
  const float4 *orig = T.lig + (size_t)lig_conf * lna;
  LaneState &me = s_lane[lane];

  // this warp's ligand atoms a = warp + W k
  int n_my = 0;
#pragma unroll
  for (int k = 0; k < MAX_APW; ++k)
    if (warp + W * k < lna) n_my = k + 1;

  // replica state lives in shared memory, owned by warp 0
  float mbeta = 0.f;
  int acs = 0, idx_tmp = 0;
  if (warp == 0) {
    if (MODE == KMODE_REMC) {
      idx_tmp = R.st.idx_tmp[rep];
      mbeta = R.st.minus_beta[idx_tmp];
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_old[i] = R.st.m_old[(size_t)rep * 6 + i];
#pragma unroll
      for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = R.st.e_old[(size_t)rep * GD_NTERM + i];
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_old[i] = 0.f;
#pragma unroll
      for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = 0.f;
    }
  }
  uint32_t k0 = 0, k1 = 0;
  rng_key(R.seed, R.stream_id, k0, k1);

  int it = 0;  // tile iteration counter (streaming ring position)
  for (int si = 0; si < n_steps; ++si) {
    const int step = R.step0 + si;

    // ---- warp 0 proposes the move and publishes it ---------------------------
    uint32_t u_acc_bits = 0;
    if (warp == 0) {
      float m_new[6];
      if (MODE == KMODE_REMC) {
        const U4 a = philox4x32_10(U4{(uint32_t)rep, (uint32_t)step, 0u, 0u}, k0, k1);
        const U4 b = philox4x32_10(U4{(uint32_t)rep, (uint32_t)step, 1u, 0u}, k0, k1);
        const uint32_t bits[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
        u_acc_bits = b.z;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const float pert = __fadd_rn(__fmul_rn(2.0f, u01(bits[i])), -1.0f);
          m_new[i] = __fadd_rn(__fmul_rn(R.move_scale[i], pert), me.m_old[i]);
        }
      } else if (MODE == KMODE_INIT) {
        const bool away = (R.flags & GD_MC_MOVE_AWAY) != 0;
#pragma unroll
        for (int i = 0; i < 6; ++i)
          m_new[i] = away ? __fadd_rn(__fmul_rn(R.move_scale[i], 44.5f), 0.0f) : 0.0f;
      } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) m_new[i] = active ? R.poses[(size_t)rep * 6 + i] : 0.f;
      }
      const Rot rot = make_rot(m_new[3], m_new[4], m_new[5]);
#pragma unroll
      for (int i = 0; i < 6; ++i) me.m_new[i] = m_new[i];
      me.rot[0] = rot.r00; me.rot[1] = rot.r01; me.rot[2] = rot.r02;
      me.rot[3] = rot.r10; me.rot[4] = rot.r11; me.rot[5] = rot.r12;
      me.rot[6] = rot.r20; me.rot[7] = rot.r21; me.rot[8] = rot.r22;
      // translation applied after the rotation: m + ligand centre
      me.tr[0] = m_new[0];
      me.tr[1] = m_new[1];
      me.tr[2] = m_new[2];
    }
    named_sync(1, W * 32);

    // ---- place this warp's atoms --------------------------------------------
    const float q00 = me.rot[0], q01 = me.rot[1], q02 = me.rot[2];
    const float q10 = me.rot[3], q11 = me.rot[4], q12 = me.rot[5];
    const float q20 = me.rot[6], q21 = me.rot[7], q22 = me.rot[8];
    const float t0 = me.tr[0], t1 = me.tr[1], t2 = me.tr[2];
    float lx[MAX_APW], ly[MAX_APW], lz[MAX_APW], hpc[MAX_APW];
#pragma unroll
    for (int k = 0; k < MAX_APW; ++k) {
      lx[k] = ly[k] = lz[k] = hpc[k] = 0.f;
      if (k < n_my) {
        const float4 o = orig[warp + W * k];
        lx[k] = q00 * o.x + q01 * o.y + q02 * o.z + t0 + T.lig_center[0];
        ly[k] = q10 * o.x + q11 * o.y + q12 * o.z + t1 + T.lig_center[1];
        lz[k] = q20 * o.x + q21 * o.y + q22 * o.z + t2 + T.lig_center[2];
      }
    }

    // ---- pair terms over the protein tiles -----------------------------------
    double dvdw = 0.0, dele = 0.0, dpmf = 0.0, dpsp = 0.0, dhdb = 0.0;
    for (int t = 0; t < n_tiles; ++t, ++it) {
      const int s = resident ? t : (it % NS);
      const uint32_t ph = resident ? 0u : (uint32_t)((it / NS) & 1);
      mbar_wait(&s_full[s], ph, R.err, 2);
      const float4 *ta = reinterpret_cast<const float4 *>(s_tiles + (size_t)s * STAGE_BYTES);
      const float2 *tb =
          reinterpret_cast<const float2 *>(s_tiles + (size_t)s * STAGE_BYTES + TILE_PTS * 16);
      const int nvalid = min(TILE_PTS, T.pnp - t * TILE_PTS);
      for (int j0 = 0; j0 < nvalid; j0 += CHUNK) {
        const int j1 = min(nvalid, j0 + CHUNK);
        float fvdw = 0.f, fele = 0.f, fpmf = 0.f, fpsp = 0.f, fhdb = 0.f;
        for (int j = j0; j < j1; ++j) {
          const float4 A = ta[j];
          const float2 B = tb[j];
          const uint32_t meta = __float_as_uint(B.y);
          const int pt = (int)(meta & META_TYPE_MASK);
          const bool is_c2 = ((meta >> META_CLASS_SHIFT) & 3u) == 2u;
          const bool hflag = (meta & META_HPC_BIT) != 0u;
#pragma unroll
          for (int k = 0; k < MAX_APW; ++k) {
            if (k < n_my) {
              const int lt = T.lig_t[warp + W * k];
              const float4 P = s_tab_a[lt * GD_NPT + pt];  // p1a p2a pmf0 pmf1
              const float2 H = s_tab_b[lt * GD_NPT + pt];  // hdb0 hdb1
              const float dx = lx[k] - A.x;
              const float dy = ly[k] - A.y;
              const float dz = lz[k] - A.z;
              const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
              const float r = rsqrtf(d2);
              const float d = d2 * r;
              // hydrophobic contact (per ligand atom)
              if (hflag) {
                if (d2 <= 81.0f) hpc[k] = fmaf(B.x, hpc_poly(d2), hpc[k]);
              }
              // soft Lennard-Jones: p1 = p1a/d^9, p2 = p2a/d^6
              const float r2 = r * r;
              const float r6 = r2 * r2 * r2;
              const float r9 = r6 * r2 * r;
              const float p1 = P.x * r9;
              const float p2 = P.y * r6;
              const float p4 = fmaf(p1, fmaf(T.lj0lj1, d2, T.lj0), 1.0f);
              fvdw += __fdividef(p1 - p2, p4);
              // soft electrostatics
              const float s1 = T.el1 * d;
              const float g = (s1 < 1.0f) ? fmaf(s1 * s1, fmaf(T.b1, s1, T.a1), T.el0)
                                          : r * T.inv_el1;
              fele = fmaf(T.lig_q[warp + W * k] * A.w, g, fele);
              // contact PMF
              const float dm = d - P.z;
              const float ex = __expf(fmaf(-0.5f, d, 6.0f) * dm);
              fpmf += __fdividef(P.w, 1.0f + ex);
              // pocket-specific potential
              if (is_c2) {
                const bool hit = dm <= 0.0f;
                if (__any_sync(0xffffffffu, hit)) {
                  const float v =
                      __ldg(&T.psp[(size_t)lt * T.psp_ncol + (meta >> META_SEQ_SHIFT)]);
                  if (hit) fpsp += v;
                }
              }
              // hydrogen bond
              if (H.x > 0.1f) {
                const float h3 = (d - H.x) * H.y;
                fhdb = fmaf(H.y, __expf(-0.5f * h3 * h3), fhdb);
              }
            }
          }
        }
        dvdw += (double)fvdw;
        dele += (double)fele;
        dpmf += (double)fpmf;
        dpsp += (double)fpsp;
        dhdb += (double)fhdb;
      }
      if (!resident) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_empty[s]);
      }
    }

    // ---- hydrophobic restraint per atom, KDE --------------------------------
    double dhpc = 0.0, dkde = 0.0, dlhm = 0.0;
#pragma unroll
    for (int k = 0; k < MAX_APW; ++k) {
      if (k < n_my) {
        const int lt = T.lig_t[warp + W * k];
        const float h = __fdiv_rn(__fsub_rn(hpc[k], T.hpl0[lt]), T.hpl1[lt]);
        dhpc += (double)__fsub_rn(__fmul_rn(__fmul_rn(0.5f, h), h), T.hpl2[lt]);
        const int kb = T.kde_off[lt], ke = T.kde_off[lt + 1];
        if (ke > kb) {
          float kv = 0.f;
          for (int q = kb; q < ke; ++q) {
            const float4 K = T.kde[q];
            const float dx = lx[k] - K.x, dy = ly[k] - K.y, dz = lz[k] - K.z;
            kv += __expf(T.kde2 * fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
          }
          dkde += (double)kv / (double)(ke - kb);
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
          const float x = q00 * o.x + q01 * o.y + q02 * o.z + t0 + T.lig_center[0];
          const float y = q10 * o.x + q11 * o.y + q12 * o.z + t1 + T.lig_center[1];
          const float z = q20 * o.x + q21 * o.y + q22 * o.z + t2 + T.lig_center[2];
          const float dx = x - M.x, dy = y - M.y, dz = z - M.z;
          sv += fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        }
      }
      dlhm += (double)T.mcs_tcc[m] * sqrt((double)sv / (double)T.mcs_cnt[m]);
    }

    // ---- cross-warp reduction and finalisation (warp 0) ----------------------
    {
      double *red = s_red + (size_t)warp * NRED * 32;
      red[0 * 32 + lane] = dvdw;
      red[1 * 32 + lane] = dele;
      red[2 * 32 + lane] = dpmf;
      red[3 * 32 + lane] = dpsp;
      red[4 * 32 + lane] = dhdb;
      red[5 * 32 + lane] = dhpc;
      red[6 * 32 + lane] = dkde;
      red[7 * 32 + lane] = dlhm;
    }
    named_sync(1, W * 32);
    if (warp == 0) {
      double S[NRED];
#pragma unroll
      for (int i = 0; i < NRED; ++i) S[i] = 0.0;
      for (int w = 0; w < W; ++w) {
        const double *red = s_red + (size_t)w * NRED * 32;
#pragma unroll
        for (int i = 0; i < NRED; ++i) S[i] += red[i * 32 + lane];
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
        const float cx = __fadd_rn(T.lig_center[0], me.m_new[0]);
        const float cy = __fadd_rn(T.lig_center[1], me.m_new[1]);
        const float cz = __fadd_rn(T.lig_center[2], me.m_new[2]);
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
          acc = metropolis(e[9], me.e_old[9], mbeta, u01(u_acc_bits));
          if (active && R.st.record && step < R.st.rec_steps) {
            gd_record *rc = R.st.record + (size_t)rep * R.st.rec_steps + step;
            const int nl = R.st.n_lig_conf, nt = R.st.n_tmp;
            rc->idx_rep = rep;
            rc->idx_prt = rep / (nt * nl);
            rc->idx_tmp = idx_tmp;
            rc->idx_lig = rep % nl;
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
          acs += 1;
#pragma unroll
          for (int i = 0; i < GD_NTERM; ++i) me.e_old[i] = e[i];
#pragma unroll
          for (int i = 0; i < 6; ++i) me.m_old[i] = me.m_new[i];
        }
      }
    }
    // the next iteration's first barrier orders warp 0's updates before any
    // other warp reads the lane state again
  }

  // ---- write the replica state back ----------------------------------------
  if (MODE != KMODE_POSES && warp == 0 && active) {
#pragma unroll
    for (int i = 0; i < 6; ++i) R.st.m_old[(size_t)rep * 6 + i] = me.m_old[i];
#pragma unroll
    for (int i = 0; i < GD_NTERM; ++i) R.st.e_old[(size_t)rep * GD_NTERM + i] = me.e_old[i];
    if (MODE == KMODE_INIT) {
      R.st.acs_mc[rep] = 0;
      R.st.idx_tmp[rep] = (rep / R.st.n_lig_conf) % R.st.n_tmp;
    } else {
      R.st.acs_mc[rep] += acs;
    }
  }
}

// Temperature exchange, one thread per (protein conf, ligand conf) group
// (exchangereplicas_d.cu:26-79).  Pairs of adjacent temperature indices
// (2 pair + mode_t, 2 pair + mode_t + 1) swap their slots when
// exp((mb1 - mb2)(E2 - E1)) > u; the counters are kept per slot.
__global__ void exchange_kernel(KState S, int n_prt, int n_lig, uint64_t seed, uint32_t stream,
                                int round, int mode_t) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_prt * n_lig) return;
  const int p = g / n_lig, l = g % n_lig;
  const int nt = S.n_tmp;
  int temps[MAX_TMP], orders[MAX_TMP];
  float en[MAX_TMP];
  for (int t = 0; t < nt; ++t) {
    const int r = nt * n_lig * p + n_lig * t + l;
    temps[t] = S.idx_tmp[r];
    en[t] = S.e_old[(size_t)r * GD_NTERM + GD_E_TOTAL];
  }
  for (int t = 0; t < nt; ++t) orders[temps[t]] = t;
  uint32_t k0, k1;
  rng_key(seed, stream, k0, k1);
  const int maxpair = nt / 2 - (nt % 2 == 0) * (mode_t == 1);
  for (int pair = 0; pair < maxpair; ++pair) {
    const int i1 = (pair << 1) + mode_t;
    const int i2 = i1 + 1;
    const int o1 = orders[i1], o2 = orders[i2];
    const int tt = temps[o1];
    const float mb1 = S.minus_beta[temps[o1]];
    const float mb2 = S.minus_beta[temps[o2]];
    const float delta = __fmul_rn(__fsub_rn(mb1, mb2), __fsub_rn(en[o2], en[o1]));
    const float prob = decision_expf(delta);
    const U4 o = philox4x32_10(U4{(uint32_t)g, (uint32_t)round, 2u, (uint32_t)pair}, k0, k1);
    if (prob > u01(o.x)) {
      temps[o1] = temps[o2];
      temps[o2] = tt;
      atomicAdd(&S.acs_exchg[o1], 1);
      atomicAdd(&S.acs_exchg[o2], 1);
    }
  }
  for (int t = 0; t < nt; ++t) S.idx_tmp[nt * n_lig * p + n_lig * t + l] = temps[t];
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
cudaError_t launch_dock(const KTables &T, const KRun &R, int grid, cudaStream_t s) {
  const size_t smem = dock_smem_bytes(R.n_warps, R.n_stages);
  const int threads = (R.n_warps + 1) * 32;
  cudaError_t e;
  switch (R.mode) {
    case KMODE_POSES:
      e = cudaFuncSetAttribute(dock_kernel<KMODE_POSES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e != cudaSuccess) return e;
      dock_kernel<KMODE_POSES><<<grid, threads, smem, s>>>(T, R);
      break;
    case KMODE_REMC:
      e = cudaFuncSetAttribute(dock_kernel<KMODE_REMC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e != cudaSuccess) return e;
      dock_kernel<KMODE_REMC><<<grid, threads, smem, s>>>(T, R);
      break;
    default:
      e = cudaFuncSetAttribute(dock_kernel<KMODE_INIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e != cudaSuccess) return e;
      dock_kernel<KMODE_INIT><<<grid, threads, smem, s>>>(T, R);
      break;
  }
  return cudaGetLastError();
}

cudaError_t launch_exchange(const KState &S, int n_prt, int n_lig, uint64_t seed,
                            uint32_t stream_id, int round, int mode_t, cudaStream_t s) {
  const int n = n_prt * n_lig;
  exchange_kernel<<<(n + 127) / 128, 128, 0, s>>>(S, n_prt, n_lig, seed, stream_id, round, mode_t);
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
