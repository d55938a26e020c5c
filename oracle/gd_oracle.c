/*
 * gd_oracle.c -- CPU oracle of the REMC docking path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (gpudock_b200/ and its
 * libgpudock.so) links, loads or calls this file; only tests/, the smoke
 * check and the bench's CPU-baseline leg do, as the checker.
 *
 * It restates, in plain C, the semantics of the reference GPU kernels of
 * gpudocksm-rem-1.2 (GeauxDock):
 *   energy      src/calcenergy_d.cu:22-374  (per-pair math in FP32, in the
 *               reference's operation order; every sum accumulated in FP64)
 *   move        src/move_d.cu:11-133
 *   accept      src/accept_d.cu:12-52
 *   MC driver   src/montecarlo_d.cu:12-104, src/gpusingle.cu:5-37
 *   exchange    src/exchangereplicas_d.cu:26-79
 *   tables      src/util.C:405-458 (OptimizeEnepara), :491-532
 *               (SetTemperature)
 * The reference draws its random numbers from a time-seeded XORWOW (curand),
 * which no run can reproduce; this build replaces it by Philox4x32-10
 * (Salmon et al., SC'11) keyed as documented below, restated here
 * independently of the device code, together with the decision exp.
 *
 * Build with -ffp-contract=off so that no a*b+c is fused behind our back;
 * every fused multiply-add below is an explicit fmaf().
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/gpudock.h"

#define ORC_PI 3.1415926535f /* size.h:86 */

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as   */
/* easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with the  */
/* published multipliers and Weyl key increments.                           */
/* ------------------------------------------------------------------------ */
#define PH_M0 0xD2511F53u
#define PH_M1 0xCD9E8D57u
#define PH_W0 0x9E3779B9u
#define PH_W1 0xBB67AE85u

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)PH_M0 * c0;
    uint64_t p1 = (uint64_t)PH_M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += PH_W0;
    k1 += PH_W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform float in [0, 1) with 24 random bits. */
static inline float orc_u01(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

/* Key and counters of the random stream (identical on the device):
 *   key  = { seed_lo, seed_hi ^ stream_id }
 *   move of replica r at MC step s:   ctr {r, s, 0, 0} -> 4 perturbations
 *                                      ctr {r, s, 1, 0} -> 2 perturbations,
 *                                                          word 2 = accept u
 *   exchange round k of group g, pair j: ctr {g, k, 2, j} -> word 0        */
static inline void orc_key(uint64_t seed, uint32_t stream, uint32_t key[2])
{
  key[0] = (uint32_t)seed;
  key[1] = (uint32_t)(seed >> 32) ^ stream;
}

/* ------------------------------------------------------------------------ */
/* Decision exp: Cody-Waite range reduction (Cody & Waite 1980) with ln 2    */
/* split into a 16-bit head and a tail, then the degree-7 Taylor polynomial  */
/* of e^r on |r| <= ln2/2 in Horner form, then scaling by 2^k in two exact    */
/* steps.  Every step is an IEEE single operation or an explicit fmaf, so    */
/* the device copy returns the same bits.                                   */
/* ------------------------------------------------------------------------ */
float orc_expf(float x)
{
  if (x != x) return x;
  if (x > 88.72f) return INFINITY;
  if (x < -87.33f) return 0.0f;
  const float kf = rintf(x * 0x1.715476p+0f);
  float r = fmaf(-kf, 0x1.62e400p-1f, x);
  r = fmaf(-kf, 0x1.7f7d1cp-20f, r);
  float p = 0x1.a01a02p-13f;
  p = fmaf(p, r, 0x1.6c16c2p-10f);
  p = fmaf(p, r, 0x1.111112p-7f);
  p = fmaf(p, r, 0x1.555556p-5f);
  p = fmaf(p, r, 0x1.555556p-3f);
  p = fmaf(p, r, 0x1.0p-1f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  const int k = (int)kf;
  const int k1 = k / 2, k2 = k - k1;
  union { uint32_t u; float f; } s1, s2;
  s1.u = (uint32_t)(k1 + 127) << 23;
  s2.u = (uint32_t)(k2 + 127) << 23;
  return (p * s1.f) * s2.f;
}

/* Metropolis rule of accept_d.cu:19-23 on given energies and uniform. */
int orc_metropolis(float e_new, float e_old, float minus_beta, uint64_t seed,
                   uint32_t stream, int rep, int step)
{
  uint32_t key[2], ctr[4] = {(uint32_t)rep, (uint32_t)step, 1u, 0u}, o[4];
  orc_key(seed, stream, key);
  orc_philox(ctr, key, o);
  const float de = e_new - e_old;
  return orc_u01(o[2]) < orc_expf(de * minus_beta);
}

/* ------------------------------------------------------------------------ */
/* Parameter tables                                                         */
/* ------------------------------------------------------------------------ */
/* OptimizeEnepara, util.C:405-458. */
void orc_enepara_optimize(const gd_enepara_raw *r, gd_enepara *e)
{
  const float sqrt_2_pi = sqrtf(2.0f * ORC_PI);
  memset(e, 0, sizeof(*e));
  for (int i = 0; i < GD_NLT; ++i)
    for (int j = 0; j < GD_NPT; ++j) {
      const float tmp = r->vdw[j][i][0] * r->lj[2];
      e->p1a[i][j] = 2.0f * r->vdw[j][i][1] * powf(tmp, 9.0f);
      e->p2a[i][j] = 3.0f * r->vdw[j][i][1] * powf(tmp, 6.0f);
    }
  e->lj0 = r->lj[0];
  e->lj1 = r->lj[1];
  e->el0 = r->el[0];
  e->a1 = 4.0f - 3.0f * r->el[0];
  e->b1 = 2.0f * r->el[0] - 3.0f;
  e->el1 = r->el[1];
  for (int i = 0; i < GD_NELE; ++i) e->ele[i] = r->ele[i];
  for (int i = 0; i < GD_NLT; ++i)
    for (int j = 0; j < GD_NPT; ++j) {
      e->pmf0[i][j] = r->pmf[j][i][0];
      e->pmf1[i][j] = r->pmf[j][i][1];
      e->hdb0[i][j] = r->hdb[j][i][0];
      e->hdb1[i][j] = 1.0f / r->hdb[j][i][1];
      e->hdb2[i][j] = -1.0f / (r->hdb[j][i][1] * sqrt_2_pi);
    }
  for (int i = 0; i < GD_NRES; ++i) e->hpp[i] = r->hpp[i];
  for (int i = 0; i < GD_NLT; ++i) {
    e->hpl0[i] = r->hpl[i][0];
    e->hpl1[i] = r->hpl[i][1];
    e->hpl2[i] = logf(1.0f / (e->hpl1[i] * sqrt_2_pi));
  }
  e->kde2 = -0.5f / (r->kde * r->kde);
  e->kde3 = powf(r->kde * sqrt_2_pi, 3.0f);
  for (int i = 0; i < GD_NTERM; ++i) {
    e->w[i] = r->w[i];
    e->a_para[i] = r->a_para[i];
    e->b_para[i] = r->b_para[i];
  }
}

/* SetTemperature, util.C:491-532 (k_B = 1). */
void orc_set_temperature(int n, float floor_t, float ceil_t, float *temps,
                         float *minus_beta)
{
  if (n == 1) {
    const float beta = 1.0f / (1.0f * floor_t);
    if (temps) temps[0] = floor_t;
    minus_beta[0] = 0.0f - beta;
    return;
  }
  const float ratio = expf(logf(ceil_t / floor_t) / (float)(n - 1));
  float a = floor_t;
  for (int i = 0; i < n; ++i) {
    const float beta = 1.0f / (1.0f * a);
    if (temps) temps[i] = a;
    minus_beta[i] = 0.0f - beta;
    a *= ratio;
  }
}

/* ------------------------------------------------------------------------ */
/* Move (move_d.cu:74-133) and MoveAway (move_d.cu:11-69)                   */
/* ------------------------------------------------------------------------ */
static void orc_place(const gd_complex *cx, int lig_conf, const float m[6],
                      float *x, float *y, float *z, float center[3])
{
  const gd_ligand *lg = &cx->lig;
  const float s1 = sinf(m[3]), c1 = cosf(m[3]);
  const float s2 = sinf(m[4]), c2 = cosf(m[4]);
  const float s3 = sinf(m[5]), c3 = cosf(m[5]);
  float rot[3][3];
  rot[0][0] = c1 * c2;
  rot[0][1] = c1 * s2 * s3 - c3 * s1;
  rot[0][2] = s1 * s3 + c1 * c3 * s2;
  rot[1][0] = c2 * s1;
  rot[1][1] = c1 * c3 + s1 * s2 * s3;
  rot[1][2] = c3 * s1 * s2 - c1 * s3;
  rot[2][0] = -1 * s2;
  rot[2][1] = c2 * s3;
  rot[2][2] = c2 * c3;
  const float cxx = lg->center[0], cyy = lg->center[1], czz = lg->center[2];
  const size_t off = (size_t)lig_conf * lg->lna;
  for (int l = 0; l < lg->lna; ++l) {
    const float ox = lg->x[off + l], oy = lg->y[off + l], oz = lg->z[off + l];
    x[l] = rot[0][0] * ox + rot[0][1] * oy + rot[0][2] * oz + m[0] + cxx;
    y[l] = rot[1][0] * ox + rot[1][1] * oy + rot[1][2] * oz + m[1] + cyy;
    z[l] = rot[2][0] * ox + rot[2][1] * oy + rot[2][2] * oz + m[2] + czz;
  }
  for (int i = 0; i < 3; ++i) center[i] = lg->center[i] + m[i];
}

/* ------------------------------------------------------------------------ */
/* Energy of placed coordinates (calcenergy_d.cu:22-374)                    */
/* raw[9]: un-normalised terms in FP64; terms[10]: normalised + total, FP32 */
/* abs_sum[5] (optional): sums of |contribution| of vdw, ele, pmf, psp, hdb */
/* after the same division, for a cancellation-aware tolerance.             */
/* ------------------------------------------------------------------------ */
void orc_energy_coords(const gd_complex *cx, int prt_conf, const float *lx,
                       const float *ly, const float *lz, const float center[3],
                       double raw[GD_NRAW], float terms[GD_NTERM],
                       double abs_sum[5])
{
  const gd_ligand *lg = &cx->lig;
  const gd_protein *pr = &cx->prt;
  const gd_enepara *ff = cx->ff;
  const int lna = lg->lna, pnp = pr->pnp;
  const size_t po = (size_t)prt_conf * pnp;
  const float *px = pr->x + po, *py = pr->y + po, *pz = pr->z + po;

  double evdw = 0, eele = 0, epmf = 0, epsp = 0, ehdb = 0, ehpc = 0;
  double avdw = 0, aele = 0, apmf = 0, apsp = 0, ahdb = 0;
  for (int l = 0; l < lna; ++l) {
    const int lt = lg->t[l];
    const float lc = lg->c[l];
    double hpc_sum = 0.0;
    for (int p = 0; p < pnp; ++p) {
      const int pt = pr->t[p];
      const float dx = lx[l] - px[p];
      const float dy = ly[l] - py[p];
      const float dz = lz[l] - pz[p];
      const float dst_pow2 = dx * dx + dy * dy + dz * dz;
      const float dst_pow4 = dst_pow2 * dst_pow2;
      const float dst = sqrtf(dst_pow2);

      if (pr->c0_and_d12_or_c2[p] == 1 && dst_pow2 <= 81.0f) {
        hpc_sum += (double)(pr->hpp[p] *
                            (1.0f - (3.5f / 81.0f * dst_pow2 -
                                     4.5f / 81.0f / 81.0f * dst_pow4 +
                                     2.5f / 81.0f / 81.0f / 81.0f * dst_pow4 * dst_pow2 -
                                     0.5f / 81.0f / 81.0f / 81.0f / 81.0f * dst_pow4 * dst_pow4)));
      }

      const float p1 = ff->p1a[lt][pt] / (dst_pow4 * dst_pow4 * dst);
      const float p2 = ff->p2a[lt][pt] / (dst_pow4 * dst_pow2);
      const float p4 = p1 * ff->lj0 * (1.0f + ff->lj1 * dst_pow2) + 1.0f;
      const float vdw = (p1 - p2) / p4;
      evdw += vdw;
      avdw += fabs((double)vdw);

      const float s1 = ff->el1 * dst;
      float g1;
      if (s1 < 1)
        g1 = ff->el0 + ff->a1 * s1 * s1 + ff->b1 * s1 * s1 * s1;
      else
        g1 = 1.0f / s1;
      const float ele = lc * pr->ele[p] * g1;
      eele += ele;
      aele += fabs((double)ele);

      const float dst_minus_pmf0 = dst - ff->pmf0[lt][pt];
      const float pmf = ff->pmf1[lt][pt] /
                        (1.0f + expf((-0.5f * dst + 6.0f) * dst_minus_pmf0));
      epmf += pmf;
      apmf += fabs((double)pmf);

      if (pr->c[p] == 2 && dst_minus_pmf0 <= 0) {
        const float v = cx->psp.psp[(size_t)lt * cx->psp.n_col + pr->seq3r[p]];
        epsp += v;
        apsp += fabs((double)v);
      }

      const float hdb0 = ff->hdb0[lt][pt];
      if (hdb0 > 0.1f) {
        const float hdb1 = ff->hdb1[lt][pt];
        const float hdb3 = (dst - hdb0) * hdb1;
        const float h = hdb1 * expf(-0.5f * hdb3 * hdb3);
        ehdb += h;
        ahdb += fabs((double)h);
      }
    }
    /* hydrophobic restraint per ligand atom, calcenergy_d.cu:143-149 */
    const float hsum = (float)hpc_sum;
    const float hpc2 = (hsum - ff->hpl0[lt]) / ff->hpl1[lt];
    ehpc += (double)(0.5f * hpc2 * hpc2 - ff->hpl2[lt]);
  }

  /* KDE, calcenergy_d.cu:175-213 */
  double ekde = 0.0;
  for (int l = 0; l < lna; ++l) {
    double kv = 0.0;
    int kn = 0;
    for (int k = 0; k < cx->kde.pnk; ++k) {
      if (lg->t[l] == cx->kde.t[k]) {
        const float dx = lx[l] - cx->kde.x[k];
        const float dy = ly[l] - cx->kde.y[k];
        const float dz = lz[l] - cx->kde.z[k];
        const float d2 = dx * dx + dy * dy + dz * dz;
        kv += (double)expf(ff->kde2 * d2);
        kn += 1;
      }
    }
    if (kn != 0) ekde += kv / (double)kn;
  }

  /* LHM position restraints, calcenergy_d.cu:229-271 */
  double elhm = 0.0;
  for (int m = 0; m < cx->mcs.pos; ++m) {
    double sv = 0.0;
    int sn = 0;
    const size_t mo = (size_t)m * cx->mcs.n_field;
    for (int l = 0; l < lna; ++l) {
      const int f = lg->n[l] + 1;
      if (cx->mcs.x[mo + f] != GD_MCS_INVALID_COORD) {
        const float dx = lx[l] - cx->mcs.x[mo + f];
        const float dy = ly[l] - cx->mcs.y[mo + f];
        const float dz = lz[l] - cx->mcs.z[mo + f];
        sv += (double)(dx * dx + dy * dy + dz * dz);
        sn += 1;
      }
    }
    /* sn == 0 gives 0/0 = NaN, as the reference does */
    elhm += (double)cx->mcs.tcc[m] * sqrt(sv / (double)sn);
  }

  /* distance to the pocket, calcenergy_d.cu:278-283 */
  const float ddx = center[0] - pr->pocket_center[0];
  const float ddy = center[1] - pr->pocket_center[1];
  const float ddz = center[2] - pr->pocket_center[2];
  const float edst = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);

  const double n = (double)lna;
  const double s2pi = (double)sqrtf(2.0f * ORC_PI);
  raw[0] = evdw / n;
  raw[1] = eele / n;
  raw[2] = epmf / n;
  raw[3] = epsp / n;
  raw[4] = -(ehdb / n / s2pi);
  raw[5] = ehpc / n;
  raw[6] = ekde / (double)ff->kde3 / n;
  raw[7] = log(elhm / (double)cx->mcs.pos);
  raw[8] = (double)edst;
  if (abs_sum) {
    abs_sum[0] = avdw / n;
    abs_sum[1] = aele / n;
    abs_sum[2] = apmf / n;
    abs_sum[3] = apsp / n;
    abs_sum[4] = ahdb / n / s2pi;
  }

  /* normalisation a*e+b and weighted total, calcenergy_d.cu:301-358 */
  float e[GD_NTERM];
  for (int i = 0; i < 9; ++i)
    e[i] = ff->a_para[i] * (float)raw[i] + ff->b_para[i];
  e[9] = ff->w[0] * e[0] + ff->w[1] * e[1] + ff->w[2] * e[2] +
         ff->w[3] * e[3] + ff->w[4] * e[4] + ff->w[5] * e[5] +
         ff->w[6] * e[6] + ff->w[7] * e[7] + ff->w[8] * e[8];
  for (int i = 0; i < GD_NTERM; ++i) terms[i] = e[i];
}

/* Bayesian total of IS_BAYE (calcenergy_d.cu:311-347): densities of
 * util_d.cu:220-290 (NormPdf, CauchyPdf, LogisticPdf, WaldPdf) with the
 * parameters of distribution.h, in the reference's float expressions and
 * pairings (low H-bond: normal density, "logistic" parameters; low PSP:
 * logistic density, "Laplace" parameters); libm's expf/powf/sqrtf/log10f. */
static const float kBayesPI = 3.1415926535f; /* PI of size.h */

static float bayes_norm(float x, float loc, float scale)
{
  const float norm_para = 1.0f / (scale * sqrtf(2.0f * kBayesPI));
  const float prob = expf(0.0f - (x - loc) * (x - loc) / (2.0f * scale * scale));
  return norm_para * prob;
}

static float bayes_cauchy(float x, float loc, float scale)
{
  const float norm_para = 1.0f / (kBayesPI * scale);
  const float prob = 1.0f / (1.0f + ((x - loc) / scale) * ((x - loc) / scale));
  return norm_para * prob;
}

static float bayes_logistic(float x, float loc, float scale)
{
  const float norm_para = 1.0f / scale;
  const float e_power = expf(-(x - loc) / scale);
  const float prob = e_power / powf(1.0f + e_power, 2.0f);
  return norm_para * prob;
}

static float bayes_wald(float x, float loc, float scale)
{
  const float normed_x = (x - loc) / scale;
  if (normed_x < 0.0f) return 0.00000001f;
  const float norm_para = 1.0f / (sqrtf(2.0f * kBayesPI * powf(normed_x, 3.0f)) * scale);
  const float prob = expf(-powf(normed_x - 1.0f, 2.0f) / (2.0f * normed_x));
  return norm_para * prob;
}

/* e: the nine normalised terms (vdw ele pmf psp hdb hpc kde lhm dst) */
float orc_bayes_total(const float *e)
{
  const float vdw = e[0], ele = e[1], pmf = e[2], psp = e[3], hdb = e[4];
  const float hpc = e[5], kde = e[6], lhm = e[7], dst = e[8];
  const float prob_h =
      log10f(bayes_norm(vdw, 0.05286683f, 0.29916642f)) +
      log10f(bayes_cauchy(ele, -0.3653806f, 0.00681102f)) +
      log10f(bayes_logistic(pmf, -0.0221777f, 0.11847532f)) +
      log10f(bayes_wald(hpc, -1.0041231f, 0.1151713f)) +
      log10f(bayes_norm(hdb, 0.60986808f, 0.30974999f)) +
      log10f(bayes_logistic(dst, -0.8246522f, 0.05218529f)) +
      log10f(bayes_logistic(psp, -0.2346999f, 0.09871713f)) +
      log10f(bayes_wald(kde, -1.0112055f, 0.09882933f)) +
      log10f(bayes_logistic(lhm, -0.3377100f, 0.09282947f));
  const float prob_l =
      log10f(bayes_norm(vdw, 0.15818486f, 0.29032471f)) +
      log10f(bayes_cauchy(ele, -0.3647824f, 0.00534225f)) +
      log10f(bayes_logistic(pmf, 0.04257942f, 0.08801551f)) +
      log10f(bayes_wald(hpc, -1.0019512f, 0.10312611f)) +
      log10f(bayes_norm(hdb, 0.76967708f, 0.11224029f)) +
      log10f(bayes_logistic(dst, -0.7509618f, 0.08757299f)) +
      log10f(bayes_logistic(psp, -0.2022064f, 0.07854212f)) +
      log10f(bayes_wald(kde, -1.004605f, 0.02967548f)) +
      log10f(bayes_logistic(lhm, -0.2387023f, 0.12134983f));
  return prob_l - prob_h;
}

/* Energy of one pose (move vector) of ligand conformation lig_conf. */
void orc_energy_pose(const gd_complex *cx, int prt_conf, int lig_conf,
                     const float m[6], double raw[GD_NRAW],
                     float terms[GD_NTERM], double abs_sum[5])
{
  const int lna = cx->lig.lna;
  float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
  float center[3];
  orc_place(cx, lig_conf, m, buf, buf + lna, buf + 2 * lna, center);
  orc_energy_coords(cx, prt_conf, buf, buf + lna, buf + 2 * lna, center, raw,
                    terms, abs_sum);
  free(buf);
}

/* Batch of poses, OpenMP over poses. */
void orc_energy_poses(const gd_complex *cx, int prt_conf, int lig_conf, int n,
                      const float *poses, float *terms, double *raw,
                      double *abs_sum, int n_threads)
{
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
  for (int i = 0; i < n; ++i) {
    double r[GD_NRAW], a[5];
    orc_energy_pose(cx, prt_conf, lig_conf, poses + 6 * (size_t)i, r,
                    terms + (size_t)GD_NTERM * i, a);
    if (raw) memcpy(raw + (size_t)GD_NRAW * i, r, sizeof(r));
    if (abs_sum) memcpy(abs_sum + (size_t)5 * i, a, sizeof(a));
  }
}

/* ------------------------------------------------------------------------ */
/* Contact-map MCC (calcmcc_d.cu): InitRefMatrix_d :57-83, CalcMcc_d        */
/* :148-213.  ref[l * pnp + p] = 1 where dst <= pmf0 for ligand conformation */
/* 0 in its start pose against protein conformation prt_conf.               */
/* ------------------------------------------------------------------------ */
static void orc_contacts(const gd_complex *cx, int prt_conf, const float *lx,
                         const float *ly, const float *lz, unsigned char *out)
{
  const gd_protein *pr = &cx->prt;
  const int pnp = pr->pnp;
  for (int l = 0; l < cx->lig.lna; ++l) {
    const int lt = cx->lig.t[l];
    for (int p = 0; p < pnp; ++p) {
      const size_t i = (size_t)prt_conf * pnp + p;
      const float dx = lx[l] - pr->x[i];
      const float dy = ly[l] - pr->y[i];
      const float dz = lz[l] - pr->z[i];
      const float dst = sqrtf(dx * dx + dy * dy + dz * dz);
      out[(size_t)l * pnp + p] = dst <= cx->ff->pmf0[lt][pr->t[p]];
    }
  }
}

static unsigned char *orc_mcc_ref(const gd_complex *cx, int prt_conf, int *nref)
{
  const int lna = cx->lig.lna;
  unsigned char *ref = (unsigned char *)malloc((size_t)lna * cx->prt.pnp);
  float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
  for (int l = 0; l < lna; ++l) {
    buf[l] = cx->lig.x[l] + cx->lig.center[0];
    buf[lna + l] = cx->lig.y[l] + cx->lig.center[1];
    buf[2 * lna + l] = cx->lig.z[l] + cx->lig.center[2];
  }
  orc_contacts(cx, prt_conf, buf, buf + lna, buf + 2 * lna, ref);
  int n = 0;
  for (size_t i = 0; i < (size_t)lna * cx->prt.pnp; ++i) n += ref[i];
  *nref = n;
  free(buf);
  return ref;
}

static float orc_mcc_of(const gd_complex *cx, int prt_conf, const float *lx,
                        const float *ly, const float *lz,
                        const unsigned char *ref)
{
  const size_t n = (size_t)cx->lig.lna * cx->prt.pnp;
  unsigned char *cur = (unsigned char *)malloc(n);
  orc_contacts(cx, prt_conf, lx, ly, lz, cur);
  int tp = 0, fn = 0, fpc = 0, tn = 0;
  for (size_t i = 0; i < n; ++i) {
    tp += ref[i] == 1 && cur[i];
    fn += ref[i] == 1 && !cur[i];
    fpc += ref[i] == 0 && cur[i];
    tn += ref[i] == 0 && !cur[i];
  }
  free(cur);
  const float tp0 = (float)tp, fn0 = (float)fn, fp0 = (float)fpc, tn0 = (float)tn;
  const float dividend = sqrtf((tp0 + fp0) * (tp0 + fn0) * (tn0 + fp0) * (tn0 + fn0));
  return dividend != 0.0f ? (tp0 * tn0 - fp0 * fn0) / dividend : GD_CMCC_INVALID;
}

/* MCC of one pose (move vector m of ligand conformation lig_conf against
 * protein conformation prt_conf), with the reference map of the complex
 * (ligand conformation 0, start pose, protein conformation ref_prt). */
float orc_mcc(const gd_complex *cx, int ref_prt, int prt_conf, int lig_conf,
              const float m[6])
{
  int nref;
  unsigned char *ref = orc_mcc_ref(cx, ref_prt, &nref);
  const int lna = cx->lig.lna;
  float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
  float center[3];
  orc_place(cx, lig_conf, m, buf, buf + lna, buf + 2 * lna, center);
  const float v = orc_mcc_of(cx, prt_conf, buf, buf + lna, buf + 2 * lna, ref);
  free(buf);
  free(ref);
  return v;
}

/* ------------------------------------------------------------------------ */
/* Contact-mode similarity matrix (SimilarityMatirxGen src/util.C:37-87     */
/* CalculateSimilarityMatrix, :90-110 InitConfMatrix, :146-193              */
/* CalculateContactModeScore).  confs[n][8] = trace rows {protein conf,     */
/* ligand conf, move[6]}; S[i][j] = the MCC of conformation j's contacts    */
/* against conformation i's map.  Each conformation's map is built once     */
/* (PlaceLigand + the dst <= pmf0 test) and kept as bits; the four counts   */
/* of a pair are those of the reference's double loop, and the score uses   */
/* its arithmetic: float products of the sums, sqrtf, the integer numerator */
/* tp tn - fp fn (two's-complement wrap, as the reference's int on the      */
/* machines it ran on).                                                     */
/* ------------------------------------------------------------------------ */
static float orc_contact_mcc(int tp, int fn, int fpc, int tn)
{
  const float dividend =
      sqrtf((float)(tp + fpc) * (float)(tp + fn) * (float)(tn + fpc) * (float)(tn + fn));
  const int num = (int)((unsigned)tp * (unsigned)tn - (unsigned)fpc * (unsigned)fn);
  return dividend != 0.0f ? (float)num / dividend : GD_CMCC_INVALID;
}

void orc_similarity_matrix(const gd_complex *cx, int n, const float *confs, float *S)
{
  const int lna = cx->lig.lna;
  const size_t npair = (size_t)lna * cx->prt.pnp;
  const size_t nw = (npair + 63) / 64;
  uint64_t *maps = (uint64_t *)calloc(nw * (size_t)(n > 0 ? n : 1), sizeof(uint64_t));
  int *pop = (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int i = 0; i < n; ++i) {
    const float *t = confs + (size_t)8 * i;
    float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
    unsigned char *c = (unsigned char *)malloc(npair);
    float center[3];
    orc_place(cx, (int)t[1], t + 2, buf, buf + lna, buf + 2 * lna, center);
    orc_contacts(cx, (int)t[0], buf, buf + lna, buf + 2 * lna, c);
    uint64_t *w = maps + nw * (size_t)i;
    int cnt = 0;
    for (size_t k = 0; k < npair; ++k)
      if (c[k]) {
        w[k >> 6] |= (uint64_t)1 << (k & 63);
        ++cnt;
      }
    pop[i] = cnt;
    free(c);
    free(buf);
  }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int i = 0; i < n; ++i) {
    const uint64_t *a = maps + nw * (size_t)i;
    for (int j = 0; j < n; ++j) {
      const uint64_t *b = maps + nw * (size_t)j;
      int tp = 0;
      for (size_t k = 0; k < nw; ++k) tp += __builtin_popcountll(a[k] & b[k]);
      const int fn = pop[i] - tp, fpc = pop[j] - tp;
      const int tn = (int)npair - tp - fn - fpc;
      S[(size_t)i * n + j] = orc_contact_mcc(tp, fn, fpc, tn);
    }
  }
  free(pop);
  free(maps);
}

/* ------------------------------------------------------------------------ */
/* Replica-exchange Monte Carlo                                             */
/* ------------------------------------------------------------------------ */
typedef struct orc_rep {
  float m_old[6];
  float e_old[GD_NTERM];
  float cmcc;
  int idx_tmp;
  int acs;
} orc_rep;

/* One MC step of one replica: Move_d, CalcEnergy_d, Accept_d.  Returns the
 * proposed total energy through *e_prop and the decision. */
static int orc_mc_step(const gd_complex *cx, const gd_mc_params *mc, int n_lig,
                       int n_tmp, int r, int step, orc_rep *st, float *buf,
                       float *e_prop, const unsigned char *mcc_ref)
{
  const int p = r / (n_tmp * n_lig);
  const int l = r % n_lig;
  uint32_t key[2], o0[4], o1[4];
  orc_key(mc->seed, mc->stream_id, key);
  const uint32_t c0[4] = {(uint32_t)r, (uint32_t)step, 0u, 0u};
  const uint32_t c1[4] = {(uint32_t)r, (uint32_t)step, 1u, 0u};
  orc_philox(c0, key, o0);
  orc_philox(c1, key, o1);
  const uint32_t bits[6] = {o0[0], o0[1], o0[2], o0[3], o1[0], o1[1]};
  float m_new[6];
  for (int k = 0; k < 6; ++k) {
    const float perturbation = 2.0f * orc_u01(bits[k]) - 1.0f;
    m_new[k] = mc->move_scale[k] * perturbation + st->m_old[k];
  }
  const int lna = cx->lig.lna;
  float center[3];
  orc_place(cx, l, m_new, buf, buf + lna, buf + 2 * lna, center);
  double raw[GD_NRAW];
  float e_new[GD_NTERM];
  orc_energy_coords(cx, p, buf, buf + lna, buf + 2 * lna, center, raw, e_new,
                    NULL);
  if (mc->flags & GD_MC_BAYES) e_new[GD_E_TOTAL] = orc_bayes_total(e_new);
  const float mb = mc->minus_beta[st->idx_tmp];
  const float de = e_new[GD_E_TOTAL] - st->e_old[GD_E_TOTAL];
  const int acc = orc_u01(o1[2]) < orc_expf(de * mb);
  *e_prop = e_new[GD_E_TOTAL];
  if (acc) {
    memcpy(st->m_old, m_new, sizeof(m_new));
    memcpy(st->e_old, e_new, sizeof(e_new));
    /* MCC follows the accepted state (accept_d.cu:50) */
    if (mcc_ref) st->cmcc = orc_mcc_of(cx, p, buf, buf + lna, buf + 2 * lna, mcc_ref);
    st->acs += 1;
  }
  return acc;
}

/* Exchange of one (p, l) group, exchangereplicas_d.cu:26-79; counters by
 * slot as the reference.  Fills swapped[t] with 1 where slot t swapped. */
static void orc_exchange_group(const gd_mc_params *mc, int n_lig, int n_tmp,
                               int p, int l, int round, int mode_t,
                               orc_rep *reps, int *acs_slot)
{
  int temps[64], orders[64];
  float energies[64];
  uint32_t key[2];
  orc_key(mc->seed, mc->stream_id, key);
  const int g = p * n_lig + l;
  for (int t = 0; t < n_tmp; ++t) {
    const int r = n_tmp * n_lig * p + n_lig * t + l;
    temps[t] = reps[r].idx_tmp;
    energies[t] = reps[r].e_old[GD_E_TOTAL];
    orders[temps[t]] = t;
  }
  const int maxpair = n_tmp / 2 - (n_tmp % 2 == 0) * (mode_t == 1);
  for (int pair = 0; pair < maxpair; ++pair) {
    const int i1 = (pair << 1) + mode_t;
    const int i2 = i1 + 1;
    const int o1 = orders[i1];
    const int o2 = orders[i2];
    const int tt = temps[o1];
    const float etot1 = energies[o1];
    const float etot2 = energies[o2];
    const float mb1 = mc->minus_beta[temps[o1]];
    const float mb2 = mc->minus_beta[temps[o2]];
    const float delta = (mb1 - mb2) * (etot2 - etot1);
    const float prob = orc_expf(delta);
    const uint32_t ctr[4] = {(uint32_t)g, (uint32_t)round, 2u, (uint32_t)pair};
    uint32_t o[4];
    orc_philox(ctr, key, o);
    if (prob > orc_u01(o[0])) {
      temps[o1] = temps[o2];
      temps[o2] = tt;
      acs_slot[o1] += 1;
      acs_slot[o2] += 1;
    }
  }
  for (int t = 0; t < n_tmp; ++t) {
    const int r = n_tmp * n_lig * p + n_lig * t + l;
    reps[r].idx_tmp = temps[t];
  }
}

/* Exchange round of all groups with given totals and temperature indices;
 * exposed for the decision-replay test.  idx_tmp is updated in place. */
void orc_exchange(const gd_mc_params *mc, int n_prt, int n_lig, int n_tmp,
                  int round, int mode_t, const float *etotal, int *idx_tmp,
                  int *acs_slot)
{
  const int n_rep = n_prt * n_lig * n_tmp;
  orc_rep *reps = (orc_rep *)calloc((size_t)n_rep, sizeof(orc_rep));
  for (int r = 0; r < n_rep; ++r) {
    reps[r].idx_tmp = idx_tmp[r];
    reps[r].e_old[GD_E_TOTAL] = etotal[r];
  }
  for (int p = 0; p < n_prt; ++p)
    for (int l = 0; l < n_lig; ++l)
      orc_exchange_group(mc, n_lig, n_tmp, p, l, round, mode_t, reps, acs_slot);
  for (int r = 0; r < n_rep; ++r) idx_tmp[r] = reps[r].idx_tmp;
  free(reps);
}

/* Full run: MonteCarlo_Init_d, then steps_total MC steps with exchanges
 * every steps_per_exchange steps (gpusingle.cu:5-37).  Outputs follow
 * gd_mc_log; record (optional) holds [n_rep][steps_total] gd_record. */
int orc_remc_run(const gd_complex *cx, const gd_mc_params *mc, gd_mc_log *log,
                 int n_threads)
{
  const int n_prt = cx->prt.n_conf, n_lig = cx->lig.n_conf, n_tmp = mc->n_tmp;
  const int n_rep = n_prt * n_lig * n_tmp;
  const int spe = mc->steps_per_exchange;
  if (spe <= 0 || mc->steps_total % spe != 0 || n_tmp > 64) return GD_EINVAL;
  const int lna = cx->lig.lna;
  orc_rep *reps = (orc_rep *)calloc((size_t)n_rep, sizeof(orc_rep));
  int *acs_slot = (int *)calloc((size_t)n_tmp, sizeof(int));
  /* MCC reference map from replica 0 before MoveAway (montecarlo_d.cu:24-25) */
  int nref = 0;
  unsigned char *mcc_ref =
      (mc->flags & GD_MC_MCC) ? orc_mcc_ref(cx, 0, &nref) : NULL;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif

  /* MonteCarlo_Init_d, montecarlo_d.cu:12-55 */
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
#ifdef _OPENMP
#pragma omp for
#endif
    for (int r = 0; r < n_rep; ++r) {
      const int p = r / (n_tmp * n_lig), t = (r / n_lig) % n_tmp, l = r % n_lig;
      orc_rep *st = &reps[r];
      memset(st->m_old, 0, sizeof(st->m_old));
      st->idx_tmp = t;
      float m[6];
      for (int k = 0; k < 6; ++k)
        m[k] = (mc->flags & GD_MC_MOVE_AWAY) ? mc->move_scale[k] * 44.5f + 0.0f
                                             : 0.0f;
      float center[3];
      orc_place(cx, l, m, buf, buf + lna, buf + 2 * lna, center);
      double raw[GD_NRAW];
      orc_energy_coords(cx, p, buf, buf + lna, buf + 2 * lna, center, raw,
                        st->e_old, NULL);
      if (mc->flags & GD_MC_BAYES) st->e_old[GD_E_TOTAL] = orc_bayes_total(st->e_old);
      st->cmcc = mcc_ref ? orc_mcc_of(cx, p, buf, buf + lna, buf + 2 * lna, mcc_ref) : 0.0f;
      /* forced accept with beta = 0 (montecarlo_d.cu:236-239) */
      memcpy(st->m_old, m, sizeof(m));
      st->acs = 0;
    }
    free(buf);
  }

  for (int s0 = 0; s0 < mc->steps_total; s0 += spe) {
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
      float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (int r = 0; r < n_rep; ++r) {
        const int p = r / (n_tmp * n_lig), l = r % n_lig;
        for (int s = s0; s < s0 + spe; ++s) {
          gd_record rec;
          if (log && log->record) {
            rec.idx_rep = r;
            rec.idx_prt = p;
            rec.idx_tmp = reps[r].idx_tmp;
            rec.idx_lig = l;
            memcpy(rec.e, reps[r].e_old, sizeof(rec.e));
            rec.cmcc = mcc_ref ? reps[r].cmcc : 0.0f;
            memcpy(rec.movematrix, reps[r].m_old, sizeof(rec.movematrix));
            rec.step = s;
          }
          float e_prop;
          const int acc =
              orc_mc_step(cx, mc, n_lig, n_tmp, r, s, &reps[r], buf, &e_prop, mcc_ref);
          if (log && log->record) {
            rec.e_prop_total = e_prop;
            rec.accepted = acc;
            log->record[(size_t)r * mc->steps_total + s] = rec;
          }
        }
      }
      free(buf);
    }
    if (mc->flags & GD_MC_EXCHANGE) {
      const int dump = mc->steps_per_dump > 0 ? mc->steps_per_dump : 0;
      const int within = dump ? (s0 % dump) : s0;
      const int mode_t = (within / spe) % 2;
      const int round = s0 / spe;
      for (int p = 0; p < n_prt; ++p)
        for (int l = 0; l < n_lig; ++l)
          orc_exchange_group(mc, n_lig, n_tmp, p, l, round, mode_t, reps,
                             acs_slot);
    }
  }

  if (log) {
    log->ac_mc = 0;
    log->ac_temp_exchg = 0;
    for (int r = 0; r < n_rep; ++r) {
      log->ac_mc += reps[r].acs;
      if (log->acs_mc) log->acs_mc[r] = reps[r].acs;
      if (log->energy) memcpy(log->energy + (size_t)GD_NTERM * r, reps[r].e_old, sizeof(float) * GD_NTERM);
      if (log->movematrix) memcpy(log->movematrix + (size_t)6 * r, reps[r].m_old, sizeof(float) * 6);
      if (log->idx_tmp) log->idx_tmp[r] = reps[r].idx_tmp;
    }
    for (int t = 0; t < n_tmp; ++t) {
      log->ac_temp_exchg += acs_slot[t];
      if (log->acs_temp_exchg) log->acs_temp_exchg[t] = acs_slot[t];
    }
  }
  free(reps);
  free(acs_slot);
  free(mcc_ref);
  return GD_OK;
}

/* Time-bounded CPU rate sample: runs MC steps of the replica range
 * [r0, r0 + n_rep_sample) of the full ensemble for n_steps steps (no
 * exchange) and returns the number of energy evaluations done. */
long long orc_mc_sample(const gd_complex *cx, const gd_mc_params *mc, int r0,
                        int n_rep_sample, int n_steps, int n_threads)
{
  const int n_lig = cx->lig.n_conf, n_tmp = mc->n_tmp, lna = cx->lig.lna;
  long long done = 0;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel reduction(+ : done)
#endif
  {
    float *buf = (float *)malloc(sizeof(float) * 3 * (size_t)lna);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int i = 0; i < n_rep_sample; ++i) {
      const int r = r0 + i;
      orc_rep st;
      memset(&st, 0, sizeof(st));
      st.idx_tmp = (r / n_lig) % n_tmp;
      st.e_old[GD_E_TOTAL] = 0.0f;
      for (int s = 0; s < n_steps; ++s) {
        float e_prop;
        orc_mc_step(cx, mc, n_lig, n_tmp, r, s, &st, buf, &e_prop, NULL);
        done += 1;
      }
    }
    free(buf);
  }
  return done;
}

int orc_max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
