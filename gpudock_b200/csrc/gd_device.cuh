// gd_device.cuh -- device building blocks of the REMC docking kernels:
// counter-based RNG, the bit-reproducible decision exp, and the mbarrier /
// bulk-copy (TMA engine, non-tensor) primitives for sm_100a.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gd {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Stream layout:
//   key  = { seed_lo, seed_hi ^ stream_id }
//   move of replica r at MC step s:      ctr {r, s, 0, 0} -> perturbations 0..3
//                                        ctr {r, s, 1, 0} -> perturbations 4..5,
//                                                            word 2: accept u
//   exchange round k, group g, pair j:   ctr {g, k, 2, j} -> word 0
// ---------------------------------------------------------------------------
struct U4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t hi0 = mulhi32(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = mulhi32(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__host__ __device__ __forceinline__ void rng_key(uint64_t seed, uint32_t stream, uint32_t &k0,
                                                 uint32_t &k1) {
  k0 = (uint32_t)seed;
  k1 = (uint32_t)(seed >> 32) ^ stream;
}

// 24-bit uniform in [0, 1); exact in single precision.
__device__ __forceinline__ float u01(uint32_t x) {
  return __fmul_rn(__uint2float_rn(x >> 8), 0x1p-24f);
}

// ---------------------------------------------------------------------------
// Decision exp: Cody-Waite reduction with ln 2 split in a 16-bit head and a
// tail, degree-7 Taylor polynomial of e^r on |r| <= ln2/2 (Horner, fused),
// scaling by 2^k in two exact multiplies.  Each step is one correctly
// rounded IEEE operation, so the host oracle's copy returns the same bits.
// Used only where a decision is taken (Metropolis, exchange); the energy uses
// the hardware exp2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float decision_expf(float x) {
  if (x != x) return x;
  if (x > 88.72f) return __int_as_float(0x7f800000);
  if (x < -87.33f) return 0.0f;
  const float kf = rintf(__fmul_rn(x, 0x1.715476p+0f));
  float r = __fmaf_rn(-kf, 0x1.62e400p-1f, x);
  r = __fmaf_rn(-kf, 0x1.7f7d1cp-20f, r);
  float p = 0x1.a01a02p-13f;
  p = __fmaf_rn(p, r, 0x1.6c16c2p-10f);
  p = __fmaf_rn(p, r, 0x1.111112p-7f);
  p = __fmaf_rn(p, r, 0x1.555556p-5f);
  p = __fmaf_rn(p, r, 0x1.555556p-3f);
  p = __fmaf_rn(p, r, 0x1.0p-1f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  const int k = (int)kf;
  const int k1 = k / 2, k2 = k - k1;
  const float s1 = __int_as_float((k1 + 127) << 23);
  const float s2 = __int_as_float((k2 + 127) << 23);
  return __fmul_rn(__fmul_rn(p, s1), s2);
}

// ---------------------------------------------------------------------------
// Bayesian total (IS_BAYE, calcenergy_d.cu:311-347): the densities of
// util_d.cu:220-290 in the reference's float expressions, with its parameter
// sets (distribution.h), including its pairing of families and parameters
// (the low-decoy H-bond density is a normal with the "logistic" parameters,
// the low-decoy PSP density a logistic with the "Laplace" parameters).
// ---------------------------------------------------------------------------
constexpr float kBayesPI = 3.1415926535f;  // PI of size.h

__device__ __forceinline__ float bayes_norm_pdf(float x, float loc, float scale) {
  const float norm_para = 1.0f / (scale * sqrtf(2.0f * kBayesPI));
  const float prob = expf(0.0f - (x - loc) * (x - loc) / (2.0f * scale * scale));
  return norm_para * prob;
}
__device__ __forceinline__ float bayes_cauchy_pdf(float x, float loc, float scale) {
  const float norm_para = 1.0f / (kBayesPI * scale);
  const float prob = 1.0f / (1.0f + ((x - loc) / scale) * ((x - loc) / scale));
  return norm_para * prob;
}
__device__ __forceinline__ float bayes_logistic_pdf(float x, float loc, float scale) {
  const float norm_para = 1.0f / scale;
  const float e_power = expf(-(x - loc) / scale);
  const float prob = e_power / powf(1.0f + e_power, 2.0f);
  return norm_para * prob;
}
__device__ __forceinline__ float bayes_wald_pdf(float x, float loc, float scale) {
  const float normed_x = (x - loc) / scale;
  if (normed_x < 0.0f) return 0.00000001f;
  const float norm_para = 1.0f / (sqrtf(2.0f * kBayesPI * powf(normed_x, 3.0f)) * scale);
  const float prob = expf(-powf(normed_x - 1.0f, 2.0f) / (2.0f * normed_x));
  return norm_para * prob;
}

// e: the nine normalised terms in rem order (vdw ele pmf psp hdb hpc kde lhm dst).
__device__ __forceinline__ float bayes_total(const float *e) {
  const float vdw = e[0], ele = e[1], pmf = e[2], psp = e[3], hdb = e[4], hpc = e[5];
  const float kde = e[6], lhm = e[7], dst = e[8];
  const float prob_h =
      log10f(bayes_norm_pdf(vdw, 0.05286683f, 0.29916642f)) +
      log10f(bayes_cauchy_pdf(ele, -0.3653806f, 0.00681102f)) +
      log10f(bayes_logistic_pdf(pmf, -0.0221777f, 0.11847532f)) +
      log10f(bayes_wald_pdf(hpc, -1.0041231f, 0.1151713f)) +
      log10f(bayes_norm_pdf(hdb, 0.60986808f, 0.30974999f)) +
      log10f(bayes_logistic_pdf(dst, -0.8246522f, 0.05218529f)) +
      log10f(bayes_logistic_pdf(psp, -0.2346999f, 0.09871713f)) +
      log10f(bayes_wald_pdf(kde, -1.0112055f, 0.09882933f)) +
      log10f(bayes_logistic_pdf(lhm, -0.3377100f, 0.09282947f));
  const float prob_l =
      log10f(bayes_norm_pdf(vdw, 0.15818486f, 0.29032471f)) +
      log10f(bayes_cauchy_pdf(ele, -0.3647824f, 0.00534225f)) +
      log10f(bayes_logistic_pdf(pmf, 0.04257942f, 0.08801551f)) +
      log10f(bayes_wald_pdf(hpc, -1.0019512f, 0.10312611f)) +
      log10f(bayes_norm_pdf(hdb, 0.76967708f, 0.11224029f)) +
      log10f(bayes_logistic_pdf(dst, -0.7509618f, 0.08757299f)) +
      log10f(bayes_logistic_pdf(psp, -0.2022064f, 0.07854212f)) +
      log10f(bayes_wald_pdf(kde, -1.004605f, 0.02967548f)) +
      log10f(bayes_logistic_pdf(lhm, -0.2387023f, 0.12134983f));
  return prob_l - prob_h;
}

// Metropolis rule (accept_d.cu:19-23) on given totals.
__device__ __forceinline__ int metropolis(float e_new, float e_old, float minus_beta, float u) {
  const float de = __fsub_rn(e_new, e_old);
  return u < decision_expf(__fmul_rn(de, minus_beta)) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Shared-memory mbarrier and bulk async copy (cp.async.bulk, TMA engine,
// plain 1-D form: no tensor map, no multicast).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each try_wait itself blocks for
// a hardware-defined slice), records `code` in *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          uint32_t limit = (1u << 22)) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, code);
  return false;
}

// Global -> shared bulk copy completing on an mbarrier (bytes % 16 == 0,
// both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Orders shared-memory accesses made through the generic proxy (ordinary
// loads of a staged tile) before later async-proxy writes (a bulk copy that
// refills the same stage).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Named barrier over nthreads threads of the CTA.
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Thread-block cluster: this CTA's rank, a barrier over every thread of the
// cluster (release / acquire: shared-memory writes before it are visible to
// the cluster's other CTAs after it), and the generic address of the same
// shared-memory location in the cluster's CTA `rank` (distributed shared
// memory).
__device__ __forceinline__ int cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return (int)r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;"
               ::: "memory");
}
template <typename T>
__device__ __forceinline__ const T *cluster_map(const T *p, int rank) {
  uint64_t out;
  asm volatile("mapa.u64 %0, %1, %2;" : "=l"(out) : "l"((uint64_t)p), "r"(rank));
  return reinterpret_cast<const T *>(out);
}

// Nanosecond clock shared by all SMs.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Release store / acquire load of a word at GPU scope (progress flags
// between CTAs of one launch).
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits until *p >= target, for at most `limit` polls about 256 ns apart
// (about four seconds by default); if it gives up it records `code` in *err
// and returns false, so a lost flag costs a wrong result, not a hung GPU.
__device__ __forceinline__ bool wait_progress(const int *p, int target, int *err, int code,
                                              uint32_t limit = (1u << 24)) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (ld_acquire(p) >= target) return true;
    __nanosleep(256);
  }
  if (err) atomicExch(err, code);
  return false;
}

}  // namespace gd
