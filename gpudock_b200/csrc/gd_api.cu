// gd_api.cu -- host side of the C-ABI in include/gpudock.h: contexts, the
// device layout of a complex, pose energies, and the REMC run loop.
//
// Boundary replaced: Run() of gpudocksm-rem-1.2/src/run.cu:41-353 (which
// staged every table with cudaMemcpy/cudaMemcpyToSymbol, launched
// MonteCarlo_d / ExchangeReplicas_d synchronously and exit()ed on errors).
// Here every call returns a status, device memory belongs to handles, and
// launches are asynchronous on the context stream.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gd_internal.h"

using namespace gd;

namespace {

thread_local std::string g_err;

gd_status fail(gd_status st, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}

#define GD_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? GD_ENOMEM : GD_ECUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                  \
  } while (0)

#define GD_TRY(call)               \
  do {                             \
    gd_status s_ = (call);         \
    if (s_ != GD_OK) return s_;    \
  } while (0)

constexpr float kPI = 3.1415926535f;  // size.h:86

}  // namespace

// ---------------------------------------------------------------------------
// Opaque handles
// ---------------------------------------------------------------------------
struct gd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int *d_err = nullptr;
  uint64_t launches = 0;
  int n_sm = 148;
};

struct gd_dcomplex {
  gd_ctx *ctx = nullptr;
  KTables T{};
  std::vector<void *> allocs;
  size_t bytes = 0;
};

struct gd_remc {
  gd_ctx *ctx = nullptr;
  const gd_dcomplex *dcx = nullptr;
  gd_mc_params mc{};
  std::vector<float> minus_beta;
  KState st{};
  int n_prt = 0, n_lig = 0, n_tmp = 0, n_rep = 0;
  int *d_cta_rep0 = nullptr, *d_cta_nrep = nullptr;
  int n_cta = 0;
  int step = 0;  // MC steps done since init
  int n_warps = 0, n_stages = 0, resident = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timing = false;
  double t_compute = 0.0;
  std::vector<void *> allocs;
  // optional per-launch timing of the MC and exchange kernels
  bool profile = false;
  std::vector<cudaEvent_t> prof_ev;  // pairs: start, stop
  std::vector<int> prof_kind;        // 0 = MC interval, 1 = exchange
};

extern "C" const char *gd_last_error(void) { return g_err.c_str(); }
extern "C" const char *gd_version(void) { return "gpudock-b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------------------
// Force-field tables (OptimizeEnepara, util.C:405-458) and temperatures
// (SetTemperature, util.C:491-532): host arithmetic in single precision with
// the same libm calls, so the tables match the reference's bit for bit.
// ---------------------------------------------------------------------------
extern "C" gd_status gd_enepara_optimize(const gd_enepara_raw *r, gd_enepara *e) {
  if (!r || !e) return fail(GD_EINVAL, "gd_enepara_optimize: NULL argument");
  const float sqrt_2_pi = sqrtf(2.0f * kPI);
  std::memset(e, 0, sizeof(*e));
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
  return GD_OK;
}

extern "C" gd_status gd_set_temperature(int n, float floor_t, float ceil_t, float *temps,
                                        float *minus_beta) {
  if (n < 1 || !minus_beta) return fail(GD_EINVAL, "gd_set_temperature: n=%d", n);
  if (!(floor_t > 0.f) || !(ceil_t > 0.f))
    return fail(GD_EINVAL, "gd_set_temperature: temperatures must be > 0");
  if (n == 1) {
    const float beta = 1.0f / (1.0f * floor_t);
    if (temps) temps[0] = floor_t;
    minus_beta[0] = 0.0f - beta;
    return GD_OK;
  }
  const float ratio = expf(logf(ceil_t / floor_t) / (float)(n - 1));
  float a = floor_t;
  for (int i = 0; i < n; ++i) {
    const float beta = 1.0f / (1.0f * a);
    if (temps) temps[i] = a;
    minus_beta[i] = 0.0f - beta;
    a *= ratio;
  }
  return GD_OK;
}

// ---------------------------------------------------------------------------
// Validation
// ---------------------------------------------------------------------------
extern "C" gd_status gd_complex_validate(const gd_complex *cx) {
  if (!cx) return fail(GD_EINVAL, "complex is NULL");
  const gd_ligand &L = cx->lig;
  const gd_protein &P = cx->prt;
  if (!cx->ff) return fail(GD_EINVAL, "force field is NULL");
  if (L.lna < 1 || L.lna > MAX_WARPS * MAX_APW)
    return fail(GD_EINVAL, "ligand atoms lna=%d outside [1, %d]", L.lna, MAX_WARPS * MAX_APW);
  if (L.n_conf < 1) return fail(GD_EINVAL, "ligand conformations n_conf=%d", L.n_conf);
  if (!L.x || !L.y || !L.z || !L.t || !L.c || !L.n) return fail(GD_EINVAL, "ligand array NULL");
  if (P.pnp < 1 || P.n_conf < 1)
    return fail(GD_EINVAL, "protein pnp=%d n_conf=%d", P.pnp, P.n_conf);
  if (!P.x || !P.y || !P.z || !P.t || !P.c || !P.ele || !P.seq3r || !P.c0_and_d12_or_c2 || !P.hpp)
    return fail(GD_EINVAL, "protein array NULL");
  if (cx->psp.n_col < 1 || !cx->psp.psp) return fail(GD_EINVAL, "psp table missing");
  for (int a = 0; a < L.lna; ++a) {
    if (L.t[a] < 0 || L.t[a] >= GD_NLT)
      return fail(GD_EINVAL, "ligand atom %d type %d outside [0, %d)", a, L.t[a], GD_NLT);
    if (cx->mcs.pos > 0 && (L.n[a] < 0 || L.n[a] + 1 >= cx->mcs.n_field))
      return fail(GD_EINVAL, "ligand atom %d number %d: MCS field n+1 outside [0, %d)", a, L.n[a],
                  cx->mcs.n_field);
  }
  for (int p = 0; p < P.pnp; ++p) {
    if (P.t[p] < 0 || P.t[p] >= GD_NPT)
      return fail(GD_EINVAL, "protein point %d type %d outside [0, %d)", p, P.t[p], GD_NPT);
    if (P.c[p] < 0 || P.c[p] > 3) return fail(GD_EINVAL, "protein point %d class %d", p, P.c[p]);
    if (P.seq3r[p] < 0 || P.seq3r[p] >= cx->psp.n_col || P.seq3r[p] > MAX_SEQ3R)
      return fail(GD_EINVAL, "protein point %d seq3r %d outside [0, %d)", p, P.seq3r[p],
                  std::min(cx->psp.n_col, MAX_SEQ3R + 1));
  }
  if (cx->kde.pnk < 0) return fail(GD_EINVAL, "kde pnk=%d", cx->kde.pnk);
  if (cx->kde.pnk > 0) {
    if (!cx->kde.x || !cx->kde.y || !cx->kde.z || !cx->kde.t) return fail(GD_EINVAL, "kde NULL");
    for (int k = 0; k < cx->kde.pnk; ++k)
      if (cx->kde.t[k] < 0 || cx->kde.t[k] >= GD_NLT)
        return fail(GD_EINVAL, "kde point %d type %d", k, cx->kde.t[k]);
  }
  if (cx->mcs.pos < 0) return fail(GD_EINVAL, "mcs pos=%d", cx->mcs.pos);
  if (cx->mcs.pos > 0 && (!cx->mcs.x || !cx->mcs.y || !cx->mcs.z || !cx->mcs.tcc))
    return fail(GD_EINVAL, "mcs arrays NULL");
  return GD_OK;
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
extern "C" gd_status gd_ctx_create(int device, void *stream, gd_ctx **out) {
  if (!out) return fail(GD_EINVAL, "gd_ctx_create: out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(GD_ENODEV, "no CUDA device (%s)", cudaGetErrorString(e));
  if (device < 0 || device >= n) return fail(GD_EINVAL, "device %d of %d", device, n);
  GD_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  GD_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(GD_ENODEV, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major,
                prop.minor);
  gd_ctx *c = new (std::nothrow) gd_ctx;
  if (!c) return fail(GD_ENOMEM, "host allocation");
  c->device = device;
  c->n_sm = prop.multiProcessorCount;
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete c;
      return fail(GD_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    c->own_stream = true;
  }
  e = cudaMalloc(&c->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return fail(GD_ENOMEM, "cudaMalloc error word: %s", cudaGetErrorString(e));
  }
  *out = c;
  return GD_OK;
}

extern "C" gd_status gd_ctx_destroy(gd_ctx *c) {
  if (!c) return GD_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaFree(c->d_err);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
  return GD_OK;
}

static gd_status ctx_check(gd_ctx *c) {
  int h = 0;
  GD_CUDA(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GD_CUDA(cudaStreamSynchronize(c->stream));
  if (h != 0) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
    cudaStreamSynchronize(c->stream);
    return fail(GD_ETIMEDOUT, "a bounded barrier wait gave up in a kernel (code %d)", h);
  }
  return GD_OK;
}

extern "C" gd_status gd_ctx_sync(gd_ctx *c) {
  if (!c) return fail(GD_EINVAL, "ctx is NULL");
  GD_CUDA(cudaSetDevice(c->device));
  return ctx_check(c);
}

extern "C" uint64_t gd_ctx_launch_count(const gd_ctx *c) { return c ? c->launches : 0; }

// ---------------------------------------------------------------------------
// Device layout of a complex
// ---------------------------------------------------------------------------
template <typename T>
static gd_status upload(gd_dcomplex *d, const std::vector<T> &h, const T **out) {
  void *p = nullptr;
  const size_t n = std::max<size_t>(h.size(), 1) * sizeof(T);
  GD_CUDA(cudaMalloc(&p, n));
  d->allocs.push_back(p);
  d->bytes += n;
  if (!h.empty())
    GD_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice,
                            d->ctx->stream));
  *out = (const T *)p;
  return GD_OK;
}

extern "C" gd_status gd_complex_free(gd_dcomplex *d) {
  if (!d) return GD_OK;
  if (d->ctx) {
    cudaSetDevice(d->ctx->device);
    cudaStreamSynchronize(d->ctx->stream);
  }
  for (void *p : d->allocs) cudaFree(p);
  delete d;
  return GD_OK;
}

extern "C" size_t gd_complex_device_bytes(const gd_dcomplex *d) { return d ? d->bytes : 0; }

static gd_status complex_upload_impl(gd_ctx *ctx, const gd_complex *cx, gd_dcomplex *d) {
  const gd_ligand &L = cx->lig;
  const gd_protein &P = cx->prt;
  const gd_enepara &F = *cx->ff;
  KTables &T = d->T;
  const int lna = L.lna, pnp = P.pnp;
  const int pnp_pad = (pnp + TILE_PTS - 1) / TILE_PTS * TILE_PTS;

  // protein points: {x, y, z, ele} per conformation, {hpp, meta} shared
  std::vector<float4> pa((size_t)P.n_conf * pnp_pad, make_float4(0.f, 0.f, 0.f, 0.f));
  for (int c = 0; c < P.n_conf; ++c)
    for (int p = 0; p < pnp; ++p) {
      const size_t i = (size_t)c * pnp + p;
      pa[(size_t)c * pnp_pad + p] = make_float4(P.x[i], P.y[i], P.z[i], P.ele[p]);
    }
  std::vector<float2> pb((size_t)pnp_pad, make_float2(0.f, 0.f));
  for (int p = 0; p < pnp; ++p) {
    uint32_t meta = (uint32_t)P.t[p] | ((uint32_t)P.c[p] << META_CLASS_SHIFT) |
                    ((uint32_t)P.seq3r[p] << META_SEQ_SHIFT);
    if (P.c0_and_d12_or_c2[p] == 1) meta |= META_HPC_BIT;
    float mf;
    std::memcpy(&mf, &meta, 4);
    pb[p] = make_float2(P.hpp[p], mf);
  }
  // type-pair table [lig type][point type]
  std::vector<float4> ta(GD_NLT * GD_NPT);
  std::vector<float2> tb(GD_NLT * GD_NPT);
  for (int i = 0; i < GD_NLT; ++i)
    for (int j = 0; j < GD_NPT; ++j) {
      ta[i * GD_NPT + j] = make_float4(F.p1a[i][j], F.p2a[i][j], F.pmf0[i][j], F.pmf1[i][j]);
      tb[i * GD_NPT + j] = make_float2(F.hdb0[i][j], F.hdb1[i][j]);
    }
  // ligand conformations
  std::vector<float4> lg((size_t)L.n_conf * lna);
  for (size_t i = 0; i < lg.size(); ++i) lg[i] = make_float4(L.x[i], L.y[i], L.z[i], 0.f);
  std::vector<int> lt(L.t, L.t + lna);
  std::vector<float> lq(L.c, L.c + lna);
  std::vector<float> psp(cx->psp.psp, cx->psp.psp + (size_t)GD_NLT * cx->psp.n_col);
  // KDE points bucketed by ligand type
  std::vector<int> koff(GD_NLT + 1, 0);
  for (int k = 0; k < cx->kde.pnk; ++k) koff[cx->kde.t[k] + 1] += 1;
  for (int i = 0; i < GD_NLT; ++i) koff[i + 1] += koff[i];
  std::vector<float4> kd((size_t)cx->kde.pnk);
  {
    std::vector<int> fill(koff.begin(), koff.end() - 1);
    for (int k = 0; k < cx->kde.pnk; ++k)
      kd[fill[cx->kde.t[k]]++] = make_float4(cx->kde.x[k], cx->kde.y[k], cx->kde.z[k], 0.f);
  }
  // MCS gathered per ligand atom: field n + 1 (calcenergy_d.cu:240-241)
  const int pos = cx->mcs.pos;
  std::vector<float4> mc((size_t)pos * lna);
  std::vector<float> tcc(pos), cnt(pos);
  for (int m = 0; m < pos; ++m) {
    int c = 0;
    for (int a = 0; a < lna; ++a) {
      const size_t f = (size_t)m * cx->mcs.n_field + L.n[a] + 1;
      const bool valid = cx->mcs.x[f] != GD_MCS_INVALID_COORD;
      mc[(size_t)m * lna + a] =
          make_float4(cx->mcs.x[f], cx->mcs.y[f], cx->mcs.z[f], valid ? 1.f : 0.f);
      c += valid;
    }
    tcc[m] = cx->mcs.tcc[m];
    cnt[m] = (float)c;
  }

  GD_TRY(upload(d, pa, &T.pt_a));
  GD_TRY(upload(d, pb, &T.pt_b));
  GD_TRY(upload(d, ta, &T.tab_a));
  GD_TRY(upload(d, tb, &T.tab_b));
  GD_TRY(upload(d, lg, &T.lig));
  GD_TRY(upload(d, lt, &T.lig_t));
  GD_TRY(upload(d, lq, &T.lig_q));
  GD_TRY(upload(d, psp, &T.psp));
  GD_TRY(upload(d, kd, &T.kde));
  GD_TRY(upload(d, koff, &T.kde_off));
  GD_TRY(upload(d, mc, &T.mcs));
  GD_TRY(upload(d, tcc, &T.mcs_tcc));
  GD_TRY(upload(d, cnt, &T.mcs_cnt));

  T.lna = lna;
  T.n_lig = L.n_conf;
  T.pnp = pnp;
  T.pnp_pad = pnp_pad;
  T.n_prt = P.n_conf;
  T.pos = pos;
  T.psp_ncol = cx->psp.n_col;
  T.lj0 = F.lj0;
  T.lj0lj1 = F.lj0 * F.lj1;
  T.el0 = F.el0;
  T.el1 = F.el1;
  T.inv_el1 = 1.0f / F.el1;
  T.a1 = F.a1;
  T.b1 = F.b1;
  T.kde2 = F.kde2;
  T.kde3 = F.kde3;
  T.s2pi = sqrtf(2.0f * kPI);
  for (int i = 0; i < GD_NLT; ++i) {
    T.hpl0[i] = F.hpl0[i];
    T.hpl1[i] = F.hpl1[i];
    T.hpl2[i] = F.hpl2[i];
  }
  for (int i = 0; i < GD_NTERM; ++i) {
    T.a_para[i] = F.a_para[i];
    T.b_para[i] = F.b_para[i];
    T.w[i] = F.w[i];
  }
  for (int i = 0; i < 3; ++i) {
    T.lig_center[i] = L.center[i];
    T.pocket[i] = P.pocket_center[i];
  }
  GD_CUDA(cudaStreamSynchronize(ctx->stream));
  return GD_OK;
}

extern "C" gd_status gd_complex_upload(gd_ctx *ctx, const gd_complex *cx, gd_dcomplex **out) {
  if (!ctx || !out) return fail(GD_EINVAL, "gd_complex_upload: NULL argument");
  *out = nullptr;
  GD_TRY(gd_complex_validate(cx));
  GD_CUDA(cudaSetDevice(ctx->device));
  gd_dcomplex *d = new (std::nothrow) gd_dcomplex;
  if (!d) return fail(GD_ENOMEM, "host allocation");
  d->ctx = ctx;
  gd_status st;
  try {
    st = complex_upload_impl(ctx, cx, d);
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation while packing the complex");
  }
  if (st != GD_OK) {
    gd_complex_free(d);
    return st;
  }
  *out = d;
  return GD_OK;
}

// ---------------------------------------------------------------------------
// Launch shape
// ---------------------------------------------------------------------------
static int pick_warps(int lna) {
  int w = (lna + 2) / 3;  // about three ligand atoms per warp
  w = std::max(4, std::min(MAX_WARPS, w));
  while (w * MAX_APW < lna) ++w;
  return w;
}

static void pick_stages(const KTables &T, int n_warps, int *n_stages, int *resident) {
  const int n_tiles = (T.pnp + TILE_PTS - 1) / TILE_PTS;
  const size_t limit = 227 * 1024;
  if (n_tiles <= MAX_RESIDENT_TILES && dock_smem_bytes(n_warps, n_tiles) <= limit) {
    *n_stages = n_tiles;
    *resident = 1;
  } else {
    *n_stages = STREAM_STAGES;
    *resident = 0;
  }
}

// ---------------------------------------------------------------------------
// Pose energies
// ---------------------------------------------------------------------------
extern "C" gd_status gd_energy_poses_dev(gd_ctx *ctx, const gd_dcomplex *d, int prt_conf,
                                         int lig_conf, int n_pose, const float *poses,
                                         float *terms, double *raw) {
  if (!ctx || !d) return fail(GD_EINVAL, "gd_energy_poses_dev: NULL handle");
  if (n_pose < 0) return fail(GD_EINVAL, "n_pose=%d", n_pose);
  if (prt_conf < 0 || prt_conf >= d->T.n_prt)
    return fail(GD_EINVAL, "prt_conf %d outside [0, %d)", prt_conf, d->T.n_prt);
  if (lig_conf < 0 || lig_conf >= d->T.n_lig)
    return fail(GD_EINVAL, "lig_conf %d outside [0, %d)", lig_conf, d->T.n_lig);
  if (n_pose == 0) return GD_OK;
  if (!poses || !terms) return fail(GD_EINVAL, "poses/terms NULL");
  KRun R{};
  R.mode = KMODE_POSES;
  R.n_warps = pick_warps(d->T.lna);
  pick_stages(d->T, R.n_warps, &R.n_stages, &R.resident);
  R.prt_conf = prt_conf;
  R.lig_conf = lig_conf;
  R.n_pose = n_pose;
  R.poses = poses;
  R.terms = terms;
  R.raw = raw;
  R.err = ctx->d_err;
  GD_CUDA(cudaSetDevice(ctx->device));
  GD_CUDA(launch_dock(d->T, R, (n_pose + 31) / 32, ctx->stream));
  ctx->launches += 1;
  return GD_OK;
}

extern "C" gd_status gd_energy_poses(gd_ctx *ctx, const gd_dcomplex *d, int prt_conf,
                                     int lig_conf, int n_pose, const float *poses, float *terms,
                                     double *raw) {
  if (!ctx || !d) return fail(GD_EINVAL, "gd_energy_poses: NULL handle");
  if (n_pose < 0) return fail(GD_EINVAL, "n_pose=%d", n_pose);
  if (n_pose == 0) return GD_OK;
  if (!poses || !terms) return fail(GD_EINVAL, "poses/terms NULL");
  GD_CUDA(cudaSetDevice(ctx->device));
  float *dp = nullptr, *dt = nullptr;
  double *dr = nullptr;
  gd_status st = GD_OK;
  cudaError_t e = cudaMallocAsync(&dp, sizeof(float) * 6 * (size_t)n_pose, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMallocAsync(&dt, sizeof(float) * GD_NTERM * (size_t)n_pose, ctx->stream);
  if (e == cudaSuccess && raw)
    e = cudaMallocAsync(&dr, sizeof(double) * GD_NRAW * (size_t)n_pose, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dp, poses, sizeof(float) * 6 * (size_t)n_pose, cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e != cudaSuccess) {
    st = fail(GD_ENOMEM, "pose buffers: %s", cudaGetErrorString(e));
  } else {
    st = gd_energy_poses_dev(ctx, d, prt_conf, lig_conf, n_pose, dp, dt, dr);
    if (st == GD_OK) {
      e = cudaMemcpyAsync(terms, dt, sizeof(float) * GD_NTERM * (size_t)n_pose,
                          cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess && raw)
        e = cudaMemcpyAsync(raw, dr, sizeof(double) * GD_NRAW * (size_t)n_pose,
                            cudaMemcpyDeviceToHost, ctx->stream);
      if (e != cudaSuccess) st = fail(GD_ECUDA, "copy back: %s", cudaGetErrorString(e));
    }
  }
  if (dp) cudaFreeAsync(dp, ctx->stream);
  if (dt) cudaFreeAsync(dt, ctx->stream);
  if (dr) cudaFreeAsync(dr, ctx->stream);
  if (st != GD_OK) {
    cudaStreamSynchronize(ctx->stream);
    return st;
  }
  return ctx_check(ctx);
}

// ---------------------------------------------------------------------------
// REMC
// ---------------------------------------------------------------------------
extern "C" int gd_remc_n_rep(const gd_remc *r) { return r ? r->n_rep : 0; }

extern "C" gd_status gd_remc_destroy(gd_remc *r) {
  if (!r) return GD_OK;
  if (r->ctx) {
    cudaSetDevice(r->ctx->device);
    cudaStreamSynchronize(r->ctx->stream);
  }
  for (void *p : r->allocs) cudaFree(p);
  for (cudaEvent_t e : r->prof_ev) cudaEventDestroy(e);
  if (r->ev0) cudaEventDestroy(r->ev0);
  if (r->ev1) cudaEventDestroy(r->ev1);
  delete r;
  return GD_OK;
}

template <typename T>
static gd_status dalloc(gd_remc *r, T **out, size_t n) {
  void *p = nullptr;
  GD_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  r->allocs.push_back(p);
  GD_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), r->ctx->stream));
  *out = (T *)p;
  return GD_OK;
}

static gd_status validate_mc(const gd_mc_params *mc) {
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

static gd_status remc_create_impl(gd_ctx *ctx, const gd_dcomplex *d, const gd_mc_params *mc,
                                  gd_remc *r) {
  r->ctx = ctx;
  r->dcx = d;
  r->mc = *mc;
  r->minus_beta.assign(mc->minus_beta, mc->minus_beta + mc->n_tmp);
  r->mc.minus_beta = r->minus_beta.data();
  r->n_prt = d->T.n_prt;
  r->n_lig = d->T.n_lig;
  r->n_tmp = mc->n_tmp;
  const long long nrep = (long long)r->n_prt * r->n_lig * r->n_tmp;
  if (nrep > (1LL << 30)) return fail(GD_EINVAL, "too many replicas: %lld", nrep);
  r->n_rep = (int)nrep;
  KState &S = r->st;
  GD_TRY(dalloc(r, &S.m_old, (size_t)r->n_rep * 6));
  GD_TRY(dalloc(r, &S.e_old, (size_t)r->n_rep * GD_NTERM));
  GD_TRY(dalloc(r, &S.idx_tmp, (size_t)r->n_rep));
  GD_TRY(dalloc(r, &S.acs_mc, (size_t)r->n_rep));
  GD_TRY(dalloc(r, &S.acs_exchg, (size_t)r->n_tmp));
  float *mb = nullptr;
  GD_TRY(dalloc(r, &mb, (size_t)r->n_tmp));
  GD_CUDA(cudaMemcpyAsync(mb, r->minus_beta.data(), sizeof(float) * r->n_tmp,
                          cudaMemcpyHostToDevice, ctx->stream));
  S.minus_beta = mb;
  S.n_rep = r->n_rep;
  S.n_tmp = r->n_tmp;
  S.n_lig_conf = r->n_lig;
  S.record = nullptr;
  S.rec_steps = 0;
  if (mc->flags & GD_MC_RECORD) {
    gd_record *rec = nullptr;
    GD_TRY(dalloc(r, &rec, (size_t)r->n_rep * std::max(1, mc->steps_total)));
    S.record = rec;
    S.rec_steps = mc->steps_total;
  }
  // CTAs: up to 32 consecutive replicas of the same protein conformation
  std::vector<int> c0, cn;
  const int per_p = r->n_tmp * r->n_lig;
  for (int p = 0; p < r->n_prt; ++p)
    for (int j = 0; j < per_p; j += 32) {
      c0.push_back(p * per_p + j);
      cn.push_back(std::min(32, per_p - j));
    }
  r->n_cta = (int)c0.size();
  GD_TRY(dalloc(r, &r->d_cta_rep0, c0.size()));
  GD_TRY(dalloc(r, &r->d_cta_nrep, cn.size()));
  GD_CUDA(cudaMemcpyAsync(r->d_cta_rep0, c0.data(), sizeof(int) * c0.size(),
                          cudaMemcpyHostToDevice, ctx->stream));
  GD_CUDA(cudaMemcpyAsync(r->d_cta_nrep, cn.data(), sizeof(int) * cn.size(),
                          cudaMemcpyHostToDevice, ctx->stream));
  r->n_warps = pick_warps(d->T.lna);
  pick_stages(d->T, r->n_warps, &r->n_stages, &r->resident);
  GD_CUDA(cudaEventCreate(&r->ev0));
  GD_CUDA(cudaEventCreate(&r->ev1));
  GD_CUDA(cudaStreamSynchronize(ctx->stream));
  return GD_OK;
}

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
    st = remc_create_impl(ctx, d, mc, r);
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation");
  }
  if (st != GD_OK) {
    gd_remc_destroy(r);
    return st;
  }
  *out = r;
  return GD_OK;
}

static KRun remc_run_desc(const gd_remc *r, int mode) {
  KRun R{};
  R.mode = mode;
  R.n_warps = r->n_warps;
  R.n_stages = r->n_stages;
  R.resident = r->resident;
  R.cta_rep0 = r->d_cta_rep0;
  R.cta_nrep = r->d_cta_nrep;
  for (int i = 0; i < 6; ++i) R.move_scale[i] = r->mc.move_scale[i];
  R.seed = r->mc.seed;
  R.stream_id = r->mc.stream_id;
  R.flags = r->mc.flags;
  R.st = r->st;
  R.err = r->ctx->d_err;
  return R;
}

extern "C" gd_status gd_remc_init(gd_remc *r) {
  if (!r) return fail(GD_EINVAL, "remc NULL");
  GD_CUDA(cudaSetDevice(r->ctx->device));
  KRun R = remc_run_desc(r, KMODE_INIT);
  R.step0 = 0;
  R.n_steps = 1;
  GD_CUDA(cudaMemsetAsync(r->st.acs_exchg, 0, sizeof(int) * r->n_tmp, r->ctx->stream));
  GD_CUDA(launch_dock(r->dcx->T, R, r->n_cta, r->ctx->stream));
  r->ctx->launches += 1;
  r->step = 0;
  r->t_compute = 0.0;
  return GD_OK;
}

extern "C" gd_status gd_remc_run(gd_remc *r, int n_steps) {
  if (!r) return fail(GD_EINVAL, "remc NULL");
  const int spe = r->mc.steps_per_exchange;
  if (n_steps < 0 || n_steps % spe != 0)
    return fail(GD_EINVAL, "n_steps %d is not a multiple of steps_per_exchange %d", n_steps, spe);
  if (n_steps == 0) return GD_OK;
  GD_CUDA(cudaSetDevice(r->ctx->device));
  GD_CUDA(cudaEventRecord(r->ev0, r->ctx->stream));
  KRun R = remc_run_desc(r, KMODE_REMC);
  auto mark = [&](int kind) -> cudaError_t {
    cudaEvent_t e;
    cudaError_t st = cudaEventCreate(&e);
    if (st != cudaSuccess) return st;
    r->prof_ev.push_back(e);
    r->prof_kind.push_back(kind);
    return cudaEventRecord(e, r->ctx->stream);
  };
  for (int s0 = r->step; s0 < r->step + n_steps; s0 += spe) {
    R.step0 = s0;
    R.n_steps = spe;
    if (r->profile) GD_CUDA(mark(0));
    GD_CUDA(launch_dock(r->dcx->T, R, r->n_cta, r->ctx->stream));
    if (r->profile) GD_CUDA(mark(0));
    r->ctx->launches += 1;
    if (r->mc.flags & GD_MC_EXCHANGE) {
      const int dump = r->mc.steps_per_dump;
      const int within = dump > 0 ? (s0 % dump) : s0;
      const int mode_t = (within / spe) % 2;
      if (r->profile) GD_CUDA(mark(1));
      GD_CUDA(launch_exchange(r->st, r->n_prt, r->n_lig, r->mc.seed, r->mc.stream_id, s0 / spe,
                              mode_t, r->ctx->stream));
      if (r->profile) GD_CUDA(mark(1));
      r->ctx->launches += 1;
    }
  }
  GD_CUDA(cudaEventRecord(r->ev1, r->ctx->stream));
  r->timing = true;
  r->step += n_steps;
  return GD_OK;
}

extern "C" gd_status gd_remc_read(gd_remc *r, gd_mc_log *log) {
  if (!r || !log) return fail(GD_EINVAL, "gd_remc_read: NULL argument");
  GD_CUDA(cudaSetDevice(r->ctx->device));
  GD_TRY(ctx_check(r->ctx));
  if (r->timing) {
    float ms = 0.f;
    GD_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
    r->t_compute += ms * 1e-3;
    r->timing = false;
  }
  const size_t n = (size_t)r->n_rep;
  std::vector<int> acs(n), acx(r->n_tmp);
  cudaStream_t s = r->ctx->stream;
  GD_CUDA(cudaMemcpyAsync(acs.data(), r->st.acs_mc, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaMemcpyAsync(acx.data(), r->st.acs_exchg, sizeof(int) * r->n_tmp,
                          cudaMemcpyDeviceToHost, s));
  if (log->energy)
    GD_CUDA(cudaMemcpyAsync(log->energy, r->st.e_old, sizeof(float) * GD_NTERM * n,
                            cudaMemcpyDeviceToHost, s));
  if (log->movematrix)
    GD_CUDA(cudaMemcpyAsync(log->movematrix, r->st.m_old, sizeof(float) * 6 * n,
                            cudaMemcpyDeviceToHost, s));
  if (log->idx_tmp)
    GD_CUDA(cudaMemcpyAsync(log->idx_tmp, r->st.idx_tmp, sizeof(int) * n, cudaMemcpyDeviceToHost,
                            s));
  if (log->record && r->st.record)
    GD_CUDA(cudaMemcpyAsync(log->record, r->st.record,
                            sizeof(gd_record) * n * std::max(1, r->st.rec_steps),
                            cudaMemcpyDeviceToHost, s));
  GD_CUDA(cudaStreamSynchronize(s));
  log->ac_mc = 0;
  for (size_t i = 0; i < n; ++i) log->ac_mc += acs[i];
  log->ac_temp_exchg = 0;
  for (int t = 0; t < r->n_tmp; ++t) log->ac_temp_exchg += acx[t];
  if (log->acs_mc) std::memcpy(log->acs_mc, acs.data(), sizeof(int) * n);
  if (log->acs_temp_exchg) std::memcpy(log->acs_temp_exchg, acx.data(), sizeof(int) * r->n_tmp);
  log->t_compute = r->t_compute;
  return GD_OK;
}

extern "C" gd_status gd_remc_set_profiling(gd_remc *r, int on) {
  if (!r) return fail(GD_EINVAL, "remc NULL");
  r->profile = on != 0;
  return GD_OK;
}

extern "C" gd_status gd_remc_kernel_times(gd_remc *r, double *mc_ms, int *mc_launches,
                                          double *exch_ms, int *exch_launches) {
  if (!r || !mc_ms || !mc_launches || !exch_ms || !exch_launches)
    return fail(GD_EINVAL, "gd_remc_kernel_times: NULL argument");
  GD_CUDA(cudaSetDevice(r->ctx->device));
  GD_CUDA(cudaStreamSynchronize(r->ctx->stream));
  *mc_ms = *exch_ms = 0.0;
  *mc_launches = *exch_launches = 0;
  for (size_t i = 0; i + 1 < r->prof_ev.size(); i += 2) {
    float ms = 0.f;
    GD_CUDA(cudaEventElapsedTime(&ms, r->prof_ev[i], r->prof_ev[i + 1]));
    if (r->prof_kind[i] == 0) {
      *mc_ms += ms;
      *mc_launches += 1;
    } else {
      *exch_ms += ms;
      *exch_launches += 1;
    }
  }
  for (cudaEvent_t e : r->prof_ev) cudaEventDestroy(e);
  r->prof_ev.clear();
  r->prof_kind.clear();
  return GD_OK;
}

extern "C" gd_status gd_run(const gd_complex *cx, const gd_mc_params *mc, gd_mc_log *log) {
  const auto t0 = std::chrono::steady_clock::now();
  GD_TRY(validate_mc(mc));
  gd_ctx *ctx = nullptr;
  GD_TRY(gd_ctx_create(0, nullptr, &ctx));
  gd_dcomplex *d = nullptr;
  gd_remc *r = nullptr;
  gd_status st = gd_complex_upload(ctx, cx, &d);
  if (st == GD_OK) st = gd_remc_create(ctx, d, mc, &r);
  if (st == GD_OK) st = gd_remc_init(r);
  if (st == GD_OK) st = gd_remc_run(r, mc->steps_total);
  if (st == GD_OK && log) st = gd_remc_read(r, log);
  gd_remc_destroy(r);
  gd_complex_free(d);
  gd_ctx_destroy(ctx);
  if (st == GD_OK && log)
    log->t_wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return st;
}

// ---------------------------------------------------------------------------
// Building blocks for tests
// ---------------------------------------------------------------------------
extern "C" gd_status gd_metropolis_dev(gd_ctx *ctx, int n, const float *e_new, const float *e_old,
                                       const float *mbeta, const int *rep, const int *step,
                                       uint64_t seed, uint32_t stream_id, int *accept) {
  if (!ctx || n < 0) return fail(GD_EINVAL, "gd_metropolis_dev: bad arguments");
  if (n == 0) return GD_OK;
  GD_CUDA(cudaSetDevice(ctx->device));
  GD_CUDA(launch_metropolis(n, e_new, e_old, mbeta, rep, step, seed, stream_id, accept,
                            ctx->stream));
  ctx->launches += 1;
  return GD_OK;
}

extern "C" gd_status gd_philox_dev(gd_ctx *ctx, int n, const uint32_t *ctr4, const uint32_t *key2,
                                   uint32_t *out4) {
  if (!ctx || n < 0) return fail(GD_EINVAL, "gd_philox_dev: bad arguments");
  if (n == 0) return GD_OK;
  GD_CUDA(cudaSetDevice(ctx->device));
  GD_CUDA(launch_philox(n, ctr4, key2, out4, ctx->stream));
  ctx->launches += 1;
  return GD_OK;
}

extern "C" gd_status gd_expf_dev(gd_ctx *ctx, int n, const float *x, float *y) {
  if (!ctx || n < 0) return fail(GD_EINVAL, "gd_expf_dev: bad arguments");
  if (n == 0) return GD_OK;
  GD_CUDA(cudaSetDevice(ctx->device));
  GD_CUDA(launch_expf(n, x, y, ctx->stream));
  ctx->launches += 1;
  return GD_OK;
}

// FP32 FMA throughput probe for the roofline denominator (not in the public
// header's main API; exported for the bench).
extern "C" gd_status gd_fma_peak(gd_ctx *ctx, int n_blocks, int iters, float *ms_out,
                                 double *flops_out) {
  if (!ctx || n_blocks < 1 || iters < 1 || !ms_out || !flops_out)
    return fail(GD_EINVAL, "gd_fma_peak: bad arguments");
  GD_CUDA(cudaSetDevice(ctx->device));
  float *dout = nullptr;
  GD_CUDA(cudaMalloc(&dout, sizeof(float) * n_blocks));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch_fma_peak(dout, n_blocks, iters, ctx->stream);  // warm-up
  cudaEventRecord(a, ctx->stream);
  cudaError_t e = launch_fma_peak(dout, n_blocks, iters, ctx->stream);
  cudaEventRecord(b, ctx->stream);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(dout);
  ctx->launches += 2;
  if (e != cudaSuccess) return fail(GD_ECUDA, "fma probe: %s", cudaGetErrorString(e));
  *ms_out = ms;
  *flops_out = 2.0 * 8.0 * 16.0 * (double)iters * 256.0 * (double)n_blocks;
  return GD_OK;
}
