// gd_api.cu -- host side of the C-ABI in include/gpudock.h: errors, force
// field and temperature tables, validation, contexts, the device layout of a
// complex, pose energies, launch-shape selection and test entry points.
//
// Boundary replaced: the table staging of Run() in
// gpudocksm-rem-1.2/src/run.cu:114-256 (cudaMemcpy / cudaMemcpyToSymbol into
// __constant__ globals, exit() on any error).  Here every call returns a
// status and device memory belongs to reference-counted handles.
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

#include "gd_common.h"

using namespace gd;

namespace gd {

static thread_local std::string g_err;

gd_status fail(gd_status st, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}

int round_na(int na) {
  for (int v : kNAValues)
    if (v >= na) return v;
  return 0;
}

// Default launch shape (used until the autotuner has timed a size class):
// atom groups to cover the ligand and as many tile groups as fit in
// MAX_WARPS (resident or streamed, the groups split the protein's chunks).
Tile default_tile(int lna) {
  // A warp's time per protein point is about NA + 1.5 pair-slots (its atoms
  // plus the per-point loads and test), and the A x P warps share the points
  // P ways: pick the shape with the smallest (NA + 1.5) / P.
  Tile best;
  double best_cost = 1e30;
  for (int na : kNAValues) {
    const int A = (lna + na - 1) / na;
    if (A > MAX_WARPS) continue;
    const int NA = round_na((lna + A - 1) / A);
    const int P = std::max(1, MAX_WARPS / A);
    const double cost = (NA + 1.5) / P;
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best.A = A;
      best.P = P;
      best.NA = NA;
    }
  }
  return best;
}

void pick_stages(const KTables &T, const Tile &t, int *n_stages, int *resident, int split) {
  const int n_tiles = (T.pnp + TILE_PTS - 1) / TILE_PTS;
  const int own = (n_tiles + split - 1) / split;  // tiles of a split's busiest CTA
  const size_t limit = 227 * 1024;
  if (own <= MAX_RESIDENT_TILES && dock_smem_bytes(t.A, t.P, t.NA, own, split) <= limit) {
    *n_stages = own;
    *resident = 1;
  } else {
    *n_stages = STREAM_STAGES;
    *resident = 0;
  }
}

int lna_bucket(int lna) { return std::min(((lna + 7) / 8) * 8, MAX_LNA); }

int split_for(gd_ctx *ctx, const KTables &T, int run_units, double min_cost) {
  if (ctx->split_mode > 0) return ctx->split_mode;
  // the largest power of two <= cost / min_cost and <= SMs / units, at most
  // 8: a run that fills the GPU with units gains nothing from splitting
  const double cost = (double)lna_bucket(T.lna) * T.pnp;
  const int free = ctx->n_sm / std::max(1, run_units);
  int k = 1;
  while (k < 8 && cost >= min_cost * 2.0 * k && 2 * k <= free) k *= 2;
  return k;
}

int units_of(int n_prt, int n_lig, int n_tmp) {
  if (32 % n_tmp == 0) {
    const int G = 32 / n_tmp;  // ligand conformations per unit
    return n_prt * ((n_lig + G - 1) / G);
  }
  return n_prt * ((n_lig * n_tmp + 31) / 32);
}

Tile tile_for(gd_ctx *ctx, const KTables &T) {
  const int n_tiles = (T.pnp + TILE_PTS - 1) / TILE_PTS;
  const int hi = lna_bucket(T.lna);
  {
    std::lock_guard<std::mutex> g(ctx->tile_mu);
    auto it = ctx->tiles.find({hi, n_tiles});
    if (it != ctx->tiles.end()) return it->second;
  }
  return default_tile(hi);
}

void ctx_retain(gd_ctx *c) {
  if (c) c->refs++;
}

gd_status fork_streams(gd_ctx *c, int n, cudaStream_t *out) {
  n = std::max(1, std::min(n, kMaxSide));
  out[0] = c->stream;
  if (n == 1) return GD_OK;
  if (!c->forked) GD_CUDA(cudaEventCreateWithFlags(&c->forked, cudaEventDisableTiming));
  while ((int)c->side.size() < n - 1) {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    GD_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    c->side.push_back(s);
    GD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->side_done.push_back(e);
  }
  GD_CUDA(cudaEventRecord(c->forked, c->stream));
  for (int k = 1; k < n; ++k) {
    GD_CUDA(cudaStreamWaitEvent(c->side[k - 1], c->forked, 0));
    out[k] = c->side[k - 1];
  }
  return GD_OK;
}

gd_status join_streams(gd_ctx *c, int n) {
  n = std::max(1, std::min(n, kMaxSide));
  for (int k = 1; k < n; ++k) {
    GD_CUDA(cudaEventRecord(c->side_done[k - 1], c->side[k - 1]));
    GD_CUDA(cudaStreamWaitEvent(c->stream, c->side_done[k - 1], 0));
  }
  return GD_OK;
}

void ctx_release(gd_ctx *c) {
  if (!c || --c->refs > 0) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (cudaStream_t s : c->side) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : c->side_done) cudaEventDestroy(e);
  if (c->forked) cudaEventDestroy(c->forked);
  cudaFree(c->d_err);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
}

void dcx_retain(gd_dcomplex *d) {
  if (d) d->refs++;
}

// The last reference frees the tables in stream order on the context stream
// (work of the library's side streams is joined into it; the server frees a
// request only after its lane's launches have ended).
void dcx_release(gd_dcomplex *d) {
  if (!d || --d->refs > 0) return;
  if (d->ctx) {
    cudaSetDevice(d->ctx->device);
    for (void *p : d->allocs) cudaFreeAsync(p, d->ctx->stream);
  }
  gd_ctx *c = d->ctx;
  gd_dcomplex *owner = d->protein_owner;
  delete d;
  dcx_release(owner);
  ctx_release(c);
}

gd_status kernel_error(int code) {
  if (code == 3)
    return fail(GD_ECUDA, "internal: a warp needs more H-bond atom pairs than its launch "
                          "shape evaluates");
  if (code == 4)
    return fail(GD_ETIMEDOUT, "a persistent CTA gave up waiting for the earlier MC steps of "
                              "its unit (code 4)");
  return fail(GD_ETIMEDOUT, "a bounded barrier wait gave up in a kernel (code %d)", code);
}

gd_status ctx_check(gd_ctx *c) {
  int h = 0;
  GD_CUDA(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GD_CUDA(cudaStreamSynchronize(c->stream));
  if (h != 0) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
    cudaStreamSynchronize(c->stream);
    return kernel_error(h);
  }
  return GD_OK;
}

}  // namespace gd

extern "C" const char *gd_last_error(void) { return gd::g_err.c_str(); }
extern "C" const char *gd_version(void) { return "gpudock-b200 0.2 (sm_100a)"; }

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

// Rigid poses given as a translation and a rotation quaternion, as the
// move vectors of Move_d (move_d.cu:90-105): R = Rz(m3) Ry(m4) Rx(m5), so
// r00 = cos m3 cos m4, r10 = sin m3 cos m4, r20 = -sin m4, r21 = cos m4 sin m5,
// r22 = cos m4 cos m5.  Where cos m4 vanishes only m5 - m3 (m4 = pi/2) or
// m5 + m3 (m4 = -pi/2) is fixed; m3 = 0 then.  Double precision throughout.
extern "C" gd_status gd_poses_from_quaternions(int n_pose, const float *quat_poses,
                                               float *poses) {
  if (n_pose < 0 || (n_pose > 0 && (!quat_poses || !poses)))
    return fail(GD_EINVAL, "gd_poses_from_quaternions: n_pose=%d", n_pose);
  for (int i = 0; i < n_pose; ++i) {
    const float *q = quat_poses + (size_t)i * 7;
    for (int k = 0; k < 7; ++k)
      if (!std::isfinite(q[k])) return fail(GD_EINVAL, "pose %d: non-finite value", i);
    double w = q[3], x = q[4], y = q[5], z = q[6];
    const double nrm = std::sqrt(w * w + x * x + y * y + z * z);
    if (!(nrm > 0.0)) return fail(GD_EINVAL, "pose %d: zero quaternion", i);
    w /= nrm, x /= nrm, y /= nrm, z /= nrm;
    const double r00 = 1.0 - 2.0 * (y * y + z * z), r01 = 2.0 * (x * y - w * z);
    const double r10 = 2.0 * (x * y + w * z), r11 = 1.0 - 2.0 * (x * x + z * z);
    const double r20 = 2.0 * (x * z - w * y), r21 = 2.0 * (y * z + w * x);
    const double r22 = 1.0 - 2.0 * (x * x + y * y);
    const double m4 = -std::asin(std::min(1.0, std::max(-1.0, r20)));
    double m3, m5;
    if (std::hypot(r00, r10) > 1e-9) {
      m3 = std::atan2(r10, r00);
      m5 = std::atan2(r21, r22);
    } else {
      m3 = 0.0;
      m5 = r20 < 0.0 ? std::atan2(r01, r11) : std::atan2(-r01, r11);
    }
    float *m = poses + (size_t)i * 6;
    m[0] = q[0], m[1] = q[1], m[2] = q[2];
    m[3] = (float)m3, m[4] = (float)m4, m[5] = (float)m5;
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
  if (L.lna < 1 || L.lna > MAX_WARPS * MAX_NA || L.lna > MAX_LNA)
    return fail(GD_EINVAL, "ligand atoms lna=%d outside [1, %d]", L.lna,
                std::min(MAX_WARPS * MAX_NA, MAX_LNA));
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
  // single attributes (cudaGetDeviceProperties queries them all: slow)
  int major = 0, minor = 0, n_sm = 0;
  GD_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  GD_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
  GD_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
  if (major != 10)
    return fail(GD_ENODEV, "device %d is sm_%d%d; this build targets sm_100a", device, major,
                minor);
  gd_ctx *c = new (std::nothrow) gd_ctx;
  if (!c) return fail(GD_ENOMEM, "host allocation");
  c->device = device;
  c->n_sm = n_sm;
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
  // the fixed scratch of gd_energy_poses_noalloc is committed now, not on
  // that entry point's first call
  const gd_status st = noalloc_attach(c);
  if (st != GD_OK) {
    cudaFree(c->d_err);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return st;
  }
  *out = c;
  return GD_OK;
}

extern "C" gd_status gd_ctx_destroy(gd_ctx *c) {
  ctx_release(c);
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
// Stream-ordered allocation on the context stream: neither this nor the
// matching cudaFreeAsync in dcx_release synchronises the device, so a
// server uploading and releasing requests never stalls the kernels of other
// streams.
template <typename T>
static gd_status upload(gd_dcomplex *d, const std::vector<T> &h, const T **out) {
  void *p = nullptr;
  const size_t n = std::max<size_t>(h.size(), 1) * sizeof(T);
  if (injected_alloc_failure(d->ctx))
    return fail(GD_ENOMEM, "cudaMallocAsync of %zu bytes: out of memory (injected)", n);
  GD_CUDA(cudaMallocAsync(&p, n, d->ctx->stream));
  d->allocs.push_back(p);
  d->bytes += n;
  if (!h.empty())
    GD_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice,
                            d->ctx->stream));
  *out = (const T *)p;
  return GD_OK;
}

extern "C" gd_status gd_complex_free(gd_dcomplex *d) {
  dcx_release(d);
  return GD_OK;
}

extern "C" size_t gd_complex_device_bytes(const gd_dcomplex *d) { return d ? d->bytes : 0; }

// Packs the protein conformations into {x, y, z, ele} and {hpp, meta}.
// The device order of the points: those whose type forms an H-bond with
// some ligand type (hdb0 > 0.1) first, each kind in the caller's order.  The
// energy is a sum over points, so the order changes nothing but the FP32
// rounding inside a 32-point chunk.
static gd_status upload_protein(const gd_protein &P, const gd_enepara &F, gd_dcomplex *d) {
  KTables &T = d->T;
  const int pnp = P.pnp;
  const int pnp_pad = (pnp + TILE_PTS - 1) / TILE_PTS * TILE_PTS;
  bool hb_type[GD_NPT];
  for (int j = 0; j < GD_NPT; ++j) {
    hb_type[j] = false;
    for (int i = 0; i < GD_NLT; ++i) hb_type[j] = hb_type[j] || F.hdb0[i][j] > 0.1f;
  }
  std::vector<int> &order = d->point_order;
  order.clear();
  order.reserve(pnp);
  for (int pass = 0; pass < 2; ++pass)
    for (int p = 0; p < pnp; ++p)
      if (hb_type[P.t[p]] == (pass == 0)) order.push_back(p);
  std::vector<float4> pa((size_t)P.n_conf * pnp_pad,
                         make_float4(PAD_POINT_COORD, PAD_POINT_COORD, PAD_POINT_COORD, 0.f));
  for (int c = 0; c < P.n_conf; ++c)
    for (int s = 0; s < pnp; ++s) {
      const int p = order[s];
      const size_t i = (size_t)c * pnp + p;
      pa[(size_t)c * pnp_pad + s] = make_float4(P.x[i], P.y[i], P.z[i], P.ele[p]);
    }
  float pad_meta;
  {
    const uint32_t m = (uint32_t)PAD_POINT_TYPE;
    std::memcpy(&pad_meta, &m, 4);
  }
  std::vector<float2> pb((size_t)pnp_pad, make_float2(0.f, pad_meta));
  for (int s = 0; s < pnp; ++s) {
    const int p = order[s];
    uint32_t meta = (uint32_t)P.t[p] | ((uint32_t)P.c[p] << META_CLASS_SHIFT) |
                    ((uint32_t)P.seq3r[p] << META_SEQ_SHIFT);
    if (P.c0_and_d12_or_c2[p] == 1) meta |= META_HPC_BIT;
    float mf;
    std::memcpy(&mf, &meta, 4);
    pb[s] = make_float2(P.hpp[p], mf);
  }
  GD_TRY(upload(d, pa, &T.pt_a));
  GD_TRY(upload(d, pb, &T.pt_b));
  T.pnp = pnp;
  T.pnp_pad = pnp_pad;
  T.n_prt = P.n_conf;
  return GD_OK;
}

// Ligand, pocket template and force-field tables of a complex.
static gd_status upload_ligand(const gd_complex *cx, gd_dcomplex *d) {
  const gd_ligand &L = cx->lig;
  const gd_enepara &F = *cx->ff;
  KTables &T = d->T;
  const int lna = L.lna;
  // type-pair table [lig type][point type], plus an all-zero row for the
  // padding atoms of the last atom group
  std::vector<float4> ta(TAB_ROWS * GD_NPT, make_float4(0.f, 0.f, 0.f, 0.f));
  std::vector<float2> tb(TAB_ROWS * GD_NPT, make_float2(0.f, 0.f));
  float max_pmf0 = 0.f;
  for (int i = 0; i < GD_NLT; ++i)
    for (int j = 0; j < GD_NPT; ++j) {
      ta[i * GD_NPT + j] = make_float4(F.p1a[i][j], F.p2a[i][j], F.pmf0[i][j], F.pmf1[i][j]);
      tb[i * GD_NPT + j] = make_float2(F.hdb0[i][j], F.hdb1[i][j]);
      max_pmf0 = std::max(max_pmf0, F.pmf0[i][j]);
    }
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
  GD_TRY(upload(d, ta, &T.tab_a));
  GD_TRY(upload(d, tb, &T.tab_b));
  GD_TRY(upload(d, lg, &T.lig));
  GD_TRY(upload(d, lt, &T.lig_t));
  GD_TRY(upload(d, lq, &T.lig_q));
  GD_TRY(upload(d, psp, &T.psp));
  {
    // residues where some atom type of this ligand has a nonzero psp entry:
    // the kernel reads the table only there (elsewhere it adds zero)
    const int n_col = cx->psp.n_col;
    bool present[GD_NLT] = {};
    for (int a = 0; a < lna; ++a) present[L.t[a]] = true;
    std::vector<uint32_t> mask((size_t)(n_col + 31) / 32, 0u);
    for (int t = 0; t < GD_NLT; ++t)
      if (present[t])
        for (int r = 0; r < n_col; ++r)
          if (psp[(size_t)t * n_col + r] != 0.0f) mask[r >> 5] |= 1u << (r & 31);
    GD_TRY(upload(d, mask, &T.psp_mask));
  }
  GD_TRY(upload(d, kd, &T.kde));
  GD_TRY(upload(d, koff, &T.kde_off));
  GD_TRY(upload(d, mc, &T.mcs));
  GD_TRY(upload(d, tcc, &T.mcs_tcc));
  GD_TRY(upload(d, cnt, &T.mcs_cnt));

  T.lna = lna;
  T.n_lig = L.n_conf;
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
  // the close-range terms fire inside these distances: near-field
  // electrostatics el1 d < 1 (every point), hydrophobic d <= 9 (points with
  // the hpc flag), psp d <= pmf0 (class-2 points); thresholds by point kind
  // (hpc flag | class 2 << 1), squared with a margin for rounding
  const float r_ele = F.el1 > 0.f ? 1.0f / F.el1 : 1e30f;
  for (int kind = 0; kind < 4; ++kind) {
    float r = r_ele;
    if (kind & 1) r = std::max(r, 9.0f);
    if (kind & 2) r = std::max(r, max_pmf0);
    T.near4[kind] = r * r * 1.0001f + 1e-3f;
  }
  T.near_ele2 = F.el1 > 0.f ? r_ele * r_ele * 1.0001f + 1e-3f : 1e30f;
  // kernel slot order: atoms with an H-bond term (some point type with
  // hdb0 > 0.1) first, so that they share atom pairs and warps
  std::vector<int> order;
  T.n_hb = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int a = 0; a < lna; ++a) {
      bool hb = false;
      for (int j = 0; j < GD_NPT; ++j) hb = hb || F.hdb0[L.t[a]][j] > 0.1f;
      if (hb == (pass == 0)) order.push_back(a);
      if (hb && pass == 0) ++T.n_hb;
    }
  GD_TRY(upload(d, order, &T.lig_order));
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
    T.pocket[i] = cx->prt.pocket_center[i];
  }
  return GD_OK;
}

// Reference contact map of the MCC score (InitRefMatrix_d,
// calcmcc_d.cu:57-83): pairs with dst <= pmf0 for ligand conformation 0 in
// its start pose (relative coordinates + centre, util.C:230-247) against the
// complex's first protein conformation, in the reference's single-precision
// order; one bit per (atom, point), rows of pnp_pad / 32 words.
static gd_status upload_mcc_ref(const gd_complex *cx, int prt_conf, gd_dcomplex *d) {
  const gd_ligand &L = cx->lig;
  const gd_protein &P = cx->prt;
  const gd_enepara &F = *cx->ff;
  KTables &T = d->T;
  const int words = T.pnp_pad / 32;
  const int pc = prt_conf < P.n_conf ? prt_conf : 0;
  // bits are indexed by the device position of a point
  const std::vector<int> &order =
      d->protein_owner ? d->protein_owner->point_order : d->point_order;
  if ((int)order.size() != P.pnp) return fail(GD_EINVAL, "protein point order missing");
  std::vector<uint32_t> bits((size_t)L.lna * words, 0u);
  int nref = 0;
  float max_pmf0 = 0.f;
  for (int i = 0; i < GD_NLT; ++i)
    for (int j = 0; j < GD_NPT; ++j) max_pmf0 = std::max(max_pmf0, F.pmf0[i][j]);
  for (int a = 0; a < L.lna; ++a) {
    const float lx = L.x[a] + L.center[0];
    const float ly = L.y[a] + L.center[1];
    const float lz = L.z[a] + L.center[2];
    for (int s = 0; s < P.pnp; ++s) {
      const int p = order[s];
      const size_t i = (size_t)pc * P.pnp + p;
      const float dx = lx - P.x[i];
      const float dy = ly - P.y[i];
      const float dz = lz - P.z[i];
      const float dst = sqrtf(dx * dx + dy * dy + dz * dz);
      if (dst <= F.pmf0[L.t[a]][P.t[p]]) {
        bits[(size_t)a * words + (s >> 5)] |= 1u << (s & 31);
        ++nref;
      }
    }
  }
  GD_TRY(upload(d, bits, &T.mcc_ref));
  T.mcc_words = words;
  T.mcc_nref = (float)nref;
  T.near_mcc2 = max_pmf0 * max_pmf0 * 1.0001f + 1e-3f;
  return GD_OK;
}

static gd_status complex_upload_common(gd_ctx *ctx, const gd_complex *cx,
                                       const gd_dcomplex *share, int prt_conf0, int n_prt,
                                       gd_dcomplex **out) {
  if (!ctx || !out) return fail(GD_EINVAL, "gd_complex_upload: NULL argument");
  *out = nullptr;
  GD_TRY(gd_complex_validate(cx));
  if (share) {
    if (share->ctx != ctx) return fail(GD_EINVAL, "shared protein belongs to another context");
    if (share->T.pnp != cx->prt.pnp)
      return fail(GD_EINVAL, "shared protein has %d points, complex %d", share->T.pnp,
                  cx->prt.pnp);
    if (prt_conf0 < 0 || n_prt < 1 || prt_conf0 + n_prt > share->T.n_prt)
      return fail(GD_EINVAL, "conformations [%d, %d) outside the shared protein's %d", prt_conf0,
                  prt_conf0 + n_prt, share->T.n_prt);
  }
  GD_CUDA(cudaSetDevice(ctx->device));
  gd_dcomplex *d = new (std::nothrow) gd_dcomplex;
  if (!d) return fail(GD_ENOMEM, "host allocation");
  d->ctx = ctx;
  ctx_retain(ctx);
  gd_status st = GD_OK;
  try {
    if (share) {
      d->protein_owner = const_cast<gd_dcomplex *>(share);
      dcx_retain(d->protein_owner);
      d->T.pt_a = share->T.pt_a + (size_t)prt_conf0 * share->T.pnp_pad;
      d->T.pt_b = share->T.pt_b;
      d->T.pnp = share->T.pnp;
      d->T.pnp_pad = share->T.pnp_pad;
      d->T.n_prt = n_prt;
    } else {
      st = upload_protein(cx->prt, *cx->ff, d);
    }
    if (st == GD_OK) st = upload_ligand(cx, d);
    if (st == GD_OK) st = upload_mcc_ref(cx, share ? prt_conf0 : 0, d);
    if (st == GD_OK) {
      cudaError_t e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) st = fail(GD_ECUDA, "upload: %s", cudaGetErrorString(e));
    }
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation while packing the complex");
  }
  if (st != GD_OK) {
    dcx_release(d);
    return st;
  }
  *out = d;
  return GD_OK;
}

extern "C" gd_status gd_complex_upload(gd_ctx *ctx, const gd_complex *cx, gd_dcomplex **out) {
  NvtxRange nvtx("gd_complex_upload");
  return complex_upload_common(ctx, cx, nullptr, 0, 0, out);
}

extern "C" gd_status gd_complex_upload_shared(gd_ctx *ctx, const gd_complex *cx,
                                              const gd_dcomplex *protein, int prt_conf0,
                                              int n_prt, gd_dcomplex **out) {
  if (!protein) return fail(GD_EINVAL, "gd_complex_upload_shared: protein is NULL");
  return complex_upload_common(ctx, cx, protein, prt_conf0, n_prt, out);
}

// ---------------------------------------------------------------------------
// Pose energies
// ---------------------------------------------------------------------------
static gd_status poses_launch(gd_ctx *ctx, const gd_dcomplex *d, const Tile &tile, int prt_conf,
                              int lig_conf, int n_pose, const float *poses, float *terms,
                              double *raw, KItem **d_item) {
  KRun R{};
  R.mode = KMODE_POSES;
  R.A = tile.A;
  R.P = tile.P;
  pick_stages(d->T, tile, &R.n_stages, &R.resident);
  R.prt_conf = prt_conf;
  R.lig_conf = lig_conf;
  R.n_pose = n_pose;
  R.poses = poses;
  R.terms = terms;
  R.raw = raw;
  R.err = ctx->d_err;
  R.hb_pairs = hb_pairs_of(d->T, tile.A);
  KItem it{};
  it.T = d->T;
  it.n_tmp = 1;
  it.n_lig_conf = d->T.n_lig;
  it.n_prt = d->T.n_prt;
  GD_CUDA(cudaMallocAsync((void **)d_item, sizeof(KItem), ctx->stream));
  GD_CUDA(cudaMemcpyAsync(*d_item, &it, sizeof(KItem), cudaMemcpyHostToDevice, ctx->stream));
  R.items = *d_item;
  GD_CUDA(launch_dock(R, tile.NA, (n_pose + 31) / 32, ctx->stream));
  ctx->launches += 1;
  return GD_OK;
}

extern "C" gd_status gd_energy_poses_dev(gd_ctx *ctx, const gd_dcomplex *d, int prt_conf,
                                         int lig_conf, int n_pose, const float *poses,
                                         float *terms, double *raw) {
  NvtxRange nvtx("gd_energy_poses_dev");
  if (!ctx || !d) return fail(GD_EINVAL, "gd_energy_poses_dev: NULL handle");
  if (n_pose < 0) return fail(GD_EINVAL, "n_pose=%d", n_pose);
  if (prt_conf < 0 || prt_conf >= d->T.n_prt)
    return fail(GD_EINVAL, "prt_conf %d outside [0, %d)", prt_conf, d->T.n_prt);
  if (lig_conf < 0 || lig_conf >= d->T.n_lig)
    return fail(GD_EINVAL, "lig_conf %d outside [0, %d)", lig_conf, d->T.n_lig);
  if (n_pose == 0) return GD_OK;
  if (!poses || !terms) return fail(GD_EINVAL, "poses/terms NULL");
  GD_CUDA(cudaSetDevice(ctx->device));
  KItem *dit = nullptr;
  gd_status st = poses_launch(ctx, d, tile_for(ctx, d->T), prt_conf, lig_conf, n_pose, poses,
                              terms, raw, &dit);
  if (dit) cudaFreeAsync(dit, ctx->stream);
  return st;
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

extern "C" gd_status gd_ctx_set_tile(gd_ctx *ctx, int lna, int pnp, const gd_tile *tile) {
  if (!ctx || !tile) return fail(GD_EINVAL, "gd_ctx_set_tile: NULL argument");
  Tile t;
  t.A = tile->atom_groups;
  t.P = tile->tile_groups;
  t.NA = tile->atoms_per_warp;
  if (!t.valid() || t.A * t.P > MAX_WARPS || round_na(t.NA) != t.NA ||
      t.A * t.NA < lna_bucket(lna))
    return fail(GD_EINVAL, "tile %dx%d with %d atoms per warp does not cover %d atoms", t.A, t.P,
                t.NA, lna);
  std::lock_guard<std::mutex> g(ctx->tile_mu);
  ctx->tiles[{lna_bucket(lna), (pnp + TILE_PTS - 1) / TILE_PTS}] = t;
  return GD_OK;
}

extern "C" gd_status gd_ctx_set_schedule(gd_ctx *ctx, int mode, int machines) {
  if (!ctx) return fail(GD_EINVAL, "gd_ctx_set_schedule: NULL context");
  if (mode < GD_SCHED_AUTO || mode > GD_SCHED_PERSISTENT)
    return fail(GD_EINVAL, "gd_ctx_set_schedule: unknown mode %d", mode);
  if (machines < 0) return fail(GD_EINVAL, "gd_ctx_set_schedule: machines=%d", machines);
  ctx->sched_mode = mode;
  ctx->sched_machines = machines;
  return GD_OK;
}

extern "C" gd_status gd_ctx_set_schedule_tail(gd_ctx *ctx, int tail) {
  if (!ctx) return fail(GD_EINVAL, "gd_ctx_set_schedule_tail: NULL context");
  if (tail < 0 || tail > 64) return fail(GD_EINVAL, "gd_ctx_set_schedule_tail: tail=%d", tail);
  ctx->sched_tail = tail;
  return GD_OK;
}

extern "C" gd_status gd_ctx_set_split(gd_ctx *ctx, int split) {
  if (!ctx) return fail(GD_EINVAL, "gd_ctx_set_split: NULL context");
  if (split < 0 || split > 8 || (split & (split - 1)))
    return fail(GD_EINVAL, "gd_ctx_set_split: %d is not 0, 1, 2, 4 or 8", split);
  ctx->split_mode = split;
  return GD_OK;
}

extern "C" gd_status gd_ctx_set_wait_test(gd_ctx *c, unsigned wait_limit, int never_release) {
  if (!c) return fail(GD_EINVAL, "ctx is NULL");
  if (never_release && wait_limit == 0)
    return fail(GD_EINVAL, "gd_ctx_set_wait_test: never_release needs a wait limit");
  c->wait_limit = wait_limit;
  // no run reaches this many MC steps, so a wait for it can only run out
  c->wait_bias = never_release ? (1 << 30) : 0;
  return GD_OK;
}

extern "C" gd_status gd_ctx_set_alloc_fail(gd_ctx *c, int nth) {
  if (!c) return fail(GD_EINVAL, "ctx is NULL");
  if (nth < 0) return fail(GD_EINVAL, "gd_ctx_set_alloc_fail: nth=%d", nth);
  c->alloc_fail_in.store(nth);
  return GD_OK;
}

extern "C" gd_status gd_schedule_queue(const double *cost, const int *steps, int n_units,
                                       int machines, int tail, int *pieces, int cap,
                                       int *piece_off, int *n_queue) {
  if (n_units < 0 || machines < 1 || tail < 0 || cap < 0 || !piece_off || !n_queue ||
      (n_units > 0 && (!cost || !steps || !pieces)))
    return fail(GD_EINVAL, "gd_schedule_queue: bad arguments");
  std::vector<double> c(cost, cost + n_units);
  std::vector<int> s(steps, steps + n_units);
  for (int u = 0; u < n_units; ++u)
    if (!(c[u] > 0.0) || s[u] < 0)
      return fail(GD_EINVAL, "gd_schedule_queue: unit %d has cost %g, %d steps", u, c[u], s[u]);
  std::vector<int4> pc;
  std::vector<int> off;
  int nq = 0;
  schedule_queue(c, s, machines, tail, &pc, &off, &nq);
  if ((int)pc.size() > cap)
    return fail(GD_EINVAL, "gd_schedule_queue: %zu pieces exceed cap %d", pc.size(), cap);
  for (size_t k = 0; k < pc.size(); ++k) {
    pieces[4 * k] = pc[k].x;
    pieces[4 * k + 1] = pc[k].y;
    pieces[4 * k + 2] = pc[k].z;
    pieces[4 * k + 3] = pc[k].w;
  }
  for (int k = 0; k <= machines; ++k) piece_off[k] = off[k];
  *n_queue = nq;
  return GD_OK;
}

extern "C" gd_status gd_schedule_pieces(const double *cost, const int *steps, int n_units,
                                        int machines, int *pieces, int cap, int *piece_off,
                                        int *n_used) {
  if (n_units < 0 || machines < 1 || cap < 0 || !piece_off || !n_used ||
      (n_units > 0 && (!cost || !steps || !pieces)))
    return fail(GD_EINVAL, "gd_schedule_pieces: bad arguments");
  std::vector<double> c(cost, cost + n_units);
  std::vector<int> s(steps, steps + n_units);
  for (int u = 0; u < n_units; ++u)
    if (!(c[u] > 0.0) || s[u] < 0)
      return fail(GD_EINVAL, "gd_schedule_pieces: unit %d has cost %g, %d steps", u, c[u], s[u]);
  std::vector<int4> pc;
  std::vector<int> off;
  const int used = schedule_pieces(c, s, machines, &pc, &off);
  if ((int)pc.size() > cap)
    return fail(GD_EINVAL, "gd_schedule_pieces: %zu pieces exceed cap %d", pc.size(), cap);
  for (size_t k = 0; k < pc.size(); ++k) {
    pieces[4 * k] = pc[k].x;
    pieces[4 * k + 1] = pc[k].y;
    pieces[4 * k + 2] = pc[k].z;
    pieces[4 * k + 3] = pc[k].w;
  }
  for (int m = 0; m <= used; ++m) piece_off[m] = off[m];
  *n_used = used;
  return GD_OK;
}

namespace gd {

int schedule_pieces(const std::vector<double> &cost, const std::vector<int> &steps, int m,
                    std::vector<int4> *pieces, std::vector<int> *piece_off) {
  pieces->clear();
  piece_off->assign(1, 0);
  double total = 0.0, longest = 0.0;
  for (size_t u = 0; u < cost.size(); ++u) {
    const double p = cost[u] * std::max(steps[u], 0);
    total += p;
    longest = std::max(longest, p);
  }
  if (total <= 0.0 || m < 1) return 0;
  const double C = std::max(longest, total / m);
  // line order: machine k holds [k C, (k+1) C) of the units laid end to end
  std::vector<std::vector<int4>> mach(1);
  double pos = 0.0;  // line length placed so far (cuts are rounded against
                     // the ideal boundaries, so rounding does not accumulate)
  for (size_t u = 0; u < cost.size(); ++u) {
    const int n = steps[u];
    const double c = cost[u];
    int lo = 0;
    while (lo < n) {
      const double end = C * (double)mach.size();  // this machine's boundary
      int s = (int)std::floor((end - pos) / c + 0.5);  // steps that fit, rounded
      if (s >= n - lo || (int)mach.size() == m) s = n - lo;
      if (s <= 0) {  // the machine is full: the unit starts the next one
        mach.emplace_back();
        continue;
      }
      mach.back().push_back(make_int4((int)u, lo, lo + s, lo > 0 ? 1 : 0));
      lo += s;
      pos += s * c;
      if (lo < n) mach.emplace_back();  // cut: the rest opens the next machine
    }
  }
  while (!mach.empty() && mach.back().empty()) mach.pop_back();
  // run order is the reverse of line order: a cut unit's first steps open
  // the lower machine, its last steps close the next one
  for (auto &v : mach) {
    for (auto p = v.rbegin(); p != v.rend(); ++p) pieces->push_back(*p);
    piece_off->push_back((int)pieces->size());
  }
  return (int)mach.size();
}

int schedule_queue(const std::vector<double> &cost, const std::vector<int> &steps, int m, int tail,
                   std::vector<int4> *pieces, std::vector<int> *piece_off, int *n_queue) {
  const size_t n = cost.size();
  std::vector<int> head(n);
  for (size_t u = 0; u < n; ++u) head[u] = std::max(0, steps[u] - std::max(tail, 0));
  const int used = schedule_pieces(cost, head, m, pieces, piece_off);
  // when each unit's first part ends, along its machine's list (cost units)
  std::vector<double> ready(n, 0.0);
  for (int k = 0; k < used; ++k) {
    double t = 0.0;
    for (int q = (*piece_off)[k]; q < (*piece_off)[k + 1]; ++q) {
      const int4 &pz = (*pieces)[q];
      t += cost[pz.x] * (pz.z - pz.y);
      if (pz.z == head[pz.x]) ready[pz.x] = t;
    }
  }
  while ((int)piece_off->size() < m + 1) piece_off->push_back(piece_off->back());
  std::vector<int> order(n);
  for (size_t u = 0; u < n; ++u) order[u] = (int)u;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return ready[a] < ready[b]; });
  *n_queue = 0;
  for (int j = 0; j < tail; ++j)
    for (int u : order)
      if (head[u] + j < steps[u]) {
        const int lo = head[u] + j;
        pieces->push_back(make_int4(u, lo, lo + 1, lo > 0 ? 1 : 0));
        *n_queue += 1;
      }
  return m;
}

}  // namespace gd

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
