// gd_noalloc.cu -- pose energies without any device allocation.
//
// gd_energy_poses (host buffers) stages its poses, terms and raw sums, and the
// launch's item descriptor, in memory it obtains from cudaMallocAsync for each
// call. gd_energy_poses_noalloc computes the same thing with the same kernel
// but stages everything in one fixed file-scope device array, so it never
// calls an allocator. The array is sized for GD_NOALLOC_MAX_POSES poses per
// call; larger calls are rejected before anything is launched.
//
// Scratch layout (each section starts on a 256-byte boundary):
//   [KItem descriptor][poses  max x 6 f32][terms  max x 10 f32][raw  max x 9 f64]
// Every byte the kernel reads from it (descriptor, poses) is written by the
// call before the launch, and the kernel writes every terms/raw element of the
// n_pose poses it is given, so nothing in it has to start at zero.
#include <cstring>

#include "gd_common.h"

namespace {

using gd::KItem;
using gd::KRun;

constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

constexpr size_t kItemBytes = align256(sizeof(KItem));
constexpr size_t kPoseBytes = align256(sizeof(float) * 6 * GD_NOALLOC_MAX_POSES);
constexpr size_t kTermBytes = align256(sizeof(float) * GD_NTERM * GD_NOALLOC_MAX_POSES);
constexpr size_t kRawBytes = align256(sizeof(double) * GD_NRAW * GD_NOALLOC_MAX_POSES);
constexpr size_t kScratchBytes = kItemBytes + kPoseBytes + kTermBytes + kRawBytes;
static_assert(kScratchBytes < (3u << 20), "pose scratch is meant to stay a few MB");

// One copy per device (each device's context has its own instance).
static __device__ __align__(256) unsigned char g_pose_scratch[kScratchBytes];

}  // namespace

// Module loading is lazy (CUDA 12): the module that holds g_pose_scratch is
// loaded, and the array committed on the device, the first time anything of
// it is touched.  Touching it here, when the context is created, means that
// a later gd_energy_poses_noalloc call neither loads a module nor commits
// memory.  The address belongs to the CUDA context current now; a gd_ctx
// does not outlive that context (after cudaDeviceReset, create a new gd_ctx).
gd_status gd::noalloc_attach(gd_ctx *c) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_pose_scratch);
  if (e != cudaSuccess || !p)
    return gd::fail(e == cudaErrorMemoryAllocation ? GD_ENOMEM : GD_ECUDA,
                    "gd_ctx_create: address of the pose scratch array: %s",
                    cudaGetErrorString(e));
  c->noalloc_scratch = static_cast<unsigned char *>(p);
  return GD_OK;
}

extern "C" gd_status gd_energy_poses_noalloc(gd_ctx *ctx, const gd_dcomplex *d, int prt_conf,
                                             int lig_conf, int n_pose, const float *poses,
                                             float *terms, double *raw) {
  if (!ctx || !d) return gd::fail(GD_EINVAL, "gd_energy_poses_noalloc: NULL handle");
  if (n_pose < 0) return gd::fail(GD_EINVAL, "gd_energy_poses_noalloc: n_pose=%d", n_pose);
  if (n_pose > GD_NOALLOC_MAX_POSES)
    return gd::fail(GD_EINVAL,
                    "gd_energy_poses_noalloc: n_pose=%d exceeds the %d poses its fixed "
                    "scratch holds; split the call or use gd_energy_poses",
                    n_pose, GD_NOALLOC_MAX_POSES);
  // an empty call succeeds whatever the indices, as gd_energy_poses does
  if (n_pose == 0) return GD_OK;
  if (prt_conf < 0 || prt_conf >= d->T.n_prt)
    return gd::fail(GD_EINVAL, "prt_conf %d outside [0, %d)", prt_conf, d->T.n_prt);
  if (lig_conf < 0 || lig_conf >= d->T.n_lig)
    return gd::fail(GD_EINVAL, "lig_conf %d outside [0, %d)", lig_conf, d->T.n_lig);
  if (!poses || !terms) return gd::fail(GD_EINVAL, "poses/terms NULL");
  unsigned char *base = ctx->noalloc_scratch;
  if (!base) return gd::fail(GD_EINVAL, "gd_energy_poses_noalloc: context has no scratch address");
  GD_CUDA(cudaSetDevice(ctx->device));
  KItem *d_item = reinterpret_cast<KItem *>(base);
  float *d_poses = reinterpret_cast<float *>(base + kItemBytes);
  float *d_terms = reinterpret_cast<float *>(base + kItemBytes + kPoseBytes);
  double *d_raw = reinterpret_cast<double *>(base + kItemBytes + kPoseBytes + kTermBytes);

  const gd::Tile tile = gd::tile_for(ctx, d->T);
  KRun R{};
  R.mode = gd::KMODE_POSES;
  R.A = tile.A;
  R.P = tile.P;
  gd::pick_stages(d->T, tile, &R.n_stages, &R.resident);
  R.prt_conf = prt_conf;
  R.lig_conf = lig_conf;
  R.n_pose = n_pose;
  R.poses = d_poses;
  R.terms = d_terms;
  R.raw = raw ? d_raw : nullptr;
  R.err = ctx->d_err;
  R.hb_pairs = gd::hb_pairs_of(d->T, tile.A);
  R.items = d_item;
  KItem it{};
  it.T = d->T;
  it.n_tmp = 1;
  it.n_lig_conf = d->T.n_lig;
  it.n_prt = d->T.n_prt;

  const size_t pose_b = sizeof(float) * 6 * (size_t)n_pose;
  GD_CUDA(cudaMemcpyAsync(d_item, &it, sizeof(KItem), cudaMemcpyHostToDevice, ctx->stream));
  GD_CUDA(cudaMemcpyAsync(d_poses, poses, pose_b, cudaMemcpyHostToDevice, ctx->stream));
  GD_CUDA(gd::launch_dock(R, tile.NA, (n_pose + 31) / 32, ctx->stream));
  ctx->launches += 1;
  cudaError_t e = cudaMemcpyAsync(terms, d_terms, sizeof(float) * GD_NTERM * (size_t)n_pose,
                                  cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && raw)
    e = cudaMemcpyAsync(raw, d_raw, sizeof(double) * GD_NRAW * (size_t)n_pose,
                        cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(ctx->stream);
    return gd::fail(GD_ECUDA, "gd_energy_poses_noalloc: copy back: %s", cudaGetErrorString(e));
  }
  return gd::ctx_check(ctx);
}
