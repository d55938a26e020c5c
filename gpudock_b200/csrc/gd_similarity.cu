// gd_similarity.cu -- contact-mode similarity of trajectory conformations:
// the similarity matrix of SimilarityMatirxGen (src/util.C:37-87
// CalculateSimilarityMatrix, :90-110 InitConfMatrix, :146-193
// CalculateContactModeScore).
//
// Entry (i, j) is the Matthews correlation of conformation j's contacts
// against conformation i's contact map, where a contact is a ligand-atom /
// protein-point pair with dst <= pmf0[ligand type][point type].  With A and
// B the two maps: tp = |A & B|, fn = |A| - tp, fp = |B| - tp and tn = the
// remaining pairs, so the matrix is a popcount "product" of bit maps:
//   contacts  one CTA per conformation places its ligand and writes its map,
//             32 protein points per word (a warp ballot), with its count;
//   union     the OR of all maps word by word: words that no conformation
//             sets are dropped (the maps of a trajectory near one pocket are
//             sparse and overlap);
//   gather    the kept words of every map, contiguous;
//   pairs     64 x 64 tiles of (i, j): popc(A & B) summed over the kept words
//             through shared memory, then the MCC from the four counts.
// Placement and distances follow the reference's float operations in its
// order (no contraction): the rotation comes from the host (PlaceLigand runs
// on the host in the reference, with sinf / cosf), x = r0 x + r1 y + r2 z +
// m + centre and dst = sqrtf(dx dx + dy dy + dz dz), so every contact and
// every entry is the reference's bit for bit.
#include <cmath>
#include <cstring>
#include <vector>

#include "gd_common.h"

namespace gd {
namespace {

// One conformation: rotation (row major) and translation as PlaceLigand
// uses them, and its protein and ligand conformations.
struct SimConf {
  float r[9];
  float m[3];
  int prt, lig;
  int pad[2];
};

constexpr int kSimThreads = 256;
constexpr int kPairTile = 64;   // conformations per tile side
constexpr int kPairChunk = 32;  // words per shared-memory chunk

__global__ void __launch_bounds__(kSimThreads)
    contacts_kernel(KTables T, const SimConf *confs, uint32_t *bits, int *pop, int W) {
  extern __shared__ float4 s_lig[];  // placed atoms, ligand type in .w
  __shared__ int s_pop;
  const SimConf c = confs[blockIdx.x];
  const int lna = T.lna;
  for (int l = threadIdx.x; l < lna; l += blockDim.x) {
    const float4 o = T.lig[(size_t)c.lig * lna + l];
    float v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float a = __fmul_rn(c.r[3 * k], o.x);
      a = __fadd_rn(a, __fmul_rn(c.r[3 * k + 1], o.y));
      a = __fadd_rn(a, __fmul_rn(c.r[3 * k + 2], o.z));
      a = __fadd_rn(a, c.m[k]);
      v[k] = __fadd_rn(a, T.lig_center[k]);
    }
    s_lig[l] = make_float4(v[0], v[1], v[2], __int_as_float(T.lig_t[l]));
  }
  if (threadIdx.x == 0) s_pop = 0;
  __syncthreads();
  const float4 *P = T.pt_a + (size_t)c.prt * T.pnp_pad;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t K = (size_t)lna * W;
  uint32_t *out = bits + (size_t)blockIdx.x * K;
  int my_pop = 0;
  // a warp takes 32 points (one word column) against every atom
  for (int w = warp; w < W; w += kSimThreads / 32) {
    const int s = w * 32 + lane;
    const bool valid = s < T.pnp;
    const float4 p = valid ? P[s] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int pt = valid ? (int)(__float_as_uint(T.pt_b[s].y) & META_TYPE_MASK) : 0;
    for (int l = 0; l < lna; ++l) {
      const float4 a = s_lig[l];
      const float dx = __fsub_rn(a.x, p.x);
      const float dy = __fsub_rn(a.y, p.y);
      const float dz = __fsub_rn(a.z, p.z);
      const float d2 =
          __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      const float pmf0 = T.tab_a[__float_as_int(a.w) * GD_NPT + pt].z;
      const bool hit = valid && __fsqrt_rn(d2) <= pmf0;
      const uint32_t word = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) {
        out[(size_t)l * W + w] = word;
        my_pop += __popc(word);
      }
    }
  }
  if (lane == 0) atomicAdd(&s_pop, my_pop);
  __syncthreads();
  if (threadIdx.x == 0) pop[blockIdx.x] = s_pop;
}

__global__ void union_kernel(const uint32_t *bits, int n, size_t K, uint32_t *mask) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  uint32_t m = 0u;
  for (int i = 0; i < n; ++i) m |= bits[(size_t)i * K + k];
  mask[k] = m;
}

__global__ void gather_kernel(const uint32_t *bits, int n, size_t K, const int *act, int n_act,
                              int Kp, uint32_t *comp) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * Kp) return;
  const int i = (int)(t / Kp), a = (int)(t % Kp);
  comp[t] = a < n_act ? bits[(size_t)i * K + act[a]] : 0u;
}

// CalculateContactModeScore's arithmetic: the four sums as floats multiplied
// left to right, sqrtf, and the integer numerator tp tn - fp fn (wrapping
// like the reference's int) over it; 10000 where the denominator is 0.
__device__ __forceinline__ float contact_mcc(int tp, int fn, int fp, int tn) {
  float q = __fmul_rn(__int2float_rn(tp + fp), __int2float_rn(tp + fn));
  q = __fmul_rn(q, __int2float_rn(tn + fp));
  q = __fmul_rn(q, __int2float_rn(tn + fn));
  const float dividend = __fsqrt_rn(q);
  const int num = (int)((unsigned)tp * (unsigned)tn - (unsigned)fp * (unsigned)fn);
  return dividend != 0.0f ? __fdiv_rn(__int2float_rn(num), dividend) : GD_CMCC_INVALID;
}

__global__ void __launch_bounds__(kSimThreads)
    pairs_kernel(const uint32_t *comp, const int *pop, int n, int Kp, int total, float *S) {
  __shared__ uint32_t sa[kPairTile][kPairChunk + 1];
  __shared__ uint32_t sb[kPairTile][kPairChunk + 1];
  const int i0 = blockIdx.y * kPairTile, j0 = blockIdx.x * kPairTile;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  // Carry-save counting (Harley and Seal; Mula, Kurz and Lemire, "Faster
  // population counts using AVX2 instructions", 2018): the AND words of an
  // entry are added bitwise into `ones` and `twos`; every 4 words the carry
  // out, `fours`, goes through one POPC (which issues on the XU pipe, 16 per
  // clock per SM) and the rest stays in bitwise operations.  The count is
  // 4 sum popc(fours) + 2 popc(twos) + popc(ones).
  uint32_t ones[4][4] = {}, twos[4][4] = {};
  int acc[4][4] = {};
  for (int k0 = 0; k0 < Kp; k0 += kPairChunk) {
    for (int q = tid; q < kPairTile * kPairChunk; q += kSimThreads) {
      const int row = q / kPairChunk, col = q % kPairChunk;
      const int i = i0 + row, j = j0 + row;
      sa[row][col] = i < n ? comp[(size_t)i * Kp + k0 + col] : 0u;
      sb[row][col] = j < n ? comp[(size_t)j * Kp + k0 + col] : 0u;
    }
    __syncthreads();
    for (int kk = 0; kk < kPairChunk; kk += 4) {
      uint32_t a[4][4], b[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) a[r][q] = sa[ty + 16 * r][kk + q];
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int q = 0; q < 4; ++q) b[c][q] = sb[tx + 16 * c][kk + q];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint32_t x0 = a[r][0] & b[c][0], x1 = a[r][1] & b[c][1];
          const uint32_t x2 = a[r][2] & b[c][2], x3 = a[r][3] & b[c][3];
          uint32_t &o = ones[r][c], &t = twos[r][c];
          // (twos_a, ones) = ones + x0 + x1; (twos_b, ones) = ones + x2 + x3
          uint32_t u = o ^ x0;
          const uint32_t ta = (o & x0) | (u & x1);
          o = u ^ x1;
          u = o ^ x2;
          const uint32_t tb = (o & x2) | (u & x3);
          o = u ^ x3;
          // (fours, twos) = twos + twos_a + twos_b
          u = t ^ ta;
          const uint32_t fours = (t & ta) | (u & tb);
          t = u ^ tb;
          acc[r][c] += __popc(fours);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
      acc[r][c] = 4 * acc[r][c] + 2 * __popc(twos[r][c]) + __popc(ones[r][c]);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i >= n) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = j0 + tx + 16 * c;
      if (j >= n) continue;
      const int tp = acc[r][c];
      const int fn = pop[i] - tp, fp = pop[j] - tp;
      S[(size_t)i * n + j] = contact_mcc(tp, fn, fp, total - tp - fn - fp);
    }
  }
}

// Device buffers of one call, freed on every path.
struct SimBuffers {
  cudaStream_t s;
  std::vector<void *> ptrs;
  ~SimBuffers() {
    for (void *p : ptrs) cudaFreeAsync(p, s);
  }
  template <typename T>
  cudaError_t get(T **p, size_t count) {
    void *v = nullptr;
    const cudaError_t e = cudaMallocAsync(&v, std::max<size_t>(count, 1) * sizeof(T), s);
    if (e == cudaSuccess) ptrs.push_back(v);
    *p = (T *)v;
    return e;
  }
};

}  // namespace
}  // namespace gd

using namespace gd;

// The matrix into S_dev (the caller's device memory) or, with S_dev null,
// into S_host through a buffer of its own.
static gd_status similarity_run(gd_ctx *ctx, const gd_dcomplex *d, int n_conf,
                                const float *confs, float *S_dev, float *S_host) {
  if (!ctx || !d) return fail(GD_EINVAL, "gd_similarity_matrix: NULL handle");
  if (n_conf < 0) return fail(GD_EINVAL, "n_conf=%d", n_conf);
  if (n_conf == 0) return GD_OK;
  if (!confs || (!S_dev && !S_host)) return fail(GD_EINVAL, "confs/similarity NULL");
  const KTables &T = d->T;
  if ((size_t)n_conf * (size_t)n_conf > ((size_t)1 << 40))
    return fail(GD_EINVAL, "n_conf=%d: the matrix is too large", n_conf);
  // PlaceLigand's rotation (util.C:496-535) on the host, as the reference
  std::vector<SimConf> hc((size_t)n_conf);
  for (int i = 0; i < n_conf; ++i) {
    const float *t = confs + (size_t)i * 8;
    for (int k = 0; k < 8; ++k)
      if (!std::isfinite(t[k])) return fail(GD_EINVAL, "conformation %d: non-finite value", i);
    const int prt = (int)t[0], lig = (int)t[1];
    if (prt < 0 || prt >= T.n_prt || lig < 0 || lig >= T.n_lig)
      return fail(GD_EINVAL, "conformation %d: protein %d / ligand %d out of range", i, prt,
                  lig);
    const float *m = t + 2;
    const float s1 = sinf(m[3]), c1 = cosf(m[3]);
    const float s2 = sinf(m[4]), c2 = cosf(m[4]);
    const float s3 = sinf(m[5]), c3 = cosf(m[5]);
    SimConf &c = hc[i];
    std::memset(&c, 0, sizeof(c));
    c.r[0] = c1 * c2;
    c.r[1] = c1 * s2 * s3 - c3 * s1;
    c.r[2] = s1 * s3 + c1 * c3 * s2;
    c.r[3] = c2 * s1;
    c.r[4] = c1 * c3 + s1 * s2 * s3;
    c.r[5] = c3 * s1 * s2 - c1 * s3;
    c.r[6] = -1 * s2;
    c.r[7] = c2 * s3;
    c.r[8] = c2 * c3;
    for (int k = 0; k < 3; ++k) c.m[k] = m[k];
    c.prt = prt;
    c.lig = lig;
  }
  GD_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const int W = (T.pnp + 31) / 32;
  const size_t K = (size_t)T.lna * W;
  const int total = T.lna * T.pnp;
  const size_t n = (size_t)n_conf;
  gd_status st = GD_OK;
  {
    SimBuffers B{s, {}};
    SimConf *d_conf = nullptr;
    uint32_t *d_bits = nullptr, *d_mask = nullptr;
    int *d_pop = nullptr;
    float *d_S = nullptr;
    cudaError_t e = B.get(&d_conf, n);
    if (e == cudaSuccess) e = B.get(&d_bits, n * K);
    if (e == cudaSuccess) e = B.get(&d_pop, n);
    if (e == cudaSuccess) e = B.get(&d_mask, K);
    if (e == cudaSuccess && !S_dev) e = B.get(&d_S, n * n);
    if (S_dev) d_S = S_dev;
    if (e != cudaSuccess) return fail(GD_ENOMEM, "similarity buffers: %s", cudaGetErrorString(e));
    GD_CUDA(cudaMemcpyAsync(d_conf, hc.data(), sizeof(SimConf) * n, cudaMemcpyHostToDevice, s));
    contacts_kernel<<<n_conf, kSimThreads, sizeof(float4) * T.lna, s>>>(T, d_conf, d_bits, d_pop,
                                                                       W);
    GD_CUDA(cudaGetLastError());
    union_kernel<<<(unsigned)((K + 255) / 256), 256, 0, s>>>(d_bits, n_conf, K, d_mask);
    GD_CUDA(cudaGetLastError());
    std::vector<uint32_t> mask(K);
    GD_CUDA(cudaMemcpyAsync(mask.data(), d_mask, sizeof(uint32_t) * K, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    std::vector<int> act;
    for (size_t k = 0; k < K; ++k)
      if (mask[k]) act.push_back((int)k);
    const int n_act = (int)act.size();
    const int Kp = (n_act + kPairChunk - 1) / kPairChunk * kPairChunk;
    int *d_act = nullptr;
    uint32_t *d_comp = nullptr;
    e = B.get(&d_act, act.size());
    if (e == cudaSuccess) e = B.get(&d_comp, n * (size_t)Kp);
    if (e != cudaSuccess) return fail(GD_ENOMEM, "similarity buffers: %s", cudaGetErrorString(e));
    if (n_act)
      GD_CUDA(cudaMemcpyAsync(d_act, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice,
                              s));
    if (Kp) {
      const size_t cells = n * (size_t)Kp;
      gather_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(d_bits, n_conf, K, d_act,
                                                                     n_act, Kp, d_comp);
      GD_CUDA(cudaGetLastError());
    }
    const unsigned tiles = (unsigned)((n + kPairTile - 1) / kPairTile);
    pairs_kernel<<<dim3(tiles, tiles), kSimThreads, 0, s>>>(d_comp, d_pop, n_conf, Kp, total,
                                                            d_S);
    GD_CUDA(cudaGetLastError());
    ctx->launches += Kp ? 4 : 3;
    if (!S_dev)
      GD_CUDA(cudaMemcpyAsync(S_host, d_S, sizeof(float) * n * n, cudaMemcpyDeviceToHost, s));
    st = ctx_check(ctx);
  }
  if (st == GD_OK) GD_CUDA(cudaStreamSynchronize(s));
  return st;
}

extern "C" gd_status gd_similarity_matrix(gd_ctx *ctx, const gd_dcomplex *d, int n_conf,
                                          const float *confs, float *similarity) {
  NvtxRange nvtx("gd_similarity_matrix");
  if (n_conf > 0 && !similarity) return fail(GD_EINVAL, "similarity NULL");
  return similarity_run(ctx, d, n_conf, confs, nullptr, similarity);
}

extern "C" gd_status gd_similarity_matrix_dev(gd_ctx *ctx, const gd_dcomplex *d, int n_conf,
                                              const float *confs, float *similarity_dev) {
  if (n_conf > 0 && !similarity_dev) return fail(GD_EINVAL, "similarity_dev NULL");
  return similarity_run(ctx, d, n_conf, confs, similarity_dev, nullptr);
}
