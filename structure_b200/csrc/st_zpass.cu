// st_zpass.cu -- the data pass of a sweep: one read of the genotypes that
// draws every allele copy's population of origin Z (Updates/UpdateZ.c:13-56,
// mymath.c:105-129), histograms the draws into the allele counts n[l][k][a]
// (Updates/UpdateP.c:60-99 GetNumFromPops) and ancestry counts m[i][k]
// (Updates/UpdateQ.c:17-35 GetNumLociPop) for the next sweep's P and Q
// updates, and, when asked, reduces ln P(D|Q,P) (CalcLike.c:75-133,387-426).
// The same tiling serves the Metropolis Q move's likelihood ratio
// (CalcLike.c:281-345) and the initial random Z (Init.c:125-169).
//
// Fast path (biallelic, 2 bits per genotype, locus-major rows):
//   CTA = W warps; lane = one locus; each warp walks the T individuals of its
//   chunk, 16 genotypes per 32-bit word.  P[l][k][0..1] lives in registers,
//   Q rows of the chunk in shared memory (broadcast reads).  n[l][k][a] is a
//   lane-private shared-memory histogram (lane-minor, conflict-free); m[i][k]
//   is reduced across the warp's 32 loci with one redux.sync per step on
//   7-bit packed fields.  Counts are added into one histogram per chain,
//   n[k][a][l] and m[i][k], with integer reductions (cleared by the host
//   before the pass); the Metropolis log ratios leave as per-CTA partials
//   ldpart[group][i].
#include <cstdio>
#include "st_device.cuh"
#include "st_kernels.h"

namespace st {

namespace {

constexpr float kLikeTinyF = 1e-30f;

// Deterministic block sum of one double per thread (fixed tree order).
__device__ __forceinline__ double block_sum_d(double v, double* sred) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sred[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; w++) s += sred[w];
  }
  return s;  // valid in thread 0
}

// Last CTA of a chain: sum the per-CTA ln-likelihood partials in a fixed
// order (each thread a compensated sum of a strided subset, then the block's
// tree) and fold them into the chain's stats.
static __device__ void finish_like(ChainDev& ch, int ntiles, bool collect, double* sred) {
  CompSum v;
  for (int j = threadIdx.x; j < ntiles; j += blockDim.x) v.add(ch.likepart[j]);
  double s = block_sum_d(v.value(), sred);
  if (threadIdx.x == 0) {
    ch.stats[kStLike] = s;
    if (collect) {
      ch.stats[kStSumLikes] += s;
      ch.stats[kStSumSq] += s * s;
      ch.stats[kStNLike] += 1.0;
    }
  }
}

}  // namespace

namespace zfast {
template <int KT, int W>
cudaError_t launch_b2g_kw(const LaunchSet& ls, int mode, int flags, size_t smem);
size_t zlayout_total(int KT, int K, int T, int nw32, int mode);
}  // namespace zfast

int ctas_zpass_b2g(const ChainDev& c) { return c.nchunks * c.ngroups; }

size_t zpass_b2g_smem(int KT, int K, int T, int W, int mode) {
  return zfast::zlayout_total(KT, K, T, 32 * W, mode);
}

int zpass_b2g_width(int KT) { return KT <= 12 ? 8 : 2; }

// smem must be sized for the largest tile among the chains of the launch; the
// CTA width is fixed per K class (zpass_b2g_width).
cudaError_t launch_zpass_b2g(const LaunchSet& ls, int KT, int W, int mode, int flags,
                             size_t smem) {
  if (W != zpass_b2g_width(KT)) return cudaErrorInvalidConfiguration;
  switch (KT) {
#define ST_KCASE(k, w) case k: return zfast::launch_b2g_kw<k, w>(ls, mode, flags, smem);
    ST_KCASE(1, 8) ST_KCASE(2, 8) ST_KCASE(3, 8) ST_KCASE(4, 8) ST_KCASE(5, 8) ST_KCASE(6, 8)
    ST_KCASE(7, 8) ST_KCASE(8, 8) ST_KCASE(9, 8) ST_KCASE(10, 8) ST_KCASE(11, 8) ST_KCASE(12, 8)
    ST_KCASE(16, 2) ST_KCASE(20, 2) ST_KCASE(24, 2) ST_KCASE(32, 2)
#undef ST_KCASE
  }
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Generic path: one thread per (individual, locus), any allele count, runtime
// K, FP32 or FP64 arithmetic, Philox or injected uniforms.  Counts go to slice
// 0 of the partial arrays with global atomics (zeroed by the host before).
// ---------------------------------------------------------------------------
template <typename TF>
__device__ __forceinline__ int pick_generic(const float* q, const float* Pl, int K, int A,
                                            int a, TF u, TF& total, int& errb);

template <>
__device__ __forceinline__ int pick_generic<float>(const float* q, const float* Pl, int K, int A,
                                                   int a, float u, float& total, int& errb) {
  float C[kMaxPops];
  C[0] = q[0] * Pl[a];
  for (int k = 1; k < K; k++) C[k] = __fmaf_rn(q[k], Pl[(size_t)k * A + a], C[k - 1]);
  total = C[K - 1];
  const float r = u * total;
  int z = 0;
  for (int k = 0; k < K - 1; k++) z += (C[k] < r);
  return z;
}

template <>
__device__ __forceinline__ int pick_generic<double>(const float* q, const float* Pl, int K, int A,
                                                    int a, double u, double& total, int& errb) {
  double Wt[kMaxPops];
  double sum = 0.0;
  for (int k = 0; k < K; k++) {
    Wt[k] = __dmul_rn((double)q[k], (double)Pl[(size_t)k * A + a]);
    sum = __dadd_rn(sum, Wt[k]);
  }
  total = sum;
  const double r = __dadd_rn(0.0, __dmul_rn(u, __dadd_rn(sum, -0.0)));
  double so = 0.0;
  int k = 0;
  for (; k < K; k++) {
    so = __dadd_rn(so, Wt[k]);
    if (r <= so) break;
  }
  if (k == K) { k = K - 1; errb |= kErrFallThrough; }
  return k;
}

template <typename TF>
__global__ void __launch_bounds__(256)
zpass_u8_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix, int nchains,
                int mode, int flags) {
  __shared__ double sred[8];
  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int N = ch.N, L = ch.L, K = ch.K, A = ch.A;
  const size_t idx = (size_t)tile * blockDim.x + threadIdx.x;
  const bool active = idx < (size_t)N * L;
  const int i = active ? (int)(idx / L) : 0;
  const int l = active ? (int)(idx - (size_t)i * L) : 0;
  const int rep = *ch.rep;
  const bool collect = rep + 1 > ch.burnin;
  const bool want_like = (mode == kZLike) ||
      (mode == kZNormal && ((flags & kZfLikeAlways) || ((flags & kZfLikeIfCollect) && collect)));
  const bool injected = (flags & kZfInjected) && ch.injected;
  int errb = 0;
  double like_acc = 0.0;

  if (active) {
    const uint8_t gv[2] = {ch.g8[((size_t)i * 2) * L + l], ch.g8[((size_t)i * 2 + 1) * L + l]};
    const float* q = ch.Q + (size_t)i * K;
    const float* Pl = ch.P + (size_t)l * K * A;
    U4 r4 = {0, 0, 0, 0};
    if (!injected && (mode == kZNormal || mode == kZInit))
      r4 = philox_s((uint32_t)l, (uint32_t)(i >> 1), mode == kZInit ? 0u : (uint32_t)rep,
                    mode == kZInit ? (uint32_t)kSInitZ : (uint32_t)kSZ, ch.key);
    const uint32_t wsel[2] = {(i & 1) ? r4.z : r4.x, (i & 1) ? r4.w : r4.y};
    int taken = 0;
    double ld = 0.0;
    for (int line = 0; line < 2; line++) {
      const int a = gv[line];
      const bool miss = a == kG8Missing;
      int z = 0;
      if (mode == kZNormal || mode == kZLike) {
        if (miss) { if (ch.Z && (flags & kZfStoreZ)) ch.Z[((size_t)i * 2 + line) * L + l] = kZMissing; continue; }
        TF total;
        TF u;
        if (injected) u = (TF)ch.injected[(size_t)i * L * 2 + (size_t)l * 2 + taken];
        else u = (TF)u23(wsel[line]);
        taken++;
        z = pick_generic<TF>(q, Pl, K, A, a, u, total, errb);
        if (want_like) like_acc += log(fmax((double)total, 1e-50));
      } else if (mode == kZInit) {
        if (miss) { if (ch.Z && (flags & kZfStoreZ)) ch.Z[((size_t)i * 2 + line) * L + l] = kZMissing; continue; }
        z = (int)(((uint64_t)(wsel[line] >> 1) * (uint64_t)K) >> 31);
        // USEPOPINFO: start at the given population (src/Init.c:74-117)
        if (ch.initpop && ch.initpop[i] >= 0) z = ch.initpop[i];
      } else if (mode == kZRecount) {
        if (miss) continue;
        z = ch.Z[((size_t)i * 2 + line) * L + l];
        if (z >= K) { errb |= kErrBounds; continue; }
      } else if (mode == kZMetro) {
        if (miss) continue;
        double tp = 0.0, tm = 0.0;
        for (int k = 0; k < K; k++) {
          const double p = (double)Pl[(size_t)k * A + a];
          tp += (double)ch.TestQ[(size_t)i * K + k] * p;
          tm += (double)q[k] * p;
        }
        ld += log(tp) - log(tm);
        continue;
      }
      if (mode == kZNormal || mode == kZInit || mode == kZRecount) {
        if (mode != kZRecount && ch.Z && (flags & kZfStoreZ))
          ch.Z[((size_t)i * 2 + line) * L + l] = (uint8_t)z;
        if (mode == kZLike) continue;
        atomicAdd(&ch.mpart[(size_t)i * K + z], 1);
        if (!ch.pfrompopflagonly || ch.popflags[i] == 1)
          atomicAdd(&ch.npart[((size_t)z * A + a) * L + l], 1);
      }
    }
    if (mode == kZMetro) atomicAdd(&ch.ldpart[i], ld);
  }
  if (errb) set_err(ch.err, errb);
  const int ntiles = (int)(((size_t)N * L + blockDim.x - 1) / blockDim.x);
  if (want_like) {
    double s = block_sum_d(like_acc, sred);
    if (threadIdx.x == 0) ch.likepart[tile] = s;
  }
  const bool advance = (flags & kZfAdvance) != 0;
  if (want_like || advance) {
    if (last_cta_arrive(&ch.ctr[kCtrZ], (unsigned)ntiles)) {
      if (want_like) finish_like(ch, ntiles, collect && (flags & kZfCollect), sred);
      if (advance && threadIdx.x == 0) *ch.rep = rep + 1;
    }
  }
}

int ctas_zpass_u8(const ChainDev& c, int block) {
  return (int)(((size_t)c.N * c.L + block - 1) / block);
}

cudaError_t launch_zpass_u8(const LaunchSet& ls, int mode, int flags) {
  dim3 grid(ls.total_ctas), block(256);
  if (flags & kZfF64)
    zpass_u8_kernel<double><<<grid, block, 0, ls.stream>>>(ls.chains, ls.prefix, ls.nchains, mode, flags);
  else
    zpass_u8_kernel<float><<<grid, block, 0, ls.stream>>>(ls.chains, ls.prefix, ls.nchains, mode, flags);
  return cudaGetLastError();
}

// int32 reference genotypes (-9 missing) -> one byte per copy (0xFF missing).
__global__ void pack_u8_kernel(const int32_t* __restrict__ geno, uint8_t* __restrict__ g8, size_t n) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    const int v = geno[j];
    g8[j] = (v < 0 || v > 254) ? kG8Missing : (uint8_t)v;
  }
}

cudaError_t launch_pack_u8(const int32_t* geno, uint8_t* g8, size_t n, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  pack_u8_kernel<<<blocks, 256, 0, s>>>(geno, g8, n);
  return cudaGetLastError();
}

// Clears the allele and ancestry histograms (n [K][A][L], m [N][K]) of every
// chain of a batch before the counting Z pass: one launch, blockIdx.y = chain.
__global__ void clear_counts_kernel(const ChainDev* __restrict__ chains) {
  const ChainDev& ch = chains[blockIdx.y];
  const size_t nn = (size_t)ch.K * ch.A * ch.L, nm = (size_t)ch.N * ch.K;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < nn + nm; j += stride) {
    if (j < nn) ch.npart[j] = 0;
    else ch.mpart[j - nn] = 0;
  }
}

cudaError_t launch_clear_counts(const ChainDev* d_table, int nchains, cudaStream_t s) {
  clear_counts_kernel<<<dim3(64, nchains), 256, 0, s>>>(d_table);
  return cudaGetLastError();
}

}  // namespace st
