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
//   7-bit packed fields.  Counts leave as per-CTA partials (plain stores, no
//   global atomics): npart[chunk][k][a][l] and mpart[group][i][k], summed by
//   the consumers.
#include <cstdio>
#include "st_device.cuh"
#include "st_kernels.h"

namespace st {

namespace {

constexpr float kLikeTinyF = 1e-30f;

__device__ __forceinline__ float like_term(float T0, float T1) {
  // ln of the two copies' mixture probabilities, each clamped at
  // sqrt(UNDERFLO) = 1e-50 like CalcLikeInd (CalcLike.c:113-118).
  float pr = T0 * T1;
  if (pr > kLikeTinyF) return __logf(pr);
  return (float)(log(fmax((double)T0, 1e-50)) + log(fmax((double)T1, 1e-50)));
}

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

// Last CTA of a chain: sum the per-CTA ln-likelihood partials in order and
// fold them into the chain's stats.
__device__ void finish_like(ChainDev& ch, int ntiles, bool collect, double* sred) {
  double v = 0.0;
  for (int j = threadIdx.x; j < ntiles; j += blockDim.x) v += ch.likepart[j];
  double s = block_sum_d(v, sred);
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

// ---------------------------------------------------------------------------
// Fast path
// ---------------------------------------------------------------------------
template <int KT, int MODE>
__global__ void __launch_bounds__(256)
zpass_b2g_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix,
                 int nchains, int flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double sred[8];
  constexpr int KS = (KT + 3) & ~3;
  constexpr int NWM = (KT + 3) / 4;
  constexpr bool kUseP = (MODE == kZNormal || MODE == kZMetro || MODE == kZLike);
  constexpr bool kCounts = (MODE == kZNormal || MODE == kZInit || MODE == kZRecount);

  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int T = ch.tileT, R = ch.tileR;
  const int W = blockDim.x >> 5;
  const int nw32 = blockDim.x;
  const int ichunk = tile % ch.nchunks, grp = tile / ch.nchunks;
  const int N = ch.N, L = ch.L, A = ch.A, K = ch.K;
  const int i0 = ichunk * T;
  const int i1 = min(N, i0 + T);
  const int nT = i1 - i0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rep = *ch.rep;
  const uint64_t key = ch.key;
  const bool collect = rep + 1 > ch.burnin;
  const bool want_like = (MODE == kZLike) ||
      (MODE == kZNormal && ((flags & kZfLikeAlways) || ((flags & kZfLikeIfCollect) && collect)));
  const bool store_z = (MODE == kZNormal || MODE == kZInit) && (flags & kZfStoreZ) && ch.Z;
  const bool pfonly = ch.pfrompopflagonly != 0;

  float* sQ = reinterpret_cast<float*>(smem);                   // [T][KS]
  float* sT = sQ + (kUseP ? T * KS : 0);                        // [T][KS] (metro)
  int* sM = reinterpret_cast<int*>(sT + (MODE == kZMetro ? T * KS : 0));  // [T][K]
  int* sN = sM + (kCounts ? T * K : 0);                         // [K][2][32W]
  double* sLD = reinterpret_cast<double*>(sN + (kCounts ? 2 * K * nw32 : 0));  // [T]

  if (kUseP) {
    for (int idx = threadIdx.x; idx < nT * KS; idx += blockDim.x) {
      int ii = idx / KS, k = idx - ii * KS;
      sQ[idx] = k < K ? ch.Q[(size_t)(i0 + ii) * K + k] : 0.0f;
      if (MODE == kZMetro) sT[idx] = k < K ? ch.TestQ[(size_t)(i0 + ii) * K + k] : 0.0f;
    }
  }
  if (kCounts)
    for (int idx = threadIdx.x; idx < nT * K; idx += blockDim.x) sM[idx] = 0;
  if (MODE == kZMetro)
    for (int idx = threadIdx.x; idx < nT; idx += blockDim.x) sLD[idx] = 0.0;
  __syncthreads();

  double like_acc = 0.0;
  int errb = 0;
  const uint32_t stream = (MODE == kZInit) ? (uint32_t)kSInitZ : (uint32_t)kSZ;
  const uint32_t prep = (MODE == kZInit) ? 0u : (uint32_t)rep;

  for (int rb = 0; rb < R; rb++) {
    const int lbase = ((grp * R + rb) * W + warp) * 32;
    if (lbase >= L) break;  // warp-uniform
    const int l = lbase + lane;
    const bool valid = l < L;
    float p0[KT], p1[KT];
    if (kUseP) {
#pragma unroll
      for (int k = 0; k < KT; k++) {
        p0[k] = (valid && k < K) ? ch.P[((size_t)l * K + k) * A] : 0.0f;
        p1[k] = (valid && k < K && A > 1) ? ch.P[((size_t)l * K + k) * A + 1] : 0.0f;
      }
    }
    if (kCounts) {
      for (int q = 0; q < 2 * K; q++) sN[q * nw32 + threadIdx.x] = 0;
    }
    const uint32_t* grow = ch.g2 + (size_t)(valid ? l : 0) * ch.wpr;
    for (int wi = i0 >> 4; wi < (i1 + 15) >> 4; wi++) {
      const uint32_t word = valid ? __ldg(grow + wi) : 0xFFFFFFFFu;
      float wlike = 0.0f;
#pragma unroll 1
      for (int j = 0; j < 16; j += 2) {
        const int ib = (wi << 4) + j;
        if (ib >= i1) break;
        U4 r4;
        if (MODE == kZNormal || MODE == kZInit)
          r4 = philox((uint32_t)l, (uint32_t)(ib >> 1), prep, stream << 24, key);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int ii = ib + h;
          if (ii >= i1) break;
          const uint32_t g = (word >> (2 * (j + h))) & 3u;
          const bool miss = (g == 3u);
          const int a0 = (g == 2u), a1 = (g != 0u);
          int z0 = 0, z1 = 0;
          if (MODE == kZNormal || MODE == kZLike || MODE == kZMetro) {
            const float* q = sQ + (ii - i0) * KS;
            float qv[KT];
#pragma unroll
            for (int k = 0; k < KT; k++) qv[k] = q[k];
            float C0[KT], C1[KT];
            C0[0] = qv[0] * p0[0];
            C1[0] = qv[0] * p1[0];
#pragma unroll
            for (int k = 1; k < KT; k++) {
              C0[k] = __fmaf_rn(qv[k], p0[k], C0[k - 1]);
              C1[k] = __fmaf_rn(qv[k], p1[k], C1[k - 1]);
            }
            const float T0 = a0 ? C1[KT - 1] : C0[KT - 1];
            const float T1 = a1 ? C1[KT - 1] : C0[KT - 1];
            if (MODE == kZNormal) {
              const float u0 = u24(h ? r4.z : r4.x), u1 = u24(h ? r4.w : r4.y);
              const float r0 = u0 * T0, r1 = u1 * T1;
#pragma unroll
              for (int k = 0; k < KT - 1; k++) {
                z0 += ((a0 ? C1[k] : C0[k]) < r0);
                z1 += ((a1 ? C1[k] : C0[k]) < r1);
              }
            }
            if (MODE == kZMetro) {
              const float* tq = sT + (ii - i0) * KS;
              float D0 = tq[0] * p0[0], D1 = tq[0] * p1[0];
#pragma unroll
              for (int k = 1; k < KT; k++) {
                D0 = __fmaf_rn(tq[k], p0[k], D0);
                D1 = __fmaf_rn(tq[k], p1[k], D1);
              }
              const float S0 = a0 ? D1 : D0, S1 = a1 ? D1 : D0;
              float term = 0.0f;
              if (!miss) {
                const float tp = S0 * S1, tm = T0 * T1;
                if (tp > kLikeTinyF && tm > kLikeTinyF)
                  term = __logf(tp) - __logf(tm);
                else
                  term = (float)(log((double)S0) + log((double)S1) - log((double)T0) - log((double)T1));
              }
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) term += __shfl_xor_sync(0xffffffffu, term, off);
              if (lane == 0) atomicAdd(&sLD[ii - i0], (double)term);
            }
            if (want_like && !miss) wlike += like_term(T0, T1);
          } else if (MODE == kZInit) {
            z0 = (int)(((uint64_t)((h ? r4.z : r4.x) >> 1) * (uint64_t)K) >> 31);
            z1 = (int)(((uint64_t)((h ? r4.w : r4.y) >> 1) * (uint64_t)K) >> 31);
          } else if (MODE == kZRecount) {
            if (valid && !miss) {
              const uint8_t b0 = ch.Z[((size_t)ii * 2) * L + l];
              const uint8_t b1 = ch.Z[((size_t)ii * 2 + 1) * L + l];
              z0 = b0; z1 = b1;
              if (b0 >= K || b1 >= K) { errb |= kErrBounds; }
            }
          }
          if (kCounts) {
            const bool cnt = valid && !miss && z0 < K && z1 < K;
            if (cnt && (!pfonly || ch.popflags[ii] == 1)) {
              atomicAdd(&sN[(z0 * 2 + a0) * nw32 + threadIdx.x], 1);
              atomicAdd(&sN[(z1 * 2 + a1) * nw32 + threadIdx.x], 1);
            }
            uint32_t mw[NWM];
#pragma unroll
            for (int q = 0; q < NWM; q++) {
              uint32_t v = 0;
              if (cnt) {
                v += (z0 >> 2) == q ? (1u << (7 * (z0 & 3))) : 0u;
                v += (z1 >> 2) == q ? (1u << (7 * (z1 & 3))) : 0u;
              }
              mw[q] = __reduce_add_sync(0xffffffffu, v);
            }
            if (lane < K) {
              uint32_t s = 0;
#pragma unroll
              for (int q = 0; q < NWM; q++) s = (lane >> 2) == q ? mw[q] : s;
              const int f = (int)((s >> (7 * (lane & 3))) & 127u);
              if (f) atomicAdd(&sM[(ii - i0) * K + lane], f);
            }
          }
          if (store_z && valid) {
            ch.Z[((size_t)ii * 2) * L + l] = miss ? kZMissing : (uint8_t)z0;
            ch.Z[((size_t)ii * 2 + 1) * L + l] = miss ? kZMissing : (uint8_t)z1;
          }
        }
      }
      if (want_like) like_acc += (double)wlike;
    }
    if (kCounts) {
      __syncwarp();
      if (valid) {
        const size_t cbase = (size_t)ichunk * K * A;
        for (int k = 0; k < K; k++) {
          ch.npart[((cbase + (size_t)k * A) + 0) * L + l] = sN[(k * 2) * nw32 + threadIdx.x];
          if (A > 1)
            ch.npart[((cbase + (size_t)k * A) + 1) * L + l] = sN[(k * 2 + 1) * nw32 + threadIdx.x];
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (kCounts) {
    int* dst = ch.mpart + ((size_t)grp * N + i0) * K;
    for (int idx = threadIdx.x; idx < nT * K; idx += blockDim.x) dst[idx] = sM[idx];
  }
  if (MODE == kZMetro) {
    double* dst = ch.ldpart + (size_t)grp * N + i0;
    for (int idx = threadIdx.x; idx < nT; idx += blockDim.x) dst[idx] = sLD[idx];
  }
  if (errb) set_err(ch.err, errb);

  const int ntiles = ch.nchunks * ch.ngroups;
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

int ctas_zpass_b2g(const ChainDev& c) { return c.nchunks * c.ngroups; }

size_t zpass_b2g_smem(int KT, int K, int T, int W, int mode) {
  const int KS = (KT + 3) & ~3;
  const bool useP = (mode == kZNormal || mode == kZMetro || mode == kZLike);
  const bool counts = (mode == kZNormal || mode == kZInit || mode == kZRecount);
  size_t b = 0;
  if (useP) b += (size_t)T * KS * 4;
  if (mode == kZMetro) b += (size_t)T * KS * 4;
  if (counts) b += (size_t)T * K * 4 + (size_t)2 * K * 32 * W * 4;
  b = (b + 7) & ~(size_t)7;
  if (mode == kZMetro) b += (size_t)T * 8;
  return b;
}

template <int KT>
static cudaError_t launch_b2g_k(const LaunchSet& ls, int W, int mode, int flags, size_t smem) {
  dim3 grid(ls.total_ctas), block(32 * W);
  switch (mode) {
#define ST_ZCASE(M)                                                                        \
  case M: {                                                                                \
    auto fn = zpass_b2g_kernel<KT, M>;                                                      \
    if (smem > 48 * 1024)                                                                  \
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);    \
    fn<<<grid, block, smem, ls.stream>>>(ls.chains, ls.prefix, ls.nchains, flags);         \
    return cudaGetLastError();                                                             \
  }
    ST_ZCASE(kZNormal)
    ST_ZCASE(kZInit)
    ST_ZCASE(kZRecount)
    ST_ZCASE(kZMetro)
    ST_ZCASE(kZLike)
#undef ST_ZCASE
  }
  return cudaErrorInvalidValue;
}

// smem must be sized for the largest tile among the chains of the launch.
cudaError_t launch_zpass_b2g(const LaunchSet& ls, int KT, int W, int mode, int flags,
                             size_t smem) {
  switch (KT) {
#define ST_KCASE(k) case k: return launch_b2g_k<k>(ls, W, mode, flags, smem);
    ST_KCASE(1) ST_KCASE(2) ST_KCASE(3) ST_KCASE(4) ST_KCASE(5) ST_KCASE(6)
    ST_KCASE(7) ST_KCASE(8) ST_KCASE(9) ST_KCASE(10) ST_KCASE(11) ST_KCASE(12)
    ST_KCASE(16) ST_KCASE(20) ST_KCASE(24) ST_KCASE(32)
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
      r4 = philox((uint32_t)l, (uint32_t)(i >> 1), mode == kZInit ? 0u : (uint32_t)rep,
                  (mode == kZInit ? (uint32_t)kSInitZ : (uint32_t)kSZ) << 24, ch.key);
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
        else u = (TF)u24(wsel[line]);
        taken++;
        z = pick_generic<TF>(q, Pl, K, A, a, u, total, errb);
        if (want_like) like_acc += log(fmax((double)total, 1e-50));
      } else if (mode == kZInit) {
        if (miss) { if (ch.Z && (flags & kZfStoreZ)) ch.Z[((size_t)i * 2 + line) * L + l] = kZMissing; continue; }
        z = (int)(((uint64_t)(wsel[line] >> 1) * (uint64_t)K) >> 31);
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

}  // namespace st
