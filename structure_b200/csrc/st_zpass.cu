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
// Shared-memory layout of one CTA (byte offsets; every piece 16-aligned).
struct ZLayout {
  size_t q2, t2, x, ld, inc, m, n, total;
};

__host__ __device__ inline size_t zalign16(size_t b) { return (b + 15) & ~(size_t)15; }

__host__ __device__ inline ZLayout zlayout(int KT, int K, int T, int nw32, int mode) {
  const bool useP = (mode == kZNormal || mode == kZMetro || mode == kZLike);
  const bool counts = (mode == kZNormal || mode == kZInit || mode == kZRecount);
  const int KT2 = (KT + 1) & ~1;
  ZLayout z;
  size_t o = 0;
  z.q2 = o; if (useP) o = zalign16(o + (size_t)T * KT2 * 8);            // (q,q) pairs
  z.t2 = o; if (mode == kZMetro) o = zalign16(o + (size_t)T * KT2 * 8);  // (t,t) pairs
  z.x = o;  if (useP) o = zalign16(o + (size_t)3 * KT * nw32 * 8);       // allele table
  z.ld = o; if (mode == kZMetro) o = zalign16(o + (size_t)T * 8);
  z.inc = o; if (counts && KT <= 8) o = zalign16(o + (size_t)(KT + 1) * (KT + 1) * 8);
  z.m = o;  if (counts) o = zalign16(o + (size_t)T * KT * 4);
  z.n = o;  if (counts) o = zalign16(o + (size_t)(2 * K + 1) * nw32 * 4);
  z.total = o;
  return z;
}

// One CTA = W warps x 32 loci (one locus per lane) x R locus blocks, over a
// chunk of T individuals that every warp walks in the same order, so Q_i is a
// shared-memory broadcast.  Per genotype both allele copies are handled as
// one packed FP32x2 lane pair (sm_100 FFMA2/FADD2):
//   X_k   = (P[l][k][a0], P[l][k][a1]) from a per-lane table indexed by the
//           genotype class, so no per-copy select is executed;
//   C_k   = fma(q_k, X_k, C_{k-1})  -- the cumulative mixture weights;
//   r     = u * C_{K-1};  z = sum_k signbit(C_k - r) for k < K-1.
// sign(C_k - r) is exactly (C_k < r) in IEEE arithmetic without flush to zero,
// so z is the reference's "first k with r <= cumsum_k" on FP32 weights.
template <int KT, int MODE, int W>
__global__ void __launch_bounds__(32 * W, 768 / (32 * W))
zpass_b2g_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix,
                 int nchains, int flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double sred[8];
  constexpr int NW32 = 32 * W;
  constexpr int KT2 = (KT + 1) & ~1;
  constexpr int NWM = (KT + 3) / 4;
  constexpr bool kUseP = (MODE == kZNormal || MODE == kZMetro || MODE == kZLike);
  constexpr bool kCounts = (MODE == kZNormal || MODE == kZInit || MODE == kZRecount);
  constexpr bool kLut = kCounts && KT <= 8;

  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int T = ch.tileT, R = ch.tileR;
  const int ichunk = tile % ch.nchunks, grp = tile / ch.nchunks;
  const int N = ch.N, L = ch.L, A = ch.A, K = ch.K;
  const int i0 = ichunk * T;
  const int i1 = min(N, i0 + T);
  const int nT = i1 - i0;
  const int nT16 = (nT + 15) & ~15;  // whole words; padding genotypes are "missing"
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rep = *ch.rep;
  const uint32_t key = ch.key;
  const bool collect = rep + 1 > ch.burnin;
  const bool want_like = (MODE == kZLike) ||
      (MODE == kZNormal && ((flags & kZfLikeAlways) || ((flags & kZfLikeIfCollect) && collect)));
  const bool store_z = (MODE == kZNormal || MODE == kZInit) && (flags & kZfStoreZ) && ch.Z;
  const bool pfonly = ch.pfrompopflagonly != 0;

  const ZLayout lay = zlayout(KT, K, T, NW32, MODE);
  float2* sQ2 = reinterpret_cast<float2*>(smem + lay.q2);
  float2* sT2 = reinterpret_cast<float2*>(smem + lay.t2);
  float2* sX = reinterpret_cast<float2*>(smem + lay.x);
  double* sLD = reinterpret_cast<double*>(smem + lay.ld);
  uint2* sInc = reinterpret_cast<uint2*>(smem + lay.inc);
  int* sM = reinterpret_cast<int*>(smem + lay.m);
  int* sN = reinterpret_cast<int*>(smem + lay.n);

  if (kUseP) {
    for (int idx = threadIdx.x; idx < nT16 * KT2; idx += NW32) {
      const int ii = idx / KT2, k = idx - ii * KT2;
      const bool in = ii < nT && k < K;
      const float q = in ? ch.Q[(size_t)(i0 + ii) * K + k] : 0.0f;
      sQ2[idx] = make_float2(q, q);
      if (MODE == kZMetro) {
        const float t = in ? ch.TestQ[(size_t)(i0 + ii) * K + k] : 0.0f;
        sT2[idx] = make_float2(t, t);
      }
    }
  }
  if (kCounts)
    for (int idx = threadIdx.x; idx < nT16 * KT; idx += NW32) sM[idx] = 0;
  if (kLut) {
    // packed one-hot increments of two copies: 7-bit field per population,
    // four fields per 32-bit half; index KT = "no copy"
    for (int idx = threadIdx.x; idx < (KT + 1) * (KT + 1); idx += NW32) {
      const int za = idx / (KT + 1), zb = idx - za * (KT + 1);
      uint64_t v = 0;
      if (za < KT) v += 1ull << (7 * (za & 3) + 32 * (za >> 2));
      if (zb < KT) v += 1ull << (7 * (zb & 3) + 32 * (zb >> 2));
      sInc[idx] = make_uint2((uint32_t)v, (uint32_t)(v >> 32));
    }
  }
  if (MODE == kZMetro)
    for (int idx = threadIdx.x; idx < nT16; idx += NW32) sLD[idx] = 0.0;
  __syncthreads();

  // lane k < K extracts population k's field from the reduced words
  const int my_word = lane >> 2, my_shift = 7 * (lane & 3);

  double like_acc = 0.0;
  int errb = 0;
  const uint32_t stream = (MODE == kZInit) ? (uint32_t)kSInitZ : (uint32_t)kSZ;
  const uint32_t prep = (MODE == kZInit) ? 0u : (uint32_t)rep;
  int* mycol = sN + threadIdx.x;   // this lane's n[l][k][a] column: stride NW32

  for (int rb = 0; rb < R; rb++) {
    const int lbase = ((grp * R + rb) * W + warp) * 32;
    if (lbase >= L) break;  // warp-uniform
    const int l = lbase + lane;
    const bool valid = l < L;
    if (kUseP) {
      // allele table of this lane's locus: class g in {0/0, 0/1, 1/1}
#pragma unroll
      for (int k = 0; k < KT; k++) {
        const float p0 = (valid && k < K) ? ch.P[((size_t)l * K + k) * A] : 0.0f;
        const float p1 = (valid && k < K && A > 1) ? ch.P[((size_t)l * K + k) * A + 1] : 0.0f;
        sX[(0 * KT + k) * NW32 + threadIdx.x] = make_float2(p0, p0);
        sX[(1 * KT + k) * NW32 + threadIdx.x] = make_float2(p0, p1);
        sX[(2 * KT + k) * NW32 + threadIdx.x] = make_float2(p1, p1);
      }
    }
    if (kCounts)
      for (int q = 0; q < 2 * K + 1; q++) mycol[q * NW32] = 0;   // row 2K: missing copies
    __syncwarp();
    const uint32_t* grow = ch.g2 + (size_t)(valid ? l : 0) * ch.wpr;
    const float2* Xlane = sX + threadIdx.x;
    for (int wi = 0; wi < (nT16 >> 4); wi++) {
      const uint32_t word = valid ? __ldg(grow + (i0 >> 4) + wi) : 0xFFFFFFFFu;
      float wlike = 0.0f;
#pragma unroll 1
      for (int j = 0; j < 16; j += 2) {
        const int row0 = (wi << 4) + j;              // chunk-relative individual
        const int ib = i0 + row0;
        U4 r4;
        if (MODE == kZNormal || MODE == kZInit)
          r4 = philox_s((uint32_t)l, (uint32_t)(ib >> 1), prep, stream, key);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int row = row0 + h;
          const uint32_t g = (word >> (2 * (j + h))) & 3u;
          const bool miss = (g == 3u);
          const uint32_t a0 = g >> 1, a1 = (g | (g >> 1)) & 1u;
          int z0 = 0, z1 = 0;
          if (kUseP) {
            const float4* q4 = reinterpret_cast<const float4*>(sQ2 + row * KT2);
            const float2* X = Xlane + (miss ? 0u : g) * (KT * NW32);
            float2 Cs[KT];
            float2 Q2[KT2];
#pragma unroll
            for (int k = 0; k < KT2; k += 2) {
              const float4 v = q4[k >> 1];
              Q2[k] = make_float2(v.x, v.y);
              Q2[k + 1] = make_float2(v.z, v.w);
            }
            Cs[0] = mul2_rn(Q2[0], X[0]);
#pragma unroll
            for (int k = 1; k < KT; k++) Cs[k] = fma2_rn(Q2[k], X[k * NW32], Cs[k - 1]);
            const float2 Tp = Cs[KT - 1];
            if (MODE == kZNormal) {
              const float2 U = make_float2(u24(h ? r4.z : r4.x), u24(h ? r4.w : r4.y));
              // r = round(u*T), negated by flipping sign bits in the integer
              // domain so the rounded product can never be fused into the add
              const float2 NR =
                  bits_f2(f2_bits(mul2_rn(U, Tp)) ^ 0x8000000080000000ull);
              uint32_t s0 = 0, s1 = 0;
#pragma unroll
              for (int k = 0; k < KT - 1; k++) {
                const float2 D = add2_rn(Cs[k], NR);
                s0 += __float_as_uint(D.x) >> 31;
                s1 += __float_as_uint(D.y) >> 31;
              }
              z0 = (int)s0;
              z1 = (int)s1;
            }
            if (MODE == kZMetro) {
              const float4* t4 = reinterpret_cast<const float4*>(sT2 + row * KT2);
              float2 T2[KT2];
#pragma unroll
              for (int k = 0; k < KT2; k += 2) {
                const float4 v = t4[k >> 1];
                T2[k] = make_float2(v.x, v.y);
                T2[k + 1] = make_float2(v.z, v.w);
              }
              float2 S = mul2_rn(T2[0], X[0]);
#pragma unroll
              for (int k = 1; k < KT; k++) S = fma2_rn(T2[k], X[k * NW32], S);
              const float tp = S.x * S.y, tm = Tp.x * Tp.y;
              const bool tiny = !miss && !(tp > kLikeTinyF && tm > kLikeTinyF);
              float term = miss ? 0.0f : __logf(tp) - __logf(tm);
              if (__any_sync(0xffffffffu, tiny)) {
                if (tiny)
                  term = (float)(log((double)S.x) + log((double)S.y) - log((double)Tp.x) -
                                 log((double)Tp.y));
              }
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) term += __shfl_xor_sync(0xffffffffu, term, off);
              if (lane == 0) atomicAdd(&sLD[row], (double)term);
            }
            if (want_like) {
              const float pr = Tp.x * Tp.y;
              const bool tiny = !miss && !(pr > kLikeTinyF);
              float lt = miss ? 0.0f : __logf(pr);
              if (__any_sync(0xffffffffu, tiny)) {
                if (tiny)
                  lt = (float)(log(fmax((double)Tp.x, 1e-50)) + log(fmax((double)Tp.y, 1e-50)));
              }
              wlike += lt;
            }
          } else if (MODE == kZInit) {
            z0 = (int)(((uint64_t)((h ? r4.z : r4.x) >> 1) * (uint64_t)K) >> 31);
            z1 = (int)(((uint64_t)((h ? r4.w : r4.y) >> 1) * (uint64_t)K) >> 31);
          } else if (MODE == kZRecount) {
            if (valid && !miss) {
              const int ii = i0 + row;
              z0 = ch.Z[((size_t)ii * 2) * L + l];
              z1 = ch.Z[((size_t)ii * 2 + 1) * L + l];
              if (z0 >= K || z1 >= K) errb |= kErrBounds;
            }
          }
          if (kCounts) {
            // invalid lanes read all-missing words, so !miss implies valid
            bool cnt = !miss;
            if (MODE == kZRecount) cnt = cnt && z0 < K && z1 < K;
            bool ncnt = cnt;
            if (pfonly) ncnt = ncnt && ch.popflags[i0 + row] == 1;
            const int trash = 2 * K;
            atomicAdd(&mycol[(ncnt ? 2 * z0 + (int)a0 : trash) * NW32], 1);
            atomicAdd(&mycol[(ncnt ? 2 * z1 + (int)a1 : trash) * NW32], 1);
            uint32_t s_lo, s_hi = 0;
            if (kLut) {
              const uint2 v = sInc[cnt ? z0 * (KT + 1) + z1 : KT * (KT + 1) + KT];
              s_lo = __reduce_add_sync(0xffffffffu, v.x);
              if (KT > 4) s_hi = __reduce_add_sync(0xffffffffu, v.y);
            } else {
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
              s_lo = 0;
#pragma unroll
              for (int q = 0; q < NWM; q++) s_lo = my_word == q ? mw[q] : s_lo;
            }
            const uint32_t s = kLut ? (my_word == 0 ? s_lo : s_hi) : s_lo;
            const int f = (int)((s >> my_shift) & 127u);
            if (lane < K) atomicAdd(&sM[row * KT + lane], f);
          }
          if (store_z && valid && i0 + row < i1) {
            const size_t zi = (size_t)(i0 + row) * 2 * L + l;
            ch.Z[zi] = miss ? kZMissing : (uint8_t)z0;
            ch.Z[zi + L] = miss ? kZMissing : (uint8_t)z1;
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
          ch.npart[((cbase + (size_t)k * A) + 0) * L + l] = mycol[(k * 2) * NW32];
          if (A > 1) ch.npart[((cbase + (size_t)k * A) + 1) * L + l] = mycol[(k * 2 + 1) * NW32];
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();
  if (kCounts) {
    int* dst = ch.mpart + ((size_t)grp * N + i0) * K;
    for (int idx = threadIdx.x; idx < nT * K; idx += NW32) {
      const int ii = idx / K;
      dst[idx] = sM[ii * KT + (idx - ii * K)];
    }
  }
  if (MODE == kZMetro) {
    double* dst = ch.ldpart + (size_t)grp * N + i0;
    for (int idx = threadIdx.x; idx < nT; idx += NW32) dst[idx] = sLD[idx];
  }
  if (errb) set_err(ch.err, errb);

  const int ntiles = ch.nchunks * ch.ngroups;
  if (want_like) {
    double sres = block_sum_d(like_acc, sred);
    if (threadIdx.x == 0) ch.likepart[tile] = sres;
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
  return zlayout(KT, K, T, 32 * W, mode).total;
}

template <int KT, int W>
static cudaError_t launch_b2g_kw(const LaunchSet& ls, int mode, int flags, size_t smem) {
  dim3 grid(ls.total_ctas), block(32 * W);
  switch (mode) {
#define ST_ZCASE(M)                                                                        \
  case M: {                                                                                \
    auto fn = zpass_b2g_kernel<KT, M, W>;                                                   \
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

int zpass_b2g_width(int KT) { return KT <= 12 ? 8 : 2; }

// smem must be sized for the largest tile among the chains of the launch; the
// CTA width is fixed per K class (zpass_b2g_width).
cudaError_t launch_zpass_b2g(const LaunchSet& ls, int KT, int W, int mode, int flags,
                             size_t smem) {
  if (W != zpass_b2g_width(KT)) return cudaErrorInvalidConfiguration;
  switch (KT) {
#define ST_KCASE(k, w) case k: return launch_b2g_kw<k, w>(ls, mode, flags, smem);
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
