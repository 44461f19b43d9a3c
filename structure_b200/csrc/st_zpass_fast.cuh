// st_zpass_fast.cuh -- the biallelic fast path of the data pass (templates).
// Instantiated per K class in st_zpass_k*.cu so the classes compile in
// parallel; st_zpass.cu holds the dispatcher and the generic path.
//
// Fast path (biallelic, 2 bits per genotype, locus-major rows):
//   CTA = W warps; lane = one locus; each warp walks the T individuals of its
//   chunk, 16 genotypes per 32-bit word.  P[l][k][0..1] lives in a per-lane
//   shared-memory table, Q rows of the chunk in shared memory (broadcast
//   reads).  n[l][k][a] is a lane-private shared-memory histogram (lane-minor,
//   conflict-free); m[i][k] is reduced across the warp's 32 loci with
//   redux.sync on 7-bit packed fields.  Each CTA adds its nonzero counts
//   into the chain's single histograms n[k][a][l] and m[i][k] with integer
//   reductions in L2 (exact, so order-free); the host clears them before the
//   pass.
#pragma once
#include "st_device.cuh"
#include "st_kernels.h"

namespace st {
namespace zfast {


constexpr float kLikeTinyF = 1e-30f;
// ln P(D) fast path: the genotype terms Q.P(copy 0) * Q.P(copy 1) of four
// genotypes are multiplied in FP32 and logged once.  A product of four above
// this bound has every factor above it too (factors are <= 1), so no partial
// product is subnormal and no factor is near the reference's 1e-50 clamp; a
// word holding a smaller product is recomputed exactly (word_like_exact).
constexpr float kLikeFastMin = 1e-30f;

// K classes 9-12 keep one (P[l][k][0], P[l][k][1]) pair per population and lane
// and select each copy's allele per genotype: a third of the per-class table
// (20 KB instead of 61 KB at K=10), so three CTAs fit on an SM instead of two.
__host__ __device__ constexpr bool zsingles(int kt) { return kt >= 9 && kt <= 12; }

// One 16-byte shared-memory load.  The Q rows are read by every lane of a warp
// at once (a broadcast): as one 16-byte load that is one wavefront per two
// populations, where the code generator otherwise splits it into 8-byte loads.
__device__ __forceinline__ float4 lds_f4(const float4* p) {
  float4 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
  return v;
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
  z.x = o;  if (useP) o = zalign16(o + (size_t)(zsingles(KT) ? 1 : 3) * KT * nw32 * 8);
  z.ld = o; if (mode == kZMetro) o = zalign16(o + (size_t)T * (nw32 / 32) * 4);   // per warp
  z.inc = o; if (counts && KT <= 12) o = zalign16(o + (size_t)(KT + 1) * (KT + 1) * (KT <= 8 ? 8 : 16));
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
//   r     = RN(u * C_{K-1});  z = sum_k signbit(C_k - r) for k < K-1.
// sign(C_k - r) is exactly (C_k < r) in IEEE arithmetic without flush to zero,
// so z is the reference's "first k with r <= cumsum_k" on FP32 weights.
// The genotype loop of one lane (one locus) over the chunk's individuals,
// specialised on the likelihood and Z-store flags so no per-genotype branch
// tests them; the 16 genotypes of a word are fully unrolled (8 at a time for K
// classes 9-12, whose longer body would not fit the instruction cache) so every
// shift and shared-memory offset is an immediate.
struct ZArgs {
  ChainDev* chp;
  const uint32_t* grow;
  const float2* Xlane;   // this lane's allele-table column: one pair per class and population
  const float2* sQ2;
  const float2* sT2;
  float* sLD;     // this warp's Metropolis log-ratio partials, one per row
  const uint2* sInc;
  int* sM;
  int* mycol;
  int i0, i1, nT16, l, K, L, lane, my_word, my_shift;
  uint32_t prep, key, stream;
  bool valid, pfonly, store_z;
};

// ln P(D) terms of one lane's 16 genotypes of a word in FP64 with the
// reference's per-copy clamp (CalcLike.c:75-133: log of max(Q.P, sqrt(1e-100))),
// from the same FP32 mixture sums as the draw.  Taken only for words that hold
// a term below kLikeFastMin.
template <int KT, int W>
__device__ __noinline__ double word_like_exact(uint32_t word, int row_base, const float2* Xlane,
                                               const float2* sQ2) {
  constexpr int NW32 = 32 * W;
  constexpr int KT2 = (KT + 1) & ~1;
  double s = 0.0;
  for (int gi = 0; gi < 16; gi++) {
    const uint32_t g = (word >> (2 * gi)) & 3u;
    if (g == 3u) continue;
    const float4* q4 = reinterpret_cast<const float4*>(sQ2 + (row_base + gi) * KT2);
    const float2* X2 = Xlane + g * (KT * NW32);
    const uint32_t a0 = g >> 1, a1 = (g | (g >> 1)) & 1u;
    float2 C = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < KT2; k += 2) {
      const float4 v = q4[k >> 1];
      float4 xv;
      if (zsingles(KT)) {
        const float2 p = Xlane[k * NW32];
        const float2 pn = k + 1 < KT ? Xlane[(k + 1) * NW32] : make_float2(0.0f, 0.0f);
        xv = make_float4(a0 ? p.y : p.x, a1 ? p.y : p.x, a0 ? pn.y : pn.x, a1 ? pn.y : pn.x);
      } else {
        const float2 t = X2[k * NW32];
        const float2 tn = k + 1 < KT ? X2[(k + 1) * NW32] : make_float2(0.0f, 0.0f);
        xv = make_float4(t.x, t.y, tn.x, tn.y);
      }
      if (k == 0) C = mul2_rn(make_float2(v.x, v.y), make_float2(xv.x, xv.y));
      else C = fma2_rn(make_float2(v.x, v.y), make_float2(xv.x, xv.y), C);
      if (k + 1 < KT) C = fma2_rn(make_float2(v.z, v.w), make_float2(xv.z, xv.w), C);
    }
    s += log(fmax((double)C.x, 1e-50)) + log(fmax((double)C.y, 1e-50));
  }
  return s;
}

// The Metropolis pass (no draws, no counts) is bound by the shared-memory
// data pipe, mostly the per-lane allele-table loads; it takes the lane's
// frequencies from registers instead (K classes up to 6, where they fit
// without spilling).
// The counting pass is bound by the ALU pipe, where the selects would cost
// more than the loads.
__host__ __device__ constexpr bool zregx(int mode, int kt) { return mode == kZMetro && kt <= 6; }
__host__ __device__ constexpr int zregn(int mode, int kt) { return zregx(mode, kt) ? kt : 1; }

// EXT: the rare per-genotype features (a stored Z, PFROMPOPFLAGONLY counts),
// tested at run time only in this instantiation, so the common one carries
// neither their loads nor their branches.
template <int KT, int MODE, int W, bool LIKE, bool EXT>
__device__ __forceinline__ void zword_loop(const ZArgs& za, double& like_acc, int& errb,
                                           const float (&p0r)[zregn(MODE, KT)],
                                           const float (&p1r)[zregn(MODE, KT)]) {
  constexpr int NW32 = 32 * W;
  constexpr int KT2 = (KT + 1) & ~1;
  constexpr int NWM = (KT + 3) / 4;
  constexpr bool kUseP = (MODE == kZNormal || MODE == kZMetro || MODE == kZLike);
  constexpr bool kCounts = (MODE == kZNormal || MODE == kZInit || MODE == kZRecount);
  constexpr bool kLut = kCounts && KT <= 12;
  constexpr bool kRegX = zregx(MODE, KT);
  constexpr int kHalves = (zsingles(KT) && MODE != kZMetro) ? 2 : 1;
  constexpr int kJN = 16 / kHalves;   // genotypes of a word per unrolled pass
  ChainDev& ch = *za.chp;
  const uint32_t* grow = za.grow;
  const float2* Xlane = za.Xlane;
  const float2* sQ2 = za.sQ2;
  const float2* sT2 = za.sT2;
  float* sLD = za.sLD;
  const uint2* sInc = za.sInc;
  int* sM = za.sM;
  int* mycol = za.mycol;
  const int i0 = za.i0, i1 = za.i1, nT16 = za.nT16, l = za.l, K = za.K, L = za.L;
  const int lane = za.lane, my_word = za.my_word, my_shift = za.my_shift;
  [[maybe_unused]] const int moff = lane < K ? lane : lane - K + KT;
  [[maybe_unused]] const bool second = lane >= K;
  const uint32_t prep = za.prep, key = za.key, stream = za.stream;
  const bool valid = za.valid, pfonly = EXT && za.pfonly, store_z = EXT && za.store_z;
    // Philox blocks of this lane's locus and sweep: b = individual pair.  i0 is
    // a multiple of 16 (whole genotype words), so a word's first pair index is
    // a multiple of 8 and pair j/2 of the word is that index ^ (j/2).
    const PhiloxRun prun((uint32_t)l, prep, stream, key);
    for (int wi = 0; wi < (nT16 >> 4); wi++) {
      const uint32_t word = valid ? __ldg(grow + (i0 >> 4) + wi) : 0xFFFFFFFFu;
      const uint32_t pw = prun.head ^ ((uint32_t)((i0 >> 1) + (wi << 3)) & 0xFFFFFFu);
      float wlike = 0.0f, wprod = 1.0f, wmin = 1.0f;
      float tr[MODE == kZMetro ? 16 : 1];   // Metropolis pass: this lane's term per row
      // the widest table classes walk a word in two halves of 8 genotypes, so
      // the unrolled loop body stays within the instruction cache
#pragma unroll 1
      for (int hb = 0; hb < kHalves; hb++) {
      const uint32_t hword = kHalves == 1 ? word : (word >> (16 * hb));
      const uint32_t phw = kHalves == 1 ? pw : (pw ^ (uint32_t)(hb << 2));
      const int rbase = (wi << 4) + hb * kJN;
#pragma unroll
      for (int j = 0; j < kJN; j += 2) {
        const int row0 = rbase + j;              // chunk-relative individual
        U4 r4;
        if (MODE == kZNormal || MODE == kZInit) r4 = prun.block_r0(phw ^ (uint32_t)(j >> 1));
        [[maybe_unused]] uint32_t pr_lo = 0, pr_hi = 0, pr_3 = 0;   // first row's reduced words
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int row = row0 + h;
          const uint32_t g = (hword >> (2 * (j + h))) & 3u;
          const bool miss = (g == 3u);
          const uint32_t a0 = g >> 1, a1 = (g | (g >> 1)) & 1u;
          int z0 = 0, z1 = 0;
          if (kUseP) {
            const float4* q4 = reinterpret_cast<const float4*>(sQ2 + row * KT2);
            const uint32_t cls = miss ? 0u : g;
            const float2* X2 = Xlane + cls * (KT * NW32);
            float2 Cs[KT];
            float2 Q2[KT2], X[KT2];
#pragma unroll
            for (int k = 0; k < KT2; k += 2) {
              const float4 v = lds_f4(q4 + (k >> 1));
              Q2[k] = make_float2(v.x, v.y);
              Q2[k + 1] = make_float2(v.z, v.w);
              if (zsingles(KT)) {
                // (P[a0][k], P[a1][k]) from the lane's pair; a missing genotype
                // takes allele 1 and its terms are discarded below
#pragma unroll
                for (int e = 0; e < 2; e++) {
                  if (k + e < KT) {
                    const float2 pv = Xlane[(k + e) * NW32];
                    X[k + e] = make_float2(a0 ? pv.y : pv.x, a1 ? pv.y : pv.x);
                  } else {
                    X[k + e] = make_float2(0.0f, 0.0f);
                  }
                }
              } else if (!kRegX) {
                // 8-byte pairs, lane-minor: a warp's load is two wavefronts
                X[k] = X2[k * NW32];
                X[k + 1] = k + 1 < KT ? X2[(k + 1) * NW32] : make_float2(0.0f, 0.0f);
              }
            }
            if (kRegX) {
              // (P[a0][k], P[a1][k]); a missing genotype reads class 1/1, and
              // its terms are discarded below
#pragma unroll
              for (int k = 0; k < KT2; k++) {
                const int kk = k < zregn(MODE, KT) ? k : 0;
                X[k] = make_float2(a0 ? p1r[kk] : p0r[kk], a1 ? p1r[kk] : p0r[kk]);
              }
            }
            Cs[0] = mul2_rn(Q2[0], X[0]);
#pragma unroll
            for (int k = 1; k < KT; k++) Cs[k] = fma2_rn(Q2[k], X[k], Cs[k - 1]);
            const float2 Tp = Cs[KT - 1];
            if (MODE == kZNormal) {
              // NR = RN(-u T) for both copies: one fma of -(1 + u), built from
              // the Philox words' low 23 bits, so the rounded threshold is
              // never contracted into the compare below
              const float2 NM = make_float2(neg_one_plus_u23(h ? r4.z : r4.x),
                                            neg_one_plus_u23(h ? r4.w : r4.y));
              const float2 NR = fma2_rn(NM, Tp, Tp);
              // the sign bits of C_k - r (k < K-1) shifted into one word per
              // copy; z = their count = #{k : C_k < r}
              uint32_t t0 = 0u, t1 = 0u;
#pragma unroll
              for (int k = 0; k < KT - 1; k++) {
                const float2 D = add2_rn(Cs[k], NR);
                t0 = __funnelshift_l(__float_as_uint(D.x), t0, 1);
                t1 = __funnelshift_l(__float_as_uint(D.y), t1, 1);
              }
              z0 = __popc(t0);
              z1 = __popc(t1);
            }
            if (MODE == kZMetro) {
              const float4* t4 = reinterpret_cast<const float4*>(sT2 + row * KT2);
              float2 T2[KT2];
#pragma unroll
              for (int k = 0; k < KT2; k += 2) {
                const float4 v = lds_f4(t4 + (k >> 1));
                T2[k] = make_float2(v.x, v.y);
                T2[k + 1] = make_float2(v.z, v.w);
              }
              float2 S = mul2_rn(T2[0], X[0]);
#pragma unroll
              for (int k = 1; k < KT; k++) S = fma2_rn(T2[k], X[k], S);
              const float tp = S.x * S.y, tm = Tp.x * Tp.y;
              const bool tiny = !miss && !(tp > kLikeTinyF && tm > kLikeTinyF);
              float term = miss ? 0.0f : __logf(tp) - __logf(tm);
              if (__any_sync(0xffffffffu, tiny)) {
                if (tiny)
                  term = (float)(log((double)S.x) + log((double)S.y) - log((double)Tp.x) -
                                 log((double)Tp.y));
              }
              tr[MODE == kZMetro ? j + h : 0] = term;
            }
            if (LIKE) {
              // j + h is a compile-time constant after unrolling
              const float pr = miss ? 1.0f : Tp.x * Tp.y;
              wprod = ((j + h) & 3) == 0 ? pr : wprod * pr;
              if (((j + h) & 3) == 3) {
                wmin = fminf(wmin, wprod);
                wlike += __logf(wprod);
              }
            }
          } else if (MODE == kZInit) {
            z0 = (int)(((uint64_t)((h ? r4.z : r4.x) >> 1) * (uint64_t)K) >> 31);
            z1 = (int)(((uint64_t)((h ? r4.w : r4.y) >> 1) * (uint64_t)K) >> 31);
            // USEPOPINFO: start at the given population (src/Init.c:74-117)
            if (ch.initpop && valid && i0 + row < i1 && ch.initpop[i0 + row] >= 0)
              z0 = z1 = ch.initpop[i0 + row];
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
            if (EXT && pfonly) ncnt = ncnt && ch.popflags[i0 + row] == 1;
            const int trash = 2 * K;
            atomicAdd(&mycol[(ncnt ? 2 * z0 + (int)a0 : trash) * NW32], 1);
            atomicAdd(&mycol[(ncnt ? 2 * z1 + (int)a1 : trash) * NW32], 1);
            uint32_t s_lo, s_hi = 0;
            [[maybe_unused]] uint32_t s_3 = 0;
            if (kLut && KT <= 8) {
              const uint2 v = sInc[cnt ? z0 * (KT + 1) + z1 : KT * (KT + 1) + KT];
              s_lo = __reduce_add_sync(0xffffffffu, v.x);
              if (KT > 4) s_hi = __reduce_add_sync(0xffffffffu, v.y);
            } else if (kLut) {
              // K classes 9-12: three packed words per pair of copies
              const uint4 v = reinterpret_cast<const uint4*>(sInc)[cnt ? z0 * (KT + 1) + z1
                                                                       : KT * (KT + 1) + KT];
              s_lo = __reduce_add_sync(0xffffffffu, v.x);
              s_hi = __reduce_add_sync(0xffffffffu, v.y);
              s_3 = __reduce_add_sync(0xffffffffu, v.z);
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
            if constexpr (kLut) {
              // one shared atomic per pair of rows: lanes 0..K-1 add the first
              // row's populations, lanes K..2K-1 the second's (my_word and
              // my_shift name population lane mod K; moff its slot)
              if (h == 0) {
                pr_lo = s_lo;
                pr_hi = s_hi;
                pr_3 = s_3;
              } else {
                uint32_t s;
                if constexpr (KT <= 4) {
                  s = second ? s_lo : pr_lo;
                } else if constexpr (KT <= 8) {
                  const uint32_t a = my_word == 0 ? pr_lo : pr_hi, b = my_word == 0 ? s_lo : s_hi;
                  s = second ? b : a;
                } else {
                  const uint32_t a = my_word == 0 ? pr_lo : (my_word == 1 ? pr_hi : pr_3);
                  const uint32_t b = my_word == 0 ? s_lo : (my_word == 1 ? s_hi : s_3);
                  s = second ? b : a;
                }
                const int f = (int)((s >> my_shift) & 127u);
                if (lane < 2 * K) atomicAdd(&sM[(row - 1) * KT + moff], f);
              }
            } else {
              const int f = (int)((s_lo >> my_shift) & 127u);
              if (lane < K) atomicAdd(&sM[row * KT + lane], f);
            }
          }
          if (EXT && store_z && valid && i0 + row < i1) {
            const size_t zi = (size_t)(i0 + row) * 2 * L + l;
            ch.Z[zi] = miss ? kZMissing : (uint8_t)z0;
            ch.Z[zi + L] = miss ? kZMissing : (uint8_t)z1;
          }
        }
      }
      }   // halves
      if constexpr (MODE == kZMetro) {
        // the word's 16 row sums over the warp's 32 loci by a transposed
        // butterfly: at the exchange across lane bit b a lane keeps the half
        // of its rows picked by its own bit b and adds its partner's partial
        // for the same rows; after lane bits 4..1 lanes 2r, 2r+1 hold row r.
        // 31 exchanges per word instead of 5 per row.
        float v8[8], v4[4], v2[2];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const bool hi = lane & 16;
          v8[i] = (hi ? tr[i + 8] : tr[i]) + __shfl_xor_sync(0xffffffffu, hi ? tr[i] : tr[i + 8], 16);
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const bool hi = lane & 8;
          v4[i] = (hi ? v8[i + 4] : v8[i]) + __shfl_xor_sync(0xffffffffu, hi ? v8[i] : v8[i + 4], 8);
        }
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const bool hi = lane & 4;
          v2[i] = (hi ? v4[i + 2] : v4[i]) + __shfl_xor_sync(0xffffffffu, hi ? v4[i] : v4[i + 2], 4);
        }
        const bool hi = lane & 2;
        float v = (hi ? v2[1] : v2[0]) + __shfl_xor_sync(0xffffffffu, hi ? v2[0] : v2[1], 2);
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        if (!(lane & 1)) sLD[(wi << 4) + (lane >> 1)] += v;   // this warp's rows only
      }
      if (LIKE) {
        double wl = (double)wlike;
        if (__any_sync(0xffffffffu, !(wmin > kLikeFastMin))) {   // once per word, rare
          if (!(wmin > kLikeFastMin))
            wl = word_like_exact<KT, W>(word, wi << 4, Xlane, sQ2);
        }
        like_acc += wl;
      }
    }
}

template <int KT, int MODE, int W>
__global__ void __launch_bounds__(32 * W, (KT <= 12 ? 768 : 512) / (32 * W))
zpass_b2g_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix,
                 int nchains, int flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double sred[8];
  constexpr int NW32 = 32 * W;
  constexpr int KT2 = (KT + 1) & ~1;
  constexpr int NWM = (KT + 3) / 4;
  constexpr bool kUseP = (MODE == kZNormal || MODE == kZMetro || MODE == kZLike);
  constexpr bool kCounts = (MODE == kZNormal || MODE == kZInit || MODE == kZRecount);
  constexpr bool kLut = kCounts && KT <= 12;

  int c, tile;
  if (flags & kZfInterleave) {   // chains of one data set and tile, interleaved
    c = (int)blockIdx.x % nchains;
    tile = (int)blockIdx.x / nchains;
  } else {
    c = find_chain(prefix, nchains, blockIdx.x);
    tile = blockIdx.x - prefix[c];
  }
  ChainDev& ch = chains[c];
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
  float* sLD = reinterpret_cast<float*>(smem + lay.ld);   // [W][nT16]
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
    // four fields per 32-bit word; index KT = "no copy"
    for (int idx = threadIdx.x; idx < (KT + 1) * (KT + 1); idx += NW32) {
      const int za = idx / (KT + 1), zb = idx - za * (KT + 1);
      auto field = [&](int z, int q) -> uint32_t {
        return (z < KT && (z >> 2) == q) ? (1u << (7 * (z & 3))) : 0u;
      };
      const uint32_t w0 = field(za, 0) + field(zb, 0), w1 = field(za, 1) + field(zb, 1);
      if (KT <= 8) sInc[idx] = make_uint2(w0, w1);
      else reinterpret_cast<uint4*>(sInc)[idx] = make_uint4(w0, w1, field(za, 2) + field(zb, 2), 0u);
    }
  }
  if (MODE == kZMetro)
    for (int idx = threadIdx.x; idx < nT16 * W; idx += NW32) sLD[idx] = 0.0f;
  __syncthreads();

  // lane k < K extracts population k's field from the reduced words
  // (table classes: lanes K..2K-1 take population lane - K of the second row
  // of a pair, stored at slot moff of the first row's)
  const int mfield = (kLut && lane >= K) ? lane - K : lane;
  const int my_word = mfield >> 2, my_shift = 7 * (mfield & 3);


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
    constexpr int NP = zregn(MODE, KT);
    float p0r[NP], p1r[NP];   // Metropolis pass: this lane's P[l][k][0], P[l][k][1]
#pragma unroll
    for (int k = 0; k < NP; k++) p0r[k] = p1r[k] = 0.0f;
    if (kUseP) {
      // allele table of this lane's locus: for class g in {0/0, 0/1, 1/1} and
      // population k the pair (P[a0][k], P[a1][k]) at [g][k][lane], 8 bytes per
      // lane and lane-minor, so a warp reads one population's pairs in two
      // shared-memory wavefronts (pairs of pairs in 16-byte slots took four
      // per half once the loads were split into 8-byte ones)
      float2* X2w = reinterpret_cast<float2*>(sX) + threadIdx.x;
#pragma unroll
      for (int k = 0; k < KT2; k += 2) {
        float p0[2], p1[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int kk = k + e;
          p0[e] = (valid && kk < K) ? ch.P[((size_t)l * K + kk) * A] : 0.0f;
          p1[e] = (valid && kk < K && A > 1) ? ch.P[((size_t)l * K + kk) * A + 1] : 0.0f;
          if (zregx(MODE, KT) && kk < NP) {
            p0r[kk < NP ? kk : 0] = p0[e];
            p1r[kk < NP ? kk : 0] = p1[e];
          }
        }
        if (zsingles(KT)) {
          float2* XSw = reinterpret_cast<float2*>(sX) + threadIdx.x;
          XSw[k * NW32] = make_float2(p0[0], p1[0]);
          if (k + 1 < KT) XSw[(k + 1) * NW32] = make_float2(p0[1], p1[1]);
        } else {
#pragma unroll
          for (int e = 0; e < 2; e++) {
            if (k + e < KT) {
              X2w[(0 * KT + k + e) * NW32] = make_float2(p0[e], p0[e]);
              X2w[(1 * KT + k + e) * NW32] = make_float2(p0[e], p1[e]);
              X2w[(2 * KT + k + e) * NW32] = make_float2(p1[e], p1[e]);
            }
          }
        }
      }
    }
    if (kCounts)
      for (int q = 0; q < 2 * K + 1; q++) mycol[q * NW32] = 0;   // row 2K: missing copies
    __syncwarp();
    const uint32_t* grow = ch.g2 + (size_t)(valid ? l : 0) * ch.wpr;
    const float2* Xlane = reinterpret_cast<const float2*>(sX) + threadIdx.x;
    {
      ZArgs za{&ch, grow, Xlane, sQ2, sT2, sLD + warp * nT16, sInc, sM, mycol, i0, i1, nT16, l,
               K, L, lane,
               my_word, my_shift, prep, key, stream, valid, pfonly, store_z};
      const bool ext = store_z || pfonly;
      if (want_like) {
        if (ext) zword_loop<KT, MODE, W, true, true>(za, like_acc, errb, p0r, p1r);
        else zword_loop<KT, MODE, W, true, false>(za, like_acc, errb, p0r, p1r);
      } else {
        if (ext) zword_loop<KT, MODE, W, false, true>(za, like_acc, errb, p0r, p1r);
        else zword_loop<KT, MODE, W, false, false>(za, like_acc, errb, p0r, p1r);
      }
    }
    if (kCounts) {
      __syncwarp();
      if (valid) {
        for (int k = 0; k < K; k++) {
          const int v0 = mycol[(k * 2) * NW32];
          if (v0) atomicAdd(&ch.npart[((size_t)k * A + 0) * L + l], v0);
          const int v1 = mycol[(k * 2 + 1) * NW32];
          if (A > 1 && v1) atomicAdd(&ch.npart[((size_t)k * A + 1) * L + l], v1);
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();
  if (kCounts) {
    int* dst = ch.mpart + (size_t)i0 * K;
    for (int idx = threadIdx.x; idx < nT * K; idx += NW32) {
      const int ii = idx / K;
      const int v = sM[ii * KT + (idx - ii * K)];
      if (v) atomicAdd(&dst[idx], v);
    }
  }
  if (MODE == kZMetro) {
    // the warps' partials in warp order: a fixed summation order
    double* dst = ch.ldpart + (size_t)grp * N + i0;
    for (int idx = threadIdx.x; idx < nT; idx += NW32) {
      double v = 0.0;
      for (int w = 0; w < W; w++) v += (double)sLD[w * nT16 + idx];
      dst[idx] = v;
    }
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

template <int KT, int W>
cudaError_t launch_b2g_kw(const LaunchSet& ls, int mode, int flags, size_t smem) {
  dim3 grid(ls.total_ctas), block(32 * W);
  switch (mode) {
#define ST_ZCASE(M)                                                                        \
  case M: {                                                                                \
    auto fn = zpass_b2g_kernel<KT, M, W>;                                                   \
    if (smem > 40 * 1024) /* above the default 48 KB with the static smem */            \
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


}  // namespace zfast
}  // namespace st
