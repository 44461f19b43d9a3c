// st_zpass_ind.cuh -- the biallelic Z update with counts and ln P(D), one lane
// per individual (K classes up to 8, mode Normal).
//
// The locus-lane pass (st_zpass_fast.cuh) gives each lane a locus and walks
// the individuals of a chunk; every genotype then reads its individual's Q row
// from shared memory and its lane's own allele table (32 distinct rows per
// warp load), which keeps the shared-memory data pipe near its peak.  Here a
// lane owns an individual instead:
//   * its Q row lives in registers for the whole CTA;
//   * all lanes of a warp walk the same loci, so the allele table of the
//     current locus is one shared-memory row read with three distinct
//     addresses (the genotype classes 0/0, 0/1, 1/1);
//   * the ancestry counts m[i][k] accumulate in the lane's registers (8-bit
//     fields, emptied every 64 loci);
//   * the allele counts n[l][k][a] of a locus are warp sums (redux.sync over
//     packed 7-bit fields looked up for the genotype's two copies), stored per
//     warp in shared memory and added across warps into the chain's histogram
//     once per 64 loci;
//   * the genotypes come from an individual-major copy of the 2-bit data
//     (st_data.g2t: per 32 individuals and 64 loci, one uint4 per lane), one
//     coalesced 16-byte load per lane per 64 loci.
// Draws are the locus-lane pass's, bit for bit: the Philox block of
// (locus l, individual pair i/2) serves both individuals of the pair (words x,y
// the even one, z,w the odd one).  Lanes 2j and 2j+1 hold such a pair, so over
// two loci each computes one block (the even lane at l, the odd lane at l+1)
// and they trade the halves the other needs with one shuffle each way.
// The categorical draw, the threshold, the ties and the FP32 arithmetic are the
// same as there (z = #{k < K-1 : C_k < RN(u T)}).
//
// CTA = 8 warps = 256 individuals of the chain's Z-pass tile (tileT
// individuals, processed 256 at a time) times the tile's loci
// (tileR * tileW * 32), in stages of 64 loci: so the tile count, the ln P(D)
// partials and the last-CTA protocol are those of the locus-lane pass.
#pragma once
#include "st_zpass_fast.cuh"

namespace st {
namespace zind {

constexpr int kIW = 8;    // warps per CTA, 32 individuals each
constexpr int kLS = 64;   // loci per stage: one uint4 of genotype words per lane

struct ILayout {
  size_t x, nsl, nlut, mlut, total;
};

// Shared memory of one CTA for K class KT (sized for K = KT).
__host__ __device__ inline ILayout ilayout(int KT) {
  const int KT2 = (KT + 1) & ~1;
  const int NB = 2 * KT;   // allele-count bins (population, allele)
  ILayout z;
  size_t o = 0;
  z.x = o;    o = zfast::zalign16(o + (size_t)kLS * 3 * KT2 * 8);          // [ls][class][k] float2
  z.nsl = o;  o = zfast::zalign16(o + (size_t)kIW * kLS * NB * 4);         // [warp][ls][bin] int
  z.nlut = o; o = zfast::zalign16(o + (size_t)(NB + 1) * (NB + 1) * 16);   // [f0][f1] uint4
  z.mlut = o; o = zfast::zalign16(o + (size_t)(KT + 1) * (KT + 1) * 8);    // [z0][z1] uint2
  z.total = o;
  return z;
}

// ln P(D) terms of one lane's 64 loci of a stage in FP64 with the reference's
// clamp (CalcLike.c:75-133: log of max(Q.P, sqrt(1e-100))), from the same FP32
// sums as the draw; taken only for stages holding a tiny four-locus product.
template <int KT>
__device__ __noinline__ double stage_like_exact(uint4 wd, const float2* sX, const float2* Q2) {
  constexpr int KT2 = (KT + 1) & ~1;
  double s = 0.0;
  const uint32_t wq[4] = {wd.x, wd.y, wd.z, wd.w};
  for (int ls = 0; ls < kLS; ls++) {
    const uint32_t g = (wq[ls >> 4] >> (2 * (ls & 15))) & 3u;
    if (g == 3u) continue;
    const float2* X = sX + ((size_t)ls * 3 + g) * KT2;
    float2 C = mul2_rn(Q2[0], X[0]);
    for (int k = 1; k < KT; k++) C = fma2_rn(Q2[k], X[k], C);
    s += log(fmax((double)C.x, 1e-50)) + log(fmax((double)C.y, 1e-50));
  }
  return s;
}

// One stage (64 loci) of one lane: draws, counts, Z bytes, ln P(D) terms.
template <int KT, bool LIKE, bool SZ>
__device__ __forceinline__ void ind_stage(ChainDev& ch, const uint4 wd, const float2 (&Q2)[(KT + 1) & ~1],
                                          const float2* __restrict__ sX, int* __restrict__ nsw,
                                          const uint4* __restrict__ sNL,
                                          const uint2* __restrict__ sML, int ls0, int i, bool ivalid,
                                          bool ncount, uint32_t prep, uint32_t key, int NB,
                                          uint32_t& acc_lo, uint32_t& acc_hi, double& like_acc) {
  constexpr int KT2 = (KT + 1) & ~1;
  constexpr int NWN = (2 * KT + 3) / 4;   // packed words of the allele-count bins
  const int lane = threadIdx.x & 31;
  const uint32_t p = lane & 1;
  const uint32_t ipair = (uint32_t)(i >> 1);
  const int L = ch.L;
  const int bw = lane >> 2, bsh = 7 * (lane & 3);   // this lane's bin: word, shift
  float wsum = 0.0f, wprod = 1.0f, wmin = 1.0f;
#pragma unroll 1
  for (int q = 0; q < 4; q++) {
    const uint32_t word = q == 0 ? wd.x : (q == 1 ? wd.y : (q == 2 ? wd.z : wd.w));
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
      const int lb = ls0 + 16 * q + j;
      // this lane's Philox block: (lb + p, pair); the partner's halves by shuffle
      const U4 r4 = philox_s((uint32_t)(lb + (int)p), ipair, prep, (uint32_t)kSZ, key);
      const uint32_t s0 = p ? r4.x : r4.z, s1 = p ? r4.y : r4.w;
      const uint32_t g0w = __shfl_xor_sync(0xffffffffu, s0, 1);
      const uint32_t g1w = __shfl_xor_sync(0xffffffffu, s1, 1);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int ls = 16 * q + j + h;            // stage-relative locus (compile-time)
        // uniform words of this lane's two copies at locus lb + h
        const uint32_t wa = h == 0 ? (p ? g0w : r4.x) : (p ? r4.z : g0w);
        const uint32_t wb = h == 0 ? (p ? g1w : r4.y) : (p ? r4.w : g1w);
        const uint32_t g = (word >> (2 * (j + h))) & 3u;
        const bool miss = (g == 3u);
        const uint32_t a0 = g >> 1, a1 = (g | (g >> 1)) & 1u;
        const uint32_t cls = miss ? 0u : g;
        const float4* X4 = reinterpret_cast<const float4*>(sX + ((size_t)ls * 3 + cls) * KT2);
        float2 X[KT2];
#pragma unroll
        for (int k = 0; k < KT2; k += 2) {
          const float4 v = X4[k >> 1];
          X[k] = make_float2(v.x, v.y);
          X[k + 1] = make_float2(v.z, v.w);
        }
        float2 Cs[KT];
        Cs[0] = mul2_rn(Q2[0], X[0]);
#pragma unroll
        for (int k = 1; k < KT; k++) Cs[k] = fma2_rn(Q2[k], X[k], Cs[k - 1]);
        const float2 Tp = Cs[KT - 1];
        const float2 NM = make_float2(neg_one_plus_u23(wa), neg_one_plus_u23(wb));
        const float2 NR = fma2_rn(NM, Tp, Tp);
        uint32_t t0 = 0u, t1 = 0u;
#pragma unroll
        for (int k = 0; k < KT - 1; k++) {
          const float2 D = add2_rn(Cs[k], NR);
          t0 = __funnelshift_l(__float_as_uint(D.x), t0, 1);
          t1 = __funnelshift_l(__float_as_uint(D.y), t1, 1);
        }
        const int z0 = __popc(t0), z1 = __popc(t1);
        const bool cnt = ivalid && !miss;
        // allele counts of this locus: warp sums of the two copies' bins
        {
          const bool nc = cnt && ncount;
          const int f0 = nc ? 2 * z0 + (int)a0 : NB, f1 = nc ? 2 * z1 + (int)a1 : NB;
          const uint4 v = sNL[f0 * (NB + 1) + f1];
          uint32_t r[NWN];
          r[0] = __reduce_add_sync(0xffffffffu, v.x);
          if (NWN > 1) r[1] = __reduce_add_sync(0xffffffffu, v.y);
          if (NWN > 2) r[2] = __reduce_add_sync(0xffffffffu, v.z);
          if (NWN > 3) r[3] = __reduce_add_sync(0xffffffffu, v.w);
          uint32_t mine = r[0];
#pragma unroll
          for (int qq = 1; qq < NWN; qq++) mine = bw == qq ? r[qq] : mine;
          if (lane < NB) nsw[ls * NB + lane] = (int)((mine >> bsh) & 127u);
        }
        // ancestry counts of this lane's individual: 8-bit fields
        {
          const uint2 v = sML[(cnt ? z0 : KT) * (KT + 1) + (cnt ? z1 : KT)];
          acc_lo += v.x;
          acc_hi += v.y;
        }
        if (SZ && ivalid && lb + h < L) {
          const size_t zi = (size_t)i * 2 * L + (size_t)(lb + h);
          ch.Z[zi] = miss ? kZMissing : (uint8_t)z0;
          ch.Z[zi + L] = miss ? kZMissing : (uint8_t)z1;
        }
        if (LIKE) {
          const float pr = miss ? 1.0f : Tp.x * Tp.y;
          wprod = (ls & 3) == 0 ? pr : wprod * pr;
          if ((ls & 3) == 3) {
            wmin = fminf(wmin, wprod);
            wsum += __logf(wprod);
          }
        }
      }
    }
  }
  if (LIKE) {
    if (wmin > zfast::kLikeFastMin) like_acc += (double)wsum;
    else like_acc += stage_like_exact<KT>(wd, sX, Q2);   // a four-locus product <= 1e-30: rare
  }
}

template <int KT>
__global__ void __launch_bounds__(kIW * 32, 3)
zpass_ind_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix, int nchains,
                 int flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double sred[kIW];
  constexpr int KT2 = (KT + 1) & ~1;
  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int T = ch.tileT, R = ch.tileR, W = ch.tileW;
  const int ichunk = tile % ch.nchunks, grp = tile / ch.nchunks;
  const int N = ch.N, L = ch.L, K = ch.K, A = ch.A;
  const int i0 = ichunk * T, i1 = min(N, i0 + T);
  const int l0 = grp * R * W * 32, l1 = min(L, l0 + R * W * 32);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rep = *ch.rep;
  const uint32_t key = ch.key;
  const bool collect = rep + 1 > ch.burnin;
  const bool want_like = (flags & kZfLikeAlways) || ((flags & kZfLikeIfCollect) && collect);
  const bool store_z = (flags & kZfStoreZ) && ch.Z;
  const bool pfonly = ch.pfrompopflagonly != 0;
  const int NB = 2 * K;

  const ILayout lay = ilayout(KT);
  float2* sX = reinterpret_cast<float2*>(smem + lay.x);
  int* sNS = reinterpret_cast<int*>(smem + lay.nsl);
  uint4* sNL = reinterpret_cast<uint4*>(smem + lay.nlut);
  uint2* sML = reinterpret_cast<uint2*>(smem + lay.mlut);
  int* nsw = sNS + warp * kLS * NB;   // this warp's per-locus bin sums of a stage

  // packed increments: allele bins (population, allele) as 7-bit fields of
  // four words for the two copies (index NB = not counted); ancestry counts as
  // 8-bit fields of two words (index KT = not counted)
  for (int idx = threadIdx.x; idx < (NB + 1) * (NB + 1); idx += kIW * 32) {
    const int f0 = idx / (NB + 1), f1 = idx - f0 * (NB + 1);
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    if (f0 < NB) w[f0 >> 2] += 1u << (7 * (f0 & 3));
    if (f1 < NB) w[f1 >> 2] += 1u << (7 * (f1 & 3));
    sNL[idx] = make_uint4(w[0], w[1], w[2], w[3]);
  }
  for (int idx = threadIdx.x; idx < (KT + 1) * (KT + 1); idx += kIW * 32) {
    const int za = idx / (KT + 1), zb = idx - za * (KT + 1);
    uint64_t v = 0;
    if (za < KT) v += 1ull << (8 * za);
    if (zb < KT) v += 1ull << (8 * zb);
    sML[idx] = make_uint2((uint32_t)v, (uint32_t)(v >> 32));
  }

  double like_acc = 0.0;
  for (int ib = i0; ib < i1; ib += kIW * 32) {
    const int i = ib + threadIdx.x;        // this lane's individual (ib is even)
    const bool ivalid = i < i1;
    float2 Q2[KT2];
#pragma unroll
    for (int k = 0; k < KT2; k++) {
      const float q = (ivalid && k < K) ? ch.Q[(size_t)i * K + k] : 0.0f;
      Q2[k] = make_float2(q, q);
    }
    const bool ncount = ivalid && (!pfonly || ch.popflags[i] == 1);
    int mtot[KT];
#pragma unroll
    for (int k = 0; k < KT; k++) mtot[k] = 0;
    const uint4* gw = reinterpret_cast<const uint4*>(ch.g2t) + ((size_t)(i >> 5) * ch.nlw4) * 32 + (i & 31);
    for (int ls0 = l0; ls0 < l1; ls0 += kLS) {
      __syncthreads();   // the previous stage's tables and bin sums are consumed
      for (int idx = threadIdx.x; idx < kLS * KT2; idx += kIW * 32) {
        const int ls = idx / KT2, k = idx - ls * KT2;
        const int l = ls0 + ls;
        const bool in = l < L && k < K;
        const float p0 = in ? ch.P[((size_t)l * K + k) * A] : 0.0f;
        const float p1 = (in && A > 1) ? ch.P[((size_t)l * K + k) * A + 1] : 0.0f;
        sX[((size_t)ls * 3 + 0) * KT2 + k] = make_float2(p0, p0);
        sX[((size_t)ls * 3 + 1) * KT2 + k] = make_float2(p0, p1);
        sX[((size_t)ls * 3 + 2) * KT2 + k] = make_float2(p1, p1);
      }
      __syncthreads();
      const uint4 wd = ivalid ? __ldg(gw + (size_t)(ls0 >> 6) * 32)
                              : make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
      uint32_t acc_lo = 0u, acc_hi = 0u;
      if (want_like) {
        if (store_z) ind_stage<KT, true, true>(ch, wd, Q2, sX, nsw, sNL, sML, ls0, i, ivalid, ncount,
                                               (uint32_t)rep, key, NB, acc_lo, acc_hi, like_acc);
        else ind_stage<KT, true, false>(ch, wd, Q2, sX, nsw, sNL, sML, ls0, i, ivalid, ncount,
                                        (uint32_t)rep, key, NB, acc_lo, acc_hi, like_acc);
      } else {
        if (store_z) ind_stage<KT, false, true>(ch, wd, Q2, sX, nsw, sNL, sML, ls0, i, ivalid, ncount,
                                                (uint32_t)rep, key, NB, acc_lo, acc_hi, like_acc);
        else ind_stage<KT, false, false>(ch, wd, Q2, sX, nsw, sNL, sML, ls0, i, ivalid, ncount,
                                         (uint32_t)rep, key, NB, acc_lo, acc_hi, like_acc);
      }
#pragma unroll
      for (int k = 0; k < KT; k++)
        mtot[k] += (int)(((k < 4 ? acc_lo : acc_hi) >> (8 * (k & 3))) & 255u);
      __syncthreads();
      // the stage's allele counts: the warps' sums per (locus, bin), into the
      // chain's histogram n[k][a][l]
      const int nl = min(kLS, l1 - ls0);
      for (int idx = threadIdx.x; idx < nl * NB; idx += kIW * 32) {
        const int ls = idx / NB, b = idx - ls * NB;
        int s = 0;
#pragma unroll
        for (int w = 0; w < kIW; w++) s += sNS[(w * kLS + ls) * NB + b];
        if (s && (A > 1 || (b & 1) == 0))
          atomicAdd(&ch.npart[((size_t)(b >> 1) * A + (b & 1)) * L + ls0 + ls], s);
      }
    }
    if (ivalid) {
#pragma unroll
      for (int k = 0; k < KT; k++)
        if (k < K && mtot[k]) atomicAdd(&ch.mpart[(size_t)i * K + k], mtot[k]);
    }
  }

  const int ntiles = ch.nchunks * ch.ngroups;
  if (want_like) {
    const double sres = zfast::block_sum_d(like_acc, sred);
    if (threadIdx.x == 0) ch.likepart[tile] = sres;
  }
  const bool advance = (flags & kZfAdvance) != 0;
  if (want_like || advance) {
    if (last_cta_arrive(&ch.ctr[kCtrZ], (unsigned)ntiles)) {
      if (want_like) zfast::finish_like(ch, ntiles, collect && (flags & kZfCollect), sred);
      if (advance && threadIdx.x == 0) *ch.rep = rep + 1;
    }
  }
}

template <int KT>
cudaError_t launch_ind_kt(const LaunchSet& ls, int flags) {
  const size_t smem = ilayout(KT).total;
  auto fn = zpass_ind_kernel<KT>;
  if (smem > 40 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  fn<<<ls.total_ctas, kIW * 32, smem, ls.stream>>>(ls.chains, ls.prefix, ls.nchains, flags);
  return cudaGetLastError();
}

}  // namespace zind
}  // namespace st
