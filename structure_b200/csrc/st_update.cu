// st_update.cu -- the per-locus and per-individual updates of a sweep.
//
// Locus kernel (one thread per locus, a loop over the populations):
//   P   : P[l][k][.] ~ Dirichlet(prior + n[l][k][.])        Updates/UpdateP.c:106-199
//   eps : two-allele shift Metropolis on eps[l][.]           Updates/UpdateEpsilon.c:71-145
//   F   : per-locus terms of FlikeFreqs(F') - FlikeFreqs(F), reduced over loci,
//         then the Metropolis test on F_k by the last CTA     Updates/UpdateFst.c:10-51,142-204
// Individual kernel (G lanes per individual, lane k = population k):
//   Gibbs  : Q_i ~ Dirichlet(alpha + m_i)                    Updates/UpdateQ.c:387-424
//   Metro  : TestQ_i ~ Dirichlet(alpha); accept with prob
//            exp(logdiff_i) once the data pass summed it     Updates/UpdateQ.c:199-307
//   alpha  : sums of log Q_ik reduced over individuals, then the Metropolis
//            test on alpha by the last CTA                    Updates/UpdateAlpha.c:12-253
// Both fold their accumulators (PSum, SumEps, FstSum, QSum, AncestDist,
// sumAlpha, sumlambda; output.c:654-707 UpdateSums) when the sweep collects.
#include <algorithm>

#include "st_device.cuh"
#include "st_kernels.h"

namespace st {

namespace {

constexpr double kLogUnderflo = -230.25850929940458;  // log(1e-100), ran.c:1262
constexpr double kLogSqrtUnderflo = -115.12925464970229;  // log(1e-50)

// Sum one value per (warp, slot) into smem table s[warp][nslot]; slots of
// lanes that share a slot are reduced by xor-shuffles over strides >= G.
__device__ __forceinline__ void warp_slot_sums(double v, int G, double* s, int nslot,
                                               int slot) {
  for (int off = G; off < 32; off <<= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane < G && slot >= 0 && slot < nslot) s[warp * nslot + slot] = v;
}

}  // namespace

// ---------------------------------------------------------------------------
// Locus kernel: one thread per locus, looping over the populations (every
// lane busy whatever K is).  The per-population constants of the sweep --
// (1-F_k)/F_k and the F proposals -- are formed once per CTA in shared memory.
// ---------------------------------------------------------------------------
constexpr int kStageKA = 16;   // populations x alleles staged per locus (P stage)

__global__ void __launch_bounds__(256, 4)
locus_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix, int nchains,
             int stages) {
  __shared__ double sF[8 * kMaxPops];
  __shared__ double sTot[kMaxPops];
  __shared__ double sFrac[kMaxPops];   // (1 - F_k) / F_k
  __shared__ double sNF[kMaxPops];     // proposed F_j (F stage)
  // P stage, one lane per locus and K * A <= kStageKA: the CTA's new P and
  // log P, written to HBM (and added into PSum) row-contiguously afterwards
  __shared__ float sPst[256 * kStageKA];
  __shared__ float sLPst[256 * kStageKA];
  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int L = ch.L, K = ch.K, A = ch.A;
  // tpl lanes per locus (1 unless the chain has few loci): the P draws of a
  // locus are spread over them; eps and F run on the first lane of each locus
  const int tpl = ch.loc_tpl;
  const int l = tile * ((int)blockDim.x / tpl) + (int)threadIdx.x / tpl;
  const int sub = (int)threadIdx.x % tpl;
  const bool lvalid = l < L && sub == 0;
  const int rep = *ch.rep;
  const uint32_t key = ch.key;
  const bool collect = (stages & kLocCollect) && (rep + 1 > ch.burnin);
  const int na = (l < L) ? ch.numalleles[l] : 0;
  const bool fstage = (stages & kLocFst) && ch.freqscorr;
  const int numfst = ch.onefst ? 1 : K;
  if (ch.freqscorr && (stages & (kLocP | kLocEps | kLocFst))) {
    if (threadIdx.x < K) sFrac[threadIdx.x] = (1.0 - ch.F[threadIdx.x]) / ch.F[threadIdx.x];
    if (fstage && threadIdx.x < numfst)
      sNF[threadIdx.x] = ch.F[threadIdx.x] +
          ch.fpriorsd * normal_draw((uint32_t)threadIdx.x, (uint32_t)rep, kSFst, key);
    __syncthreads();
  }
  int errb = 0;

  // ---- P ------------------------------------------------------------------
  if ((stages & kLocP) && tpl > 1) {
    // lanes (k, j) of the locus: population k (strided by tpl / J when K
    // exceeds it), alleles a = j, j + J, ...; the Dirichlet's log-sum over the
    // alleles of (l, k) is a width-J butterfly over contiguous lanes
    int J = 1;
    while (J * 2 * K <= tpl && J * 2 <= 32) J *= 2;
    const int kslots = tpl / J;
    const int j = sub % J, k0 = sub / J;
    // lanes of a locus stay together through the loop: every lane runs the
    // same number of rounds
    for (int kb = 0; kb < K; kb += kslots) {
      const int k = kb + k0;
      const bool kv = l < L && na > 0 && k < K;
      const size_t base = ((size_t)(l < L ? l : 0) * K + (k < K ? k : 0)) * A;
      double lg[kMaxAlleles];
      double M = -INFINITY;
      int nmine = 0;
      if (kv) {
        for (int a = j; a < na && a < kMaxAlleles; a += J) {
          int n = 0;
          for (int cc = 0; cc < ch.cnt_chunks; cc++)
            n += ch.npart[(((size_t)cc * K + k) * A + a) * L + l];
          const double shape = ch.freqscorr ? ch.eps[(size_t)l * A + a] * sFrac[k] + (double)n
                                            : ch.lambda[k] + (double)n;
          lg[nmine] = (double)log_gamma_draw_f32((float)shape, (uint32_t)(base + a),
                                                 (uint32_t)rep, kSP, key, &errb);
          M = lg[nmine] > M ? lg[nmine] : M;
          nmine++;
        }
      }
      M = group_max(M, J);
      double S = 0.0;
      for (int t = 0; t < nmine; t++) S += exp(lg[t] - M);
      S = group_sum(S, J);
      const double ls = M + log(S);
      const int nac = na < kMaxAlleles ? na : kMaxAlleles;
      if (kv) {
        if (na > kMaxAlleles) errb |= kErrBounds;
        int t = 0;
        for (int a = j; a < nac; a += J, t++) {
          double lp, p;
          if (ls < kLogUnderflo) {
            p = 1.0 / (double)nac;
            lp = -log((double)nac);
          } else {
            lp = lg[t] - ls;
            p = exp(lp);
          }
          const float pf = (float)p;
          ch.P[base + a] = pf;
          ch.logP[base + a] = (float)lp;
          if (collect) ch.PSum[base + a] += (double)pf;
          if (!(pf == pf)) errb |= kErrNaN;
        }
      }
    }
  }
  // CTA-uniform (one chain per CTA): stage this CTA's P rows in shared memory
  const bool pstage = (stages & kLocP) && tpl == 1 && K * A <= kStageKA && blockDim.x <= 256;
  if ((stages & kLocP) && tpl == 1 && lvalid && na > 0) {
    for (int k = 0; k < K; k++) {
      const size_t base = ((size_t)l * K + k) * A;
      auto shape_of = [&](int a) {
        int n = 0;
        for (int cc = 0; cc < ch.cnt_chunks; cc++)
          n += ch.npart[(((size_t)cc * K + k) * A + a) * L + l];
        // eps (1-F)/F + n (Updates/UpdateP.c:161-164), with (1-F)/F formed once per CTA
        if (ch.freqscorr) return ch.eps[(size_t)l * A + a] * sFrac[k] + (double)n;
        return ch.lambda[k] + (double)n;
      };
      auto emit = [&](int a, double lg, double ls, int nac) {
        double lp, p;
        if (ls < kLogUnderflo) {
          p = 1.0 / (double)nac;
          lp = -log((double)nac);
        } else {
          lp = lg - ls;
          p = exp(lp);
        }
        const float pf = (float)p;
        if (pstage) {
          sPst[threadIdx.x * (K * A) + k * A + a] = pf;
          sLPst[threadIdx.x * (K * A) + k * A + a] = (float)lp;
        } else {
          ch.P[base + a] = pf;
          ch.logP[base + a] = (float)lp;
          if (collect) ch.PSum[base + a] += (double)pf;
        }
        if (!(pf == pf)) errb |= kErrNaN;
      };
      if (na <= 2) {
        // biallelic (and monomorphic) loci stay in registers
        const double lg0 = (double)log_gamma_draw_f32((float)shape_of(0), (uint32_t)base,
                                                      (uint32_t)rep, kSP, key, &errb);
        const double lg1 = na > 1 ? (double)log_gamma_draw_f32((float)shape_of(1),
                                                               (uint32_t)(base + 1),
                                                               (uint32_t)rep, kSP, key, &errb)
                                  : -INFINITY;
        const double M = (na > 1 && lg1 > lg0) ? lg1 : lg0;
        double S = exp(lg0 - M);
        if (na > 1) S += exp(lg1 - M);
        const double ls = M + log(S);
        emit(0, lg0, ls, na);
        if (na > 1) emit(1, lg1, ls, na);
      } else {
        double lg[kMaxAlleles];
        const int nac = na < kMaxAlleles ? na : kMaxAlleles;
        if (na > kMaxAlleles) errb |= kErrBounds;
        for (int a = 0; a < nac; a++)
          lg[a] = (double)log_gamma_draw_f32((float)shape_of(a), (uint32_t)(base + a),
                                             (uint32_t)rep, kSP, key, &errb);
        double M = lg[0];
        for (int a = 1; a < nac; a++) M = lg[a] > M ? lg[a] : M;
        double S = 0.0;
        for (int a = 0; a < nac; a++) S += exp(lg[a] - M);
        const double ls = M + log(S);
        for (int a = 0; a < nac; a++) emit(a, lg[a], ls, nac);
      }
    }
  }

  if (pstage) {
    // rows l0 .. l0 + nl - 1 of P, log P and PSum are contiguous: [l][k][a]
    __syncthreads();
    const int KA = K * A;
    const int l0 = tile * (int)blockDim.x;
    const int nl = min((int)blockDim.x, L - l0);
    const size_t g0 = (size_t)l0 * KA;
    for (int idx = threadIdx.x; idx < nl * KA; idx += blockDim.x) {
      const int li = idx / KA;
      const int a = (idx - li * KA) % A;
      const int nal = ch.numalleles[l0 + li];
      if (a < (nal < kMaxAlleles ? nal : kMaxAlleles)) {
        const float pf = sPst[idx];
        ch.P[g0 + idx] = pf;
        ch.logP[g0 + idx] = sLPst[idx];
        if (collect) ch.PSum[g0 + idx] += (double)pf;
      }
    }
    __syncthreads();   // the eps stage reads this CTA's log P rows
  }

  // ---- eps ----------------------------------------------------------------
  if ((stages & kLocEps) && ch.freqscorr && lvalid) {
    if (na > 1) {
      const U4 w = philox_s((uint32_t)l, 0, (uint32_t)rep, kSEps, key);
      const int a1 = (int)(((double)(w.x >> 1) / 2147483648.0) * na);
      int a2 = (int)(((double)(w.y >> 1) / 2147483648.0) * (na - 1));
      if (a2 >= a1) a2 += 1;
      const double d = 0.0 + ((double)(w.z >> 1) / 2147483648.0) * (ch.invsqrtnuminds - 0.0);
      const double e1 = ch.eps[(size_t)l * A + a1];
      const double e2 = ch.eps[(size_t)l * A + a2];
      if ((e1 + d < 1.0) && (e2 - d > 0.0)) {
        double sum = 0.0;
        for (int k = 0; k < K; k++) {
          const double frac = sFrac[k];
          const size_t base = ((size_t)l * K + k) * A;
          const double lp1 = (double)ch.logP[base + a1];
          const double lp2 = (double)ch.logP[base + a2];
          double s = lanczos_lgamma_fast(frac * e1);
          s += lanczos_lgamma_fast(frac * e2);
          s -= lanczos_lgamma_fast(frac * (e1 + d));
          s -= lanczos_lgamma_fast(frac * (e2 - d));
          s += frac * d * lp1;
          s -= frac * d * lp2;
          sum += s;
        }
        const double lam = ch.lambda[0];
        if (lam != 1.0) sum += log(pow((e1 + d) * (e2 - d) / e1 / e2, lam - 1.0));
        const U4 u = philox_s((uint32_t)l, 1, (uint32_t)rep, kSEps, key);
        if (rnd31(u) < exp(sum)) {
          ch.eps[(size_t)l * A + a1] = e1 + d;
          ch.eps[(size_t)l * A + a2] = e2 - d;
        }
      }
    }
    if (collect)
      for (int a = 0; a < na; a++) ch.SumEps[(size_t)l * A + a] += ch.eps[(size_t)l * A + a];
  }

  // ---- F ------------------------------------------------------------------
  if (fstage) {
    // per-warp sums of each proposal's locus terms, then CTA sums in warp order
    const int nwarps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto fterm = [&](int k, double nf) {
      double v = 0.0;
      if (lvalid && nf > 0.0 && nf < 1.0) {
        const double nfr = (1.0 - nf) / nf, ofr = sFrac[k];
        const size_t base = ((size_t)l * K + k) * A;
        for (int a = 0; a < na; a++) {
          const double e = ch.eps[(size_t)l * A + a];
          const double lp = (double)ch.logP[base + a];
          v += (nfr - ofr) * e * lp - (lanczos_lgamma_fast(nfr * e) - lanczos_lgamma_fast(ofr * e));
        }
      }
      return v;
    };
    for (int j = 0; j < numfst; j++) {
      double v = 0.0;
      if (ch.onefst) {
        for (int k = 0; k < K; k++) v += fterm(k, sNF[0]);
      } else {
        v = fterm(j, sNF[j]);
      }
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) sF[warp * numfst + j] = v;
    }
    __syncthreads();
    const int nblocks = (L * tpl + blockDim.x - 1) / blockDim.x;
    if (threadIdx.x < numfst) {
      double s = 0.0;
      for (int w = 0; w < nwarps; w++) s += sF[w * numfst + threadIdx.x];
      ch.redpart[(size_t)tile * numfst + threadIdx.x] = s;
    }
    if (last_cta_arrive(&ch.ctr[kCtrLocus], (unsigned)nblocks)) {
      if (threadIdx.x < numfst) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += ch.redpart[(size_t)b * numfst + threadIdx.x];
        sTot[threadIdx.x] = s;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        const double m = ch.fpriormean, sd = ch.fpriorsd;
        for (int jj = 0; jj < numfst; jj++) {
          const double oldf = ch.F[jj];
          const double nf = sNF[jj];
          ch.stats[kStFstNew + jj] = nf;
          ch.stats[kStFstDiff + jj] = sTot[jj];
          if (!(nf > 0.0 && nf < 1.0)) { ch.stats[kStFstLpd + jj] = 0.0; continue; }
          double lpd = (m * m / (sd * sd) - 1) * log(nf / oldf) + (oldf - nf) * m / (sd * sd);
          const double nfr = (1.0 - nf) / nf, ofr = (1.0 - oldf) / oldf;
          const int npops = ch.onefst ? K : 1;
          lpd += (double)ch.Leff * npops * (lanczos_lgamma_fast(nfr) - lanczos_lgamma_fast(ofr)) + sTot[jj];
          ch.stats[kStFstLpd + jj] = lpd;
          bool acc = lpd >= 0.0;
          if (!acc) acc = rnd31(philox_s((uint32_t)jj, 1, (uint32_t)rep, kSFst, key)) < exp(lpd);
          if (acc) {
            if (ch.onefst) { for (int q = 0; q < K; q++) ch.F[q] = nf; }
            else ch.F[jj] = nf;
          }
        }
        if (collect)
          for (int q = 0; q < K; q++) ch.FstSum[q] += ch.F[q];
      }
    }
  } else if ((stages & kLocCollect) && collect && ch.freqscorr && tile == 0 && threadIdx.x == 0) {
    for (int q = 0; q < K; q++) ch.FstSum[q] += ch.F[q];
  }
  if (errb) set_err(ch.err, errb);
}

// A new chain's start (src/Init.c:329-444): its descriptor and prefix, Q = 1/K,
// the initial eps of its data set (computed once per data set and prior on the
// host, kept on the device), F, alpha and lambda; the rest of the chain's arrays
// are zeroed by memsets.  Written by a kernel rather than copied from host
// memory, so creating a chain does not wait for the previous chain's initial
// Z pass.
__global__ void init_chain_kernel(ChainDev h, ChainDev* d_chain, int* d_prefix,
                                  const double* __restrict__ eps0, size_t LA, size_t NK,
                                  int arows, float q0, float lq0, double f0, double alpha0,
                                  double lambda0) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  if (t == 0) {
    *d_chain = h;
    *d_prefix = 0;
  }
  for (size_t j = t; j < NK; j += stride) {
    h.Q[j] = q0;
    h.logQ[j] = lq0;
  }
  for (size_t j = t; j < LA; j += stride) h.eps[j] = eps0[j];
  for (size_t j = t; j < (size_t)arows * h.K; j += stride) h.alpha[j] = alpha0;
  if (t < (size_t)h.K) {
    h.F[t] = f0;
    h.lambda[t] = lambda0;
  }
}

cudaError_t launch_init_chain(const ChainDev& h, ChainDev* d_chain, int* d_prefix,
                              const double* eps0, int arows, float q0, float lq0, double f0,
                              double alpha0, double lambda0, cudaStream_t s) {
  const size_t LA = (size_t)h.L * h.A, NK = (size_t)h.N * h.K;
  const size_t n = std::max(std::max(LA, NK), (size_t)arows * h.K);
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
  init_chain_kernel<<<grid > 0 ? grid : 1, 256, 0, s>>>(h, d_chain, d_prefix, eps0, LA, NK, arows,
                                                        q0, lq0, f0, alpha0, lambda0);
  return cudaGetLastError();
}

int ctas_locus(const ChainDev& c, int block) { return (c.L * c.loc_tpl + block - 1) / block; }

// Lanes per locus of the locus kernel: 1 for most chains; with fewer loci
// than about two waves of threads, up to 32 per locus (a power of two), so a
// small chain's Dirichlet draws run in parallel over populations and alleles,
// but no more lanes than there are (population, allele) draws to spread:
// the lanes of a locus cover populations x alleles in powers of two.
int locus_lanes(int L, int K, int A) {
  int t = 1;
  while (t < 32 && (size_t)L * t * 2 <= (size_t)148 * 256 * 2) t *= 2;
  int kp = 1, ap = 1;
  while (kp < K) kp *= 2;
  while (ap < A) ap *= 2;
  return t < kp * ap ? t : kp * ap;
}

cudaError_t launch_locus(const LaunchSet& ls, int stages, int block) {
  locus_kernel<<<ls.total_ctas, block, 0, ls.stream>>>(ls.chains, ls.prefix, ls.nchains, stages);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Lambda kernel: UpdateLambda / UpdatePopLambda (Updates/UpdateLambda.c:8-102).
// Metropolis on lambda under a uniform prior on (0, LAMBDAMAX = 10), proposal
// N(lambda, LAMBDAPROPSD = 0.3); one value (all populations share it), or one
// per population with POPSPECIFICLAMBDA.  Log ratio, summed over loci with
// more than one allele:
//   reps * [lgamma(na new) - lgamma(na lambda) + na lgamma(lambda) - na lgamma(new)]
//   + (new - lambda) * sum_reps sum_a log freq,
// where the frequencies are P of population q (per population), or eps
// (FREQSCORR, reps = 1) or P of every population (reps = K).  Thread = locus;
// per-CTA sums go to redpart, the last CTA adds them in order and decides.
// Draws: the normal at (q, 0), the rand()-style uniform at (q, 1) of stream
// kSLambda.
// ---------------------------------------------------------------------------
namespace {
constexpr double kLambdaMax = 10.0;      // structure.h:19 LAMBDAMAX
constexpr double kLambdaPropSd = 0.3;    // structure.h:20 LAMBDAPROPSD
}  // namespace

__global__ void __launch_bounds__(256)
lambda_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix, int nchains) {
  __shared__ double sred[8];
  __shared__ double snew[kMaxPops];
  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int L = ch.L, K = ch.K, A = ch.A;
  const int rep = *ch.rep;
  const uint32_t key = ch.key;
  const int npop = ch.popspecificlambda ? K : 1;
  const int nblocks = (L + blockDim.x - 1) / blockDim.x;
  if (threadIdx.x < npop)
    snew[threadIdx.x] = ch.lambda[threadIdx.x] +
                        kLambdaPropSd * normal_draw((uint32_t)threadIdx.x, (uint32_t)rep, kSLambda, key);
  __syncthreads();
  const int l = tile * blockDim.x + threadIdx.x;
  const int na = l < L ? ch.numalleles[l] : 0;
  for (int q = 0; q < npop; q++) {
    const double lam = ch.lambda[q], nw = snew[q];
    double term = 0.0;
    if (na > 1 && nw > 0.0 && nw < kLambdaMax) {
      const double reps = ch.popspecificlambda ? 1.0 : (ch.freqscorr ? 1.0 : (double)K);
      term = reps * (lanczos_lgamma(na * nw) - lanczos_lgamma(na * lam) +
                     na * lanczos_lgamma(lam) - na * lanczos_lgamma(nw));
      double slog = 0.0;
      if (ch.popspecificlambda) {
        for (int a = 0; a < na; a++) slog += (double)ch.logP[((size_t)l * K + q) * A + a];
      } else if (ch.freqscorr) {
        for (int a = 0; a < na; a++) slog += log(ch.eps[(size_t)l * A + a]);
      } else {
        for (int k = 0; k < K; k++)
          for (int a = 0; a < na; a++) slog += (double)ch.logP[((size_t)l * K + k) * A + a];
      }
      term += (nw - lam) * slog;
    }
    for (int off = 16; off > 0; off >>= 1) term += __shfl_down_sync(0xffffffffu, term, off);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = term;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += sred[w];
      ch.redpart[(size_t)tile * npop + q] = sum;
    }
    __syncthreads();
  }
  if (last_cta_arrive(&ch.ctr[kCtrLambda], (unsigned)nblocks) && threadIdx.x < npop) {
    const int q = threadIdx.x;
    double sum = 0.0;
    for (int b = 0; b < nblocks; b++) sum += ch.redpart[(size_t)b * npop + q];
    const double nw = snew[q];
    ch.stats[kStLambdaLpd + q] = sum;
    if (nw > 0.0 && nw < kLambdaMax &&
        rnd31(philox_s((uint32_t)q, 1, (uint32_t)rep, kSLambda, key)) < exp(sum)) {
      if (ch.popspecificlambda) {
        ch.lambda[q] = nw;
      } else {
        for (int k = 0; k < K; k++) ch.lambda[k] = nw;
      }
    }
  }
}

int ctas_lambda(const ChainDev& c, int block) { return (c.L + block - 1) / block; }

cudaError_t launch_lambda(const LaunchSet& ls, int block) {
  lambda_kernel<<<ls.total_ctas, block, 0, ls.stream>>>(ls.chains, ls.prefix, ls.nchains);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Individual kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
ind_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix, int nchains,
           int G, int mode, int stages) {
  __shared__ double sA[8 * (kMaxPops + 1)];
  __shared__ double sTot[kMaxPops + 1];
  __shared__ int sHits;
  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int N = ch.N, K = ch.K;
  const int gpb = blockDim.x / G;
  const int gid = threadIdx.x / G, k = threadIdx.x - gid * G;
  const int i = tile * gpb + gid;
  const bool ivalid = i < N;
  const bool kvalid = ivalid && k < K;
  const int rep = *ch.rep;
  const uint32_t key = ch.key;
  const bool collect = (stages & kIndCollect) && (rep + 1 > ch.burnin);
  const size_t qi = (size_t)(ivalid ? i : 0) * K + (k < K ? k : 0);
  // USEPOPINFO: flagged individuals keep the migrant-model Q drawn before this
  // kernel in both the Gibbs and the Metropolis sweep and are left out of the
  // alpha update (src/Updates/UpdateQ.c:247,407,727-729, UpdateAlpha.c:37)
  const bool flagged = ch.usepopinfo && ivalid && ch.popflags[i];
  int errb = 0;
  if (threadIdx.x == 0) sHits = 0;
  __syncthreads();

  float qf = 0.0f, lqf = 0.0f;  // Q_ik and log Q_ik after this kernel's update
  if (mode == kIndGibbs || mode == kIndPropose) {
    double lg = -INFINITY;
    if (kvalid) {
      // LOCPRIOR with admixture: the individual's location row of alpha
      // (src/Updates/UpdateQ.c:255-257,409-413)
      double shape = ch.alpha[(ch.lp_admix ? (size_t)(1 + ch.myloc[i]) * K : 0) + k];
      uint32_t stream = kSQM;
      if (mode == kIndGibbs) {
        int m = 0;
        for (int g = 0; g < ch.cnt_groups; g++) m += ch.mpart[((size_t)g * N + i) * K + k];
        shape += (double)m;
        stream = kSQG;
      }
      lg = log_gamma_draw(shape, (uint32_t)(i * K + k), (uint32_t)rep, stream, key, &errb);
    }
    const double M = group_max(lg, G);
    const double e = kvalid ? exp(lg - M) : 0.0;
    const double S = group_sum(e, G);
    const double ls = M + log(S);
    if (kvalid && flagged && mode == kIndGibbs) {
      qf = ch.Q[qi];
      lqf = ch.logQ[qi];
    } else if (kvalid) {
      const double lq = lg - ls;
      lqf = (float)lq;
      qf = (float)exp(lq);
      if (!(qf == qf)) errb |= kErrNaN;
      if (mode == kIndGibbs) { ch.Q[qi] = qf; ch.logQ[qi] = lqf; }
      else { ch.TestQ[qi] = qf; ch.logTestQ[qi] = lqf; }
    }
  } else if (mode == kIndAccept) {
    double ld = 0.0;
    if (ivalid)
      for (int g = 0; g < ch.ngroups; g++) ld += ch.ldpart[(size_t)g * N + i];
    bool acc = false;
    if (ivalid && !flagged) {
      const U4 w = philox_s((uint32_t)i, 0, (uint32_t)rep, kSQMA, key);
      acc = u01(w.x, w.y) < exp(ld);
    }
    if (kvalid) {
      if (acc) {
        qf = ch.TestQ[qi]; lqf = ch.logTestQ[qi];
        ch.Q[qi] = qf; ch.logQ[qi] = lqf;
      } else {
        qf = ch.Q[qi]; lqf = ch.logQ[qi];
      }
    }
    if (acc && k == 0) atomicAdd(&sHits, 1);
  } else if (kvalid) {
    qf = ch.Q[qi];
    lqf = ch.logQ[qi];
  }

  if (collect && kvalid && mode != kIndPropose) {
    ch.QSum[qi] += (double)qf;
    if (ch.ancestdist) {
      int box = (int)((double)qf * (double)ch.numboxes);
      if (box >= ch.numboxes) box = ch.numboxes - 1;
      if (box < 0) box = 0;
      ch.AncestDist[qi * ch.numboxes + box] += 1;
    }
  }

  if ((stages & kIndAlpha) && ch.inferalpha && mode != kIndPropose) {
    const int nslot = K + 1;
    const int nwarps = blockDim.x >> 5;
    for (int idx = threadIdx.x; idx < nwarps * nslot; idx += blockDim.x) sA[idx] = 0.0;
    __syncthreads();
    const bool counted = kvalid && !flagged;
    const double lq = counted ? (double)lqf : 0.0;
    const double lc = counted ? (lq > kLogSqrtUnderflo ? lq : kLogSqrtUnderflo) : 0.0;
    warp_slot_sums(lq, G, sA, nslot, k < K ? k : -1);
    double tsum = lc;
    for (int off = 1; off < 32; off <<= 1) tsum += __shfl_xor_sync(0xffffffffu, tsum, off);
    if ((threadIdx.x & 31) == 0) sA[(threadIdx.x >> 5) * nslot + K] = tsum;
    __syncthreads();
    const int nblocks = (N + gpb - 1) / gpb;
    if (threadIdx.x < nslot) {
      double s = 0.0;
      for (int w = 0; w < nwarps; w++) s += sA[w * nslot + threadIdx.x];
      ch.redpart[(size_t)tile * nslot + threadIdx.x] = s;
    }
    if (sHits && threadIdx.x == 0) atomicAdd(&ch.stats[kStMetroHits], (double)sHits);
    if (last_cta_arrive(&ch.ctr[kCtrInd], (unsigned)nblocks)) {
      if (threadIdx.x < nslot) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += ch.redpart[(size_t)b * nslot + threadIdx.x];
        sTot[threadIdx.x] = s;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double* alpha = ch.alpha;
        const double T = sTot[K];
        ch.stats[kStAlphaT] = T;
        for (int q = 0; q < K; q++) ch.stats[kStAlphaS + q] = sTot[q];
        const int numalphas = ch.popalphas ? K : 1;
        double logprobdiff = 0.0;
        for (int pop = 0; pop < numalphas; pop++) {
          const double newalpha = alpha[pop] + ch.alphapropsd *
              normal_draw((uint32_t)pop, (uint32_t)rep, kSAlpha, key);
          ch.stats[kStAlphaNew + pop] = newalpha;
          if ((newalpha > 0) && ((newalpha < ch.alphamax) || (!(ch.unifprioralpha)))) {
            if (!(ch.unifprioralpha))
              logprobdiff = (ch.alphapriora - 1) * log(newalpha / alpha[pop]) +
                            (alpha[pop] - newalpha) / ch.alphapriorb;
            if (ch.popalphas) {
              double sumalphas = 0.0;
              for (int q = 0; q < K; q++) sumalphas += alpha[q];
              logprobdiff -= (alpha[pop] - 1.0) * sTot[pop] +
                             (lanczos_lgamma_fast(sumalphas) - lanczos_lgamma_fast(alpha[pop])) * ch.alpha_n;
              sumalphas += newalpha - alpha[pop];
              logprobdiff += (newalpha - 1.0) * sTot[pop] +
                             (lanczos_lgamma_fast(sumalphas) - lanczos_lgamma_fast(newalpha)) * ch.alpha_n;
            } else {
              logprobdiff += (newalpha - 1.0) * T +
                             (lanczos_lgamma_fast(K * newalpha) - K * lanczos_lgamma_fast(newalpha)) * ch.alpha_n;
              logprobdiff -= (alpha[pop] - 1.0) * T +
                             (lanczos_lgamma_fast(K * alpha[pop]) - K * lanczos_lgamma_fast(alpha[pop])) * ch.alpha_n;
            }
            ch.stats[kStAlphaLpd + pop] = logprobdiff;
            const double unifrv = rnd31(philox_s((uint32_t)pop, 1, (uint32_t)rep, kSAlpha, key));
            if (unifrv < exp(logprobdiff)) {
              alpha[pop] = newalpha;
              if (!(ch.popalphas))
                for (int q = 1; q < K; q++) alpha[q] = newalpha;
            }
          }
        }
        if (collect) {
          for (int q = 0; q < K; q++) {
            ch.sumAlpha[q] += alpha[q];
            ch.sumlambda[q] += ch.lambda[q];
          }
        }
      }
    }
  } else {
    __syncthreads();
    if (sHits && threadIdx.x == 0) atomicAdd(&ch.stats[kStMetroHits], (double)sHits);
    if (collect && tile == 0 && threadIdx.x == 0)
      for (int q = 0; q < K; q++) {
        // src/output.c:72-83: no alpha sums under NOADMIX or NOALPHA; with
        // LOCPRIOR and admixture the location-alpha kernels add them
        if (!ch.inferalpha && !ch.noadmix && !ch.noalpha && !ch.lp_admix)
          ch.sumAlpha[q] += ch.alpha[q];
        ch.sumlambda[q] += ch.lambda[q];
      }
  }
  if (errb) set_err(ch.err, errb);
}

int ctas_ind(const ChainDev& c, int block) {
  const int gpb = block / c.G;
  return (c.N + gpb - 1) / gpb;
}

cudaError_t launch_ind(const LaunchSet& ls, int G, int mode, int stages, int block) {
  ind_kernel<<<ls.total_ctas, block, 0, ls.stream>>>(ls.chains, ls.prefix, ls.nchains, G,
                                                      mode, stages);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Standalone DataCollection (output.c:50-101 with UpdateSums 654-707); the
// fused sweep folds these sums into the kernels above instead.
// ---------------------------------------------------------------------------
__global__ void collect_kernel(ChainDev* __restrict__ chains, const int* __restrict__ prefix,
                               int nchains) {
  const int c = find_chain(prefix, nchains, blockIdx.x);
  ChainDev& ch = chains[c];
  const int tile = blockIdx.x - prefix[c];
  const int N = ch.N, L = ch.L, K = ch.K, A = ch.A;
  const size_t t = (size_t)tile * blockDim.x + threadIdx.x;
  if (t < (size_t)N * K) {
    const float q = ch.Q[t];
    ch.QSum[t] += (double)q;
    if (ch.ancestdist) {
      int box = (int)((double)q * (double)ch.numboxes);
      if (box >= ch.numboxes) box = ch.numboxes - 1;
      if (box < 0) box = 0;
      ch.AncestDist[t * ch.numboxes + box] += 1;
    }
  }
  if (t < (size_t)L * K * A) {
    const int l = (int)(t / ((size_t)K * A));
    const int a = (int)(t % A);
    if (a < ch.numalleles[l]) ch.PSum[t] += (double)ch.P[t];
  }
  if (ch.freqscorr && t < (size_t)L * A) {
    const int l = (int)(t / A), a = (int)(t % A);
    if (a < ch.numalleles[l]) ch.SumEps[t] += ch.eps[t];
  }
  if (tile == 0 && threadIdx.x == 0) {
    for (int q = 0; q < K; q++) {
      ch.sumlambda[q] += ch.lambda[q];
      ch.sumAlpha[q] += ch.alpha[q];
      if (ch.freqscorr) ch.FstSum[q] += ch.F[q];
    }
    if (ch.computeprob) {
      const double like = ch.stats[kStLike];
      ch.stats[kStSumLikes] += like;
      ch.stats[kStSumSq] += like * like;
      ch.stats[kStNLike] += 1.0;
    }
  }
}

int ctas_collect(const ChainDev& c, int block) {
  size_t n = (size_t)c.N * c.K;
  const size_t np = (size_t)c.L * c.K * c.A;
  if (np > n) n = np;
  return (int)((n + block - 1) / block);
}

cudaError_t launch_collect(const LaunchSet& ls, int block) {
  collect_kernel<<<ls.total_ctas, block, 0, ls.stream>>>(ls.chains, ls.prefix, ls.nchains);
  return cudaGetLastError();
}

}  // namespace st
