// st_injected.cu -- parity modes of UpdateP and of the Metropolis Q update fed
// from caller arrays laid out like the reference's randomArr, with the
// reference's own samplers, so that a fixed chain state and the same array give
// the reference's results (up to the FP32 storage of P and Q):
//   * UpdateP (src/Updates/UpdateP.c:106-199): for each (locus, population) a
//     block of MAXALLELES*64 uniforms at (loc*K*A + pop*A)*64, consumed by
//     LogRDirichletDisc (src/ran.c:1248-1272) over RGammaDisc (ran.c:1094-1188);
//   * UpdateQMetro (src/Updates/UpdateQ.c:199-307): for each individual a block
//     of 64 uniforms at ind*64: RDirichletDisc (ran.c:1197-1210) of TestQ from
//     alpha, then the accept uniform (u < exp(logdiff)).
// The sweep itself draws from Philox with Marsaglia-Tsang; these entry points
// exist to pin the device's handling of the same state to the reference's
// functions.  Arithmetic is FP64 without contraction (this file is built with
// -fmad=false), in the reference's operation order.  Reading past a block's
// end (the reference exits) sets kErrGammaCap in the chain's error word and
// stops that draw.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "st_device.cuh"
#include "st_kernels.h"
#include "st_types.h"

namespace st {
namespace {

constexpr int kMaxRandom = 64;   // MAXRANDOM, src/structuredefs.h:11
constexpr double kUnderflo = 1e-100;

// Sequential reader of one block of the caller's array (RndDiscState,
// src/randGen.c:8-36): `taken` counts the values read, `cap` is the block's
// length; a read past it flags the caller and returns 0.5.
struct Cursor {
  const double* base;
  int taken, cap;
  bool over;
  __device__ double next() {
    if (taken >= cap) { over = true; return 0.5; }
    return base[taken++];
  }
};

// Gamma(n, 1) by the reference's sampler (Ripley 1987, p. 230): three regimes,
// n < 1 (a mixture rejection), n == 1 (von Neumann's exponential) and n > 1
// (a ratio-of-uniforms scheme with the extra squeeze above 2.5).  The
// rejection loops end on their own for any uniforms in (0,1); a block that
// runs out ends them as well (Cursor.over).
__device__ double ref_rgamma(double n, Cursor& cu) {
  if (n < 1.0) {
    const double e = 2.71828182;
    const double b = (n + e) / e;
    while (!cu.over) {
      const double p = b * cu.next();
      if (p > 1.0) {
        const double x = -log((b - p) / n);
        if (!(((n - 1.0) * log(x)) < log(cu.next()))) return x;
      } else {
        const double x = exp(log(p) / n);
        if (!(x > -log(cu.next()))) return x;
      }
    }
    return 1.0;
  }
  if (n == 1.0) {
    double a = 0.0;
    while (!cu.over) {
      double u = cu.next();
      const double u0 = u;
      for (;;) {
        const double ustar = cu.next();
        if (u < ustar) return (a + u0) / 1.0;
        u = cu.next();
        if (!(u < ustar) || cu.over) break;
      }
      a += 1.0;
    }
    return 1.0;
  }
  const double c1 = n - 1.0;
  const double aa = 1.0 / c1;
  const double c2 = aa * (n - 1.0 / (6.0 * n));
  const double c3 = 2.0 * aa;
  const double c4 = c3 + 2.0;
  const double c5 = n > 2.5 ? 1.0 / sqrt(n) : 0.0;
  while (!cu.over) {
    double u1 = cu.next();
    const double u2 = cu.next();
    if (n > 2.5) {
      u1 = u2 + c5 * (1.0 - 1.86 * u1);
      if (u1 <= 0.0 || u1 >= 1.0) continue;
    }
    const double w = c2 * u2 / u1;
    if (c3 * u1 + w + 1.0 / w < c4) return c1 * w;
    if (!(c3 * log(u1) - log(w) + w >= 1.0)) return c1 * w;
  }
  return 1.0;
}

// UpdateP with the reference's sampler: one thread per (locus, population).
__global__ void inj_p_kernel(ChainDev* __restrict__ chp, const double* __restrict__ uni) {
  ChainDev& ch = *chp;
  const int L = ch.L, K = ch.K, A = ch.A;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)L * K) return;
  const int l = (int)(t / K), k = (int)(t - (size_t)l * K);
  const int na = ch.numalleles[l];
  double g[kMaxAlleles];
  Cursor cu{uni + ((size_t)l * K * A + (size_t)k * A) * kMaxRandom, 0, A * kMaxRandom, false};
  double sum = 0.0;
  for (int a = 0; a < na; a++) {
    const double cnt = (double)ch.npart[((size_t)k * A + a) * L + l];
    const double par = ch.freqscorr
                           ? ch.eps[(size_t)l * A + a] * (1.0 - ch.F[k]) / ch.F[k] + cnt
                           : ch.lambda[k] + cnt;
    g[a] = ref_rgamma(par, cu);
    sum += g[a];
  }
  float* P = ch.P + ((size_t)l * K + k) * A;
  float* lP = ch.logP + ((size_t)l * K + k) * A;
  for (int a = 0; a < na; a++) {
    // the underflow patch of LogRDirichletDisc (ran.c:1262-1265)
    const double p = sum < kUnderflo ? 1.0 / (double)na : g[a] / sum;
    P[a] = (float)p;
    lP[a] = (float)log(p);
  }
  if (cu.over) set_err(ch.err, kErrGammaCap);
}

// The proposal of UpdateQMetro with the reference's sampler: one thread per
// individual; records how many of its 64 values the draw took (the accept
// uniform is the next one).
__global__ void inj_metro_propose_kernel(ChainDev* __restrict__ chp, const double* __restrict__ uni,
                                         int* __restrict__ taken) {
  ChainDev& ch = *chp;
  const int N = ch.N, K = ch.K;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (ch.usepopinfo && ch.popflags[i]) { taken[i] = -1; return; }   // UpdateQ.c:247
  const double* alpha = ch.alpha + (ch.lp_admix ? (size_t)(1 + ch.myloc[i]) * K : 0);
  Cursor cu{uni + (size_t)i * kMaxRandom, 0, kMaxRandom, false};
  double g[kMaxPops];
  double sum = 0.0;
  for (int k = 0; k < K; k++) {
    g[k] = ref_rgamma(alpha[k], cu);
    sum += g[k];
  }
  for (int k = 0; k < K; k++) {
    const double q = g[k] / sum;
    ch.TestQ[(size_t)i * K + k] = (float)q;
    ch.logTestQ[(size_t)i * K + k] = (float)log(q);
  }
  taken[i] = cu.over ? kMaxRandom : cu.taken;
  if (cu.over) set_err(ch.err, kErrGammaCap);
}

// The accept step of UpdateQMetro on the data pass's log ratios.
__global__ void inj_metro_accept_kernel(ChainDev* __restrict__ chp, const double* __restrict__ uni,
                                        const int* __restrict__ taken) {
  ChainDev& ch = *chp;
  const int N = ch.N, K = ch.K;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || taken[i] < 0) return;
  if (taken[i] >= kMaxRandom) { set_err(ch.err, kErrGammaCap); return; }
  double ld = 0.0;
  for (int g = 0; g < ch.ngroups; g++) ld += ch.ldpart[(size_t)g * N + i];
  if (uni[(size_t)i * kMaxRandom + taken[i]] < exp(ld)) {
    for (int k = 0; k < K; k++) {
      ch.Q[(size_t)i * K + k] = ch.TestQ[(size_t)i * K + k];
      ch.logQ[(size_t)i * K + k] = ch.logTestQ[(size_t)i * K + k];
    }
    atomicAdd(&ch.stats[kStMetroHits], 1.0);
  }
}

}  // namespace

cudaError_t launch_inj_p(const ChainDev& h, ChainDev* d_chain, const double* uni, cudaStream_t s) {
  const size_t n = (size_t)h.L * h.K;
  inj_p_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_chain, uni);
  return cudaGetLastError();
}

cudaError_t launch_inj_metro_propose(const ChainDev& h, ChainDev* d_chain, const double* uni,
                                     int* taken, cudaStream_t s) {
  inj_metro_propose_kernel<<<(unsigned)((h.N + 127) / 128), 128, 0, s>>>(d_chain, uni, taken);
  return cudaGetLastError();
}

cudaError_t launch_inj_metro_accept(const ChainDev& h, ChainDev* d_chain, const double* uni,
                                    const int* taken, cudaStream_t s) {
  inj_metro_accept_kernel<<<(unsigned)((h.N + 127) / 128), 128, 0, s>>>(d_chain, uni, taken);
  return cudaGetLastError();
}

}  // namespace st
