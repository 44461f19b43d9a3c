// st_popinfo.cu -- USEPOPINFO: Q of individuals flagged with a given
// population under the migrant model (src/Updates/UpdateQ.c:499-706
// UpdateQWithPops).
//
// An individual from population h is either not a migrant (prior
// 1 - MIGRPRIOR) or has one ancestor from population k != h exactly `gen`
// generations back, gen = 0..GENSBACK, with prior MIGRPRIOR * 2^gen /
// sum_gen' 2^gen' (K-1).  The likelihood of its genotype at a locus under
// (k, gen) mixes P_k and P_h:
//   gen 0      : P_k(a0) P_k(a1)
//   gen g > 0  : p/2 P_k(a0) P_h(a1) + p/2 P_h(a0) P_k(a1) + (1-p) P_h(a0) P_h(a1),
//                p = 2^-(g-1)
//   one copy   : p P_k(a0) + (1-p) P_h(a0) if only copy 0 is present, and
//                P_h(a1) if only copy 1 is (kept from the reference)
// each clamped below at sqrt(1e-100) as the reference's running product is.
// Thread = flagged individual; CTAs split the loci into chunks whose sums of
// log likelihoods go to pipart[chunk][i][k][gen].  The pick kernel adds the
// chunks, forms the posterior, adds it to UsePopProbs from sweep BURNIN on,
// and picks (gen, k) in gen-major order with u * sum < cumulative sum, u =
// rand()/2^31 from the Philox word at (i, 0) of stream kSPopInfo; then
// Q_k = 2^-gen and Q_h += 1 - 2^-gen.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "st_device.cuh"
#include "st_kernels.h"

namespace st {
namespace {

constexpr int kPiBlock = 256;
constexpr int kMaxGens = 8;     // GENSBACK <= 7
constexpr double kSqrtUnderflo = 1e-50;

__global__ void __launch_bounds__(kPiBlock) popinfo_ll_kernel(const ChainDev* __restrict__ chp) {
  const ChainDev& ch = *chp;
  const int N = ch.N, L = ch.L, K = ch.K, A = ch.A, G = ch.gensback + 1;
  const int i = blockIdx.x * kPiBlock + threadIdx.x;
  if (i >= N || !ch.popflags[i]) return;
  const int home = ch.population[i] - 1;
  const int l0 = blockIdx.y * ch.pi_lchunk_len;
  const int l1 = min(L, l0 + ch.pi_lchunk_len);
  double* out = ch.pipart + ((size_t)blockIdx.y * N + i) * K * G;
  for (int k = 0; k < K; k++) {
    double acc[kMaxGens];
    for (int g = 0; g < G; g++) acc[g] = 0.0;
    for (int l = l0; l < l1; l++) {
      int a0, a1;
      if (ch.layout == kLayoutB2G) {
        const uint32_t gt = (__ldg(ch.g2 + (size_t)l * ch.wpr + (i >> 4)) >> (2 * (i & 15))) & 3u;
        if (gt == 3u) continue;               // both copies missing: likelihood 1
        a0 = (int)(gt >> 1);
        a1 = (int)((gt | (gt >> 1)) & 1u);
      } else {
        const uint8_t b0 = __ldg(ch.g8 + ((size_t)i * 2) * L + l);
        const uint8_t b1 = __ldg(ch.g8 + ((size_t)i * 2 + 1) * L + l);
        a0 = b0 == kG8Missing ? -1 : b0;
        a1 = b1 == kG8Missing ? -1 : b1;
        if (a0 < 0 && a1 < 0) continue;
      }
      const float* P = ch.P + (size_t)l * K * A;
      const double pk0 = a0 >= 0 ? (double)P[k * A + a0] : 0.0;
      const double ph0 = a0 >= 0 ? (double)P[home * A + a0] : 0.0;
      const double pk1 = a1 >= 0 ? (double)P[k * A + a1] : 0.0;
      const double ph1 = a1 >= 0 ? (double)P[home * A + a1] : 0.0;
      for (int g = 0; g < G; g++) {
        const double p = g > 0 ? exp((g - 1) * log(0.5)) : 1.0;
        double like;
        if (a0 >= 0 && a1 >= 0) {
          like = g == 0 ? pk0 * pk1
                        : 0.5 * p * pk0 * ph1 + 0.5 * p * ph0 * pk1 + (1.0 - p) * ph0 * ph1;
        } else if (a0 >= 0) {
          like = p * pk0 + (1.0 - p) * ph0;
        } else {
          like = p * ph1 + (1.0 - p) * ph1;
        }
        acc[g] += log(like > kSqrtUnderflo ? like : kSqrtUnderflo);
      }
    }
    for (int g = 0; g < G; g++) out[k * G + g] = acc[g];
  }
}

__global__ void __launch_bounds__(kPiBlock) popinfo_pick_kernel(const ChainDev* __restrict__ chp) {
  const ChainDev& ch = *chp;
  const int N = ch.N, K = ch.K, G = ch.gensback + 1;
  const int i = blockIdx.x * kPiBlock + threadIdx.x;
  if (i >= N || !ch.popflags[i]) return;
  const int home = ch.population[i] - 1;
  const int rep = *ch.rep;
  double post[kMaxPops * kMaxGens];
  double mx = 0.0;
  for (int j = 0; j < K * G; j++) {
    double s = 0.0;
    for (int c = 0; c < ch.pi_lchunks; c++) s += ch.pipart[((size_t)c * N + i) * K * G + j];
    post[j] = s;
    if (j == 0 || s > mx) mx = s;
  }
  double pri[kMaxGens], w = 0.5, sw = 0.0;
  for (int g = 0; g < G; g++) {
    w *= 2.0;
    pri[g] = w;
    sw += w * (K - 1);
  }
  for (int g = 0; g < G; g++) pri[g] = ch.migrprior * pri[g] / sw;
  double sum = 0.0;
  for (int g = 0; g < G; g++)
    for (int k = 0; k < K; k++) {
      double& v = post[k * G + g];
      v = exp(v - mx);
      if (k == home) v = g == 0 ? v * (1.0 - ch.migrprior) : 0.0;
      else v *= pri[g];
      sum += v;
    }
  if (rep >= ch.burnin)
    for (int j = 0; j < K * G; j++) ch.usepop[(size_t)i * K * G + j] += post[j] / sum;
  const U4 u = philox_s((uint32_t)i, 0u, (uint32_t)rep, kSPopInfo, ch.key);
  const double r = (double)(u.x >> 1) / 2147483648.0 * sum;
  double cum = 0.0;
  int pk = home, pg = 0;
  bool done = false;
  for (int g = 0; g < G && !done; g++)
    for (int k = 0; k < K; k++) {
      cum += post[k * G + g];
      if (r < cum) {
        pk = k;
        pg = g;
        done = true;
        break;
      }
    }
  float* Q = ch.Q + (size_t)i * K;
  float* lQ = ch.logQ + (size_t)i * K;
  double q[kMaxPops];
  for (int k = 0; k < K; k++) q[k] = 0.0;
  const double p = exp(pg * log(0.5));
  q[pk] = p;
  q[home] += 1.0 - p;
  for (int k = 0; k < K; k++) {
    Q[k] = (float)q[k];
    lQ[k] = q[k] > 0.0 ? (float)log(q[k]) : -INFINITY;
  }
}

}  // namespace

void popinfo_plan(int N, int L, int* lchunks, int* lchunk_len) {
  const int tiles = (N + kPiBlock - 1) / kPiBlock;
  int ch = (148 * 4 + tiles - 1) / tiles;
  if (ch < 1) ch = 1;
  int len = (L + ch - 1) / ch;
  if (len < 64) len = 64;
  *lchunk_len = len;
  *lchunks = (L + len - 1) / len;
}

cudaError_t launch_popinfo(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s) {
  const dim3 g((h.N + kPiBlock - 1) / kPiBlock, h.pi_lchunks);
  popinfo_ll_kernel<<<g, kPiBlock, 0, s>>>(d_chain);
  popinfo_pick_kernel<<<(h.N + kPiBlock - 1) / kPiBlock, kPiBlock, 0, s>>>(d_chain);
  return cudaGetLastError();
}

}  // namespace st
