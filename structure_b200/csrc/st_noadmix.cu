// st_noadmix.cu -- the no-admixture Q update (NOADMIX=1): every individual
// comes from one population (src/Updates/UpdateQ.c:310-383 UpdateQNoAdmix).
//
// For individual i and population k the log likelihood of all its allele
// copies, ll_ik = sum_l sum_copy log P[l][k][allele], is accumulated in FP64
// from the stored log P.  (The reference keeps a running product rescaled
// below 1e-100; the two agree to rounding.)  Thread = individual, CTAs split
// the loci into chunks whose partial sums go to napart[chunk][i][k]; the
// pick kernel adds the chunks in order, forms exp(ll_ik - max_k ll_ik) and
// picks population k with the reference's PickAnOption rule (the first k
// with u * sum <= cumulative sum, src/mymath.c:80-100), u = rand()/2^31 from
// the Philox word at (i, 0) of stream kSNoAdmix.  Q_i becomes one-hot.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "st_device.cuh"
#include "st_kernels.h"

namespace st {
namespace {

constexpr int kNaBlock = 256;

template <int KC>
__global__ void __launch_bounds__(kNaBlock) noadmix_ll_kernel(const ChainDev* __restrict__ chp) {
  const ChainDev& ch = *chp;
  const int N = ch.N, L = ch.L, K = ch.K, A = ch.A;
  const int i = blockIdx.x * kNaBlock + threadIdx.x;
  if (i >= N || (ch.usepopinfo && ch.popflags[i])) return;   // flagged: migrant model
  double ll[KC];
#pragma unroll
  for (int k = 0; k < KC; k++) ll[k] = 0.0;
  const int l0 = blockIdx.y * ch.na_lchunk_len;
  const int l1 = min(L, l0 + ch.na_lchunk_len);
  for (int l = l0; l < l1; l++) {
    int a0, a1;
    if (ch.layout == kLayoutB2G) {
      const uint32_t g = (__ldg(ch.g2 + (size_t)l * ch.wpr + (i >> 4)) >> (2 * (i & 15))) & 3u;
      if (g == 3u) continue;
      a0 = (int)(g >> 1);
      a1 = (int)((g | (g >> 1)) & 1u);
    } else {
      const uint8_t b0 = __ldg(ch.g8 + ((size_t)i * 2) * L + l);
      const uint8_t b1 = __ldg(ch.g8 + ((size_t)i * 2 + 1) * L + l);
      a0 = b0 == kG8Missing ? -1 : b0;
      a1 = b1 == kG8Missing ? -1 : b1;
    }
    const float* lp = ch.logP + (size_t)l * K * A;
#pragma unroll
    for (int k = 0; k < KC; k++) {
      if (k >= K) break;
      double v = 0.0;
      if (a0 >= 0) v += (double)__ldg(lp + k * A + a0);
      if (a1 >= 0) v += (double)__ldg(lp + k * A + a1);
      ll[k] += v;
    }
  }
  double* out = ch.napart + ((size_t)blockIdx.y * N + i) * K;
#pragma unroll
  for (int k = 0; k < KC; k++)
    if (k < K) out[k] = ll[k];
}

__global__ void __launch_bounds__(kNaBlock) noadmix_pick_kernel(const ChainDev* __restrict__ chp) {
  const ChainDev& ch = *chp;
  const int N = ch.N, K = ch.K;
  const int i = blockIdx.x * kNaBlock + threadIdx.x;
  if (i >= N || (ch.usepopinfo && ch.popflags[i])) return;
  double p[kMaxPops];
  double mx = 0.0;
  // LOCPRIOR: the product starts at gamma of the individual's location
  // (src/Updates/UpdateQ.c:339-345)
  const double* gam = ch.locprior ? ch.locp + 1 + (size_t)K * (ch.myloc[i] + 1) : nullptr;
  for (int k = 0; k < K; k++) {
    double s = gam ? log(gam[k]) : 0.0;
    for (int c = 0; c < ch.na_lchunks; c++) s += ch.napart[((size_t)c * N + i) * K + k];
    p[k] = s;
    if (k == 0 || s > mx) mx = s;
  }
  double sum = 0.0;
  for (int k = 0; k < K; k++) sum += (p[k] = exp(p[k] - mx));
  const U4 w = philox_s((uint32_t)i, 0u, (uint32_t)*ch.rep, kSNoAdmix, ch.key);
  const double r = (double)(w.x >> 1) / 2147483648.0 * sum;
  double cum = 0.0;
  int pick = K - 1;
  for (int k = 0; k < K; k++) {
    cum += p[k];
    if (r <= cum) {
      pick = k;
      break;
    }
  }
  for (int k = 0; k < K; k++) {
    ch.Q[(size_t)i * K + k] = k == pick ? 1.0f : 0.0f;
    ch.logQ[(size_t)i * K + k] = k == pick ? 0.0f : -INFINITY;
  }
}

}  // namespace

void noadmix_plan(int N, int L, int* lchunks, int* lchunk_len) {
  const int tiles = (N + kNaBlock - 1) / kNaBlock;
  int ch = (148 * 4 + tiles - 1) / tiles;
  if (ch < 1) ch = 1;
  int len = (L + ch - 1) / ch;
  if (len < 64) len = 64;
  *lchunk_len = len;
  *lchunks = (L + len - 1) / len;
}

cudaError_t launch_noadmix(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s) {
  const dim3 g((h.N + kNaBlock - 1) / kNaBlock, h.na_lchunks);
  if (h.K <= 8) noadmix_ll_kernel<8><<<g, kNaBlock, 0, s>>>(d_chain);
  else if (h.K <= 16) noadmix_ll_kernel<16><<<g, kNaBlock, 0, s>>>(d_chain);
  else noadmix_ll_kernel<32><<<g, kNaBlock, 0, s>>>(d_chain);
  noadmix_pick_kernel<<<(h.N + kNaBlock - 1) / kNaBlock, kNaBlock, 0, s>>>(d_chain);
  return cudaGetLastError();
}

}  // namespace st
