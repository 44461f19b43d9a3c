// st_locprior.cu -- the LOCPRIOR model: sampling locations inform ancestry.
//
// With admixture each location has its own alpha vector, drawn around the
// global one: UpdateAlphaLocPrior (src/Updates/UpdateAlpha.c:257-305) moves
// the global alphas, then each location's alphas against Pr(Q of the
// location's individuals | alpha_loc); UpdateLocPriorAdmix
// (src/Updates/UpdateLocPrior.c:110-139) moves r, the concentration of the
// location alphas around the global ones.  Without admixture each location
// has a prior gamma over populations around nu: UpdateLocPriorNoAdmix
// (src/Updates/UpdateLocPrior.c:12-107) moves r, one pair of nu and one pair
// of gamma per location.  The Q updates read alpha_loc / gamma
// (st_update.cu, st_noadmix.cu).
//
// Arrays keep the reference's layouts: locp = LocPrior ([0] r, [1+k] nu,
// [1+K*(loc+1)+k] gamma), alpha = [global K][loc 0 K][loc 1 K]...
//
// Every proposal is a few FP64 terms per location, so the kernels are small:
// one CTA for the global moves (block-wide FP64 reductions over locations)
// and one CTA per location for the per-location moves, which sum the Q (or
// log Q) of the location's individuals through a location-sorted index and
// run the location's sequential Metropolis steps in one warp.  The uniforms
// take the reference's RandomReal / RandomInteger form on a 31-bit word of
// a Philox draw: r at (0, 0) of stream kSLocPrior, nu at (0, 1), gamma of
// location l at (l, 2); the alpha normals at (idx, 0) of kSLocAlpha with
// their acceptance word at (idx, 1), idx = k for the global alphas and
// K*(loc+1)+k for location loc.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "st_device.cuh"
#include "st_kernels.h"

namespace st {
namespace {

constexpr int kLpBlock = 256;

// ran.c:128-147: low + (rand()/2^31) * (high - low), and the integer form
__device__ __forceinline__ double rand_real(uint32_t w, double lo, double hi) {
  return lo + (double)(w >> 1) / 2147483648.0 * (hi - lo);
}
__device__ __forceinline__ int rand_int(uint32_t w, int lo, int hi) {
  return lo + (int)((double)(w >> 1) / 2147483648.0 * (hi - lo + 1));
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Block-wide FP64 sum in a fixed order (butterfly in each warp, then over
// the warp partials); every thread gets the total.
__device__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) sh[32] = t;
  }
  __syncthreads();
  return sh[32];
}

// r (both models) and nu (no admixture); sums of r and nu when collecting.
__global__ void __launch_bounds__(kLpBlock) locprior_global_kernel(const ChainDev* __restrict__ chp) {
  __shared__ double sh[33];
  const ChainDev& ch = *chp;
  const int K = ch.K, nloc = ch.nloc;
  const int rep = *ch.rep;
  const uint32_t key = ch.key;
  double* lp = ch.locp;
  const double* alpha = ch.alpha;
  if (ch.updatelocprior) {
    const U4 w = philox_s(0, 0, (uint32_t)rep, kSLocPrior, key);
    const double cur = lp[0];
    const double nw = rand_real(w.x, cur - ch.locpriorstep, cur + ch.locpriorstep);
    if (nw > 0.0 && nw < ch.maxlocprior) {
      const double d = nw - cur;
      double part = 0.0;
      if (!ch.noadmix) {
        // src/Updates/UpdateLocPrior.c:118-137
        for (int j = threadIdx.x; j < K * nloc; j += blockDim.x) {
          const int k = j / nloc, loc = j - k * nloc;
          const double ga = alpha[k], la = alpha[(size_t)K * (loc + 1) + k];
          part += ga * d * log(la) - d * la - lanczos_lgamma(ga * nw) + lanczos_lgamma(ga * cur) +
                  ga * nw * log(nw) - ga * cur * log(cur);
        }
        const double diff = block_sum(part, sh);
        if (threadIdx.x == 0 && (diff > 0.0 || rand_real(w.y, 0.0, 1.0) < exp(diff))) lp[0] = nw;
      } else {
        // src/Updates/UpdateLocPrior.c:35-51
        const double* eta = lp + 1;
        const double* gam = lp + 1 + K;
        for (int j = threadIdx.x; j < K * nloc; j += blockDim.x)
          part += d * eta[j % K] * log(gam[j]);
        const double sum = block_sum(part, sh);
        if (threadIdx.x == 0) {
          double ld = lanczos_lgamma(nw) - lanczos_lgamma(cur);
          for (int k = 0; k < K; k++)
            ld += lanczos_lgamma(cur * eta[k]) - lanczos_lgamma(nw * eta[k]);
          ld = ld * nloc + sum;
          if (ld >= 0.0 || rand_real(w.y, 0.0, 1.0) < exp(ld)) lp[0] = nw;
        }
      }
    }
    __syncthreads();
    if (ch.noadmix) {
      // nu: one pair of populations (src/Updates/UpdateLocPrior.c:53-78)
      double* eta = lp + 1;
      const double* gam = lp + 1 + K;
      const double r = lp[0];
      const U4 u = philox_s(0, 1, (uint32_t)rep, kSLocPrior, key);
      const int p1 = rand_int(u.x, 0, K - 1);
      int p2 = rand_int(u.y, 0, K - 2);
      if (p2 >= p1) p2++;
      const double dd = rand_real(u.z, 0.0, ch.alphapropsd);
      const double e1 = eta[p1] + dd, e2 = eta[p2] - dd;
      if (e1 < 1.0 && e2 > 0.0) {
        double part = 0.0;
        for (int loc = threadIdx.x; loc < nloc; loc += blockDim.x)
          part += r * ((e1 - eta[p1]) * log(gam[(size_t)loc * K + p1]) +
                       (e2 - eta[p2]) * log(gam[(size_t)loc * K + p2]));
        const double sum = block_sum(part, sh);
        if (threadIdx.x == 0) {
          const double ld = nloc * (lanczos_lgamma(r * eta[p1]) + lanczos_lgamma(r * eta[p2]) -
                                    lanczos_lgamma(r * e1) - lanczos_lgamma(r * e2)) + sum;
          if (ld >= 0.0 || rand_real(u.w, 0.0, 1.0) < exp(ld)) {
            eta[p1] = e1;
            eta[p2] = e2;
          }
        }
      }
    }
    __syncthreads();
  }
  if (rep + 1 > ch.burnin) {
    // src/output.c:654-707 UpdateSums: sumLocPrior += LocPrior
    if (threadIdx.x == 0) ch.sumlocp[0] += lp[0];
    if (ch.noadmix && threadIdx.x < K) ch.sumlocp[1 + threadIdx.x] += lp[1 + threadIdx.x];
  }
}

// gamma of one location per CTA (no admixture), src/Updates/UpdateLocPrior.c:80-103;
// dcount = sum of Q over the location's individuals.
__global__ void __launch_bounds__(kLpBlock) locprior_gamma_kernel(const ChainDev* __restrict__ chp) {
  __shared__ double sh[33];
  const ChainDev& ch = *chp;
  const int K = ch.K, loc = blockIdx.x;
  const int rep = *ch.rep;
  double* gl = ch.locp + 1 + (size_t)K * (loc + 1);
  if (ch.updatelocprior) {
    const double* eta = ch.locp + 1;
    const double r = ch.locp[0];
    const U4 u = philox_s((uint32_t)loc, 2, (uint32_t)rep, kSLocPrior, ch.key);
    const int p1 = rand_int(u.x, 0, K - 1);
    int p2 = rand_int(u.y, 0, K - 2);
    if (p2 >= p1) p2++;
    const double dd = rand_real(u.z, 0.0, ch.alphapropsd);
    const double g1 = gl[p1] + dd, g2 = gl[p2] - dd;
    if (g1 < 1.0 && g2 > 0.0) {
      double s1 = 0.0, s2 = 0.0;
      for (int j = ch.loc_start[loc] + threadIdx.x; j < ch.loc_start[loc + 1]; j += blockDim.x) {
        const size_t i = (size_t)ch.loc_inds[j];
        s1 += (double)ch.Q[i * K + p1];
        s2 += (double)ch.Q[i * K + p2];
      }
      const double dc1 = block_sum(s1, sh);
      const double dc2 = block_sum(s2, sh);
      if (threadIdx.x == 0) {
        const double l1 = log(g1) - log(gl[p1]), l2 = log(g2) - log(gl[p2]);
        const double ld = (r * eta[p1] - 1.0) * l1 + (r * eta[p2] - 1.0) * l2 + dc1 * l1 + dc2 * l2;
        if (ld >= 0.0 || rand_real(u.w, 0.0, 1.0) < exp(ld)) {
          gl[p1] = g1;
          gl[p2] = g2;
        }
      }
    }
    __syncthreads();
  }
  if (rep + 1 > ch.burnin && threadIdx.x < K)
    ch.sumlocp[1 + (size_t)K * (loc + 1) + threadIdx.x] += gl[threadIdx.x];
}

// Global alphas under LOCPRIOR (src/Updates/UpdateAlpha.c:264-281): K
// sequential Metropolis steps, each a sum over locations.
__global__ void __launch_bounds__(kLpBlock) alpha_lp_global_kernel(const ChainDev* __restrict__ chp) {
  __shared__ double sh[33];
  const ChainDev& ch = *chp;
  const int K = ch.K, nloc = ch.nloc;
  const int rep = *ch.rep;
  double* alpha = ch.alpha;
  const double r = ch.locp[0];
  for (int k = 0; k < K; k++) {
    const double old = alpha[k];
    const double nw = old + ch.alphapropsd * normal_draw((uint32_t)k, (uint32_t)rep, kSLocAlpha, ch.key);
    if (nw >= ch.alphamax || nw <= 0.0) continue;
    double part = 0.0;
    for (int loc = threadIdx.x; loc < nloc; loc += blockDim.x)
      part += (nw - old) * r * log(alpha[(size_t)K * (loc + 1) + k]) - lanczos_lgamma(nw * r) +
              lanczos_lgamma(old * r) + (nw - old) * r * log(r);
    const double diff = block_sum(part, sh);
    if (threadIdx.x == 0 &&
        (diff > 0.0 ||
         rand_real(philox_s((uint32_t)k, 1, (uint32_t)rep, kSLocAlpha, ch.key).x, 0.0, 1.0) < exp(diff)))
      alpha[k] = nw;
    __syncthreads();
  }
  if (rep + 1 > ch.burnin && threadIdx.x < K) ch.sumAlpha[threadIdx.x] += alpha[threadIdx.x];
}

// One location's alphas per CTA (src/Updates/UpdateAlpha.c:118-139,283-303):
// S_k = sum of log Q_ik over the location's n individuals (FP64), then in
// warp 0 (lane k holds alpha_loc[k]) K sequential steps against
//   log Pr(Q | a) = sum_k (a_k - 1) S_k + n (lgamma(sum_k a_k) - sum_k lgamma(a_k)).
__global__ void __launch_bounds__(kLpBlock) alpha_lp_loc_kernel(const ChainDev* __restrict__ chp) {
  __shared__ double sS[kMaxPops];
  const ChainDev& ch = *chp;
  const int K = ch.K, loc = blockIdx.x;
  const int rep = *ch.rep;
  const int j0 = ch.loc_start[loc], j1 = ch.loc_start[loc + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int k = warp; k < K; k += nwarps) {
    double v = 0.0;
    for (int j = j0 + lane; j < j1; j += 32)
      v += (double)ch.logQ[(size_t)ch.loc_inds[j] * K + k];
    v = warp_sum(v);
    if (lane == 0) sS[k] = v;
  }
  __syncthreads();
  if (warp != 0) return;
  double* al = ch.alpha + (size_t)K * (loc + 1);
  const bool on = lane < K;
  const double n = (double)(j1 - j0);
  const double S = on ? sS[lane] : 0.0;
  const double ga = on ? ch.alpha[lane] : 0.0;
  const double r = ch.locp[0];
  double a = on ? al[lane] : 0.0;
  auto logprob = [&](double av) {
    const double t = on ? (av - 1.0) * S - n * lanczos_lgamma(av) : 0.0;
    const double sa = warp_sum(on ? av : 0.0);
    return warp_sum(t) + n * lanczos_lgamma(sa);
  };
  double lp = logprob(a);
  for (int k = 0; k < K; k++) {
    const uint32_t idx = (uint32_t)(K * (loc + 1) + k);
    const double old = __shfl_sync(0xffffffffu, a, k);
    const double nw = old + ch.alphapropsd * normal_draw(idx, (uint32_t)rep, kSLocAlpha, ch.key);
    if (nw <= 0.0) continue;
    const double lpn = logprob(lane == k ? nw : a);
    const double gk = __shfl_sync(0xffffffffu, ga, k);
    const double diff = (gk * r - 1.0) * log(nw / old) - r * (nw - old) + lpn - lp;
    const bool acc = diff >= 0.0 ||
        rand_real(philox_s(idx, 1, (uint32_t)rep, kSLocAlpha, ch.key).x, 0.0, 1.0) < exp(diff);
    if (acc) {
      lp = lpn;
      if (lane == k) a = nw;
    }
  }
  if (on) {
    al[lane] = a;
    if (rep + 1 > ch.burnin) ch.sumAlpha[(size_t)K * (loc + 1) + lane] += a;
  }
}

}  // namespace

cudaError_t launch_locprior(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s) {
  locprior_global_kernel<<<1, kLpBlock, 0, s>>>(d_chain);
  if (h.noadmix) locprior_gamma_kernel<<<h.nloc, kLpBlock, 0, s>>>(d_chain);
  return cudaGetLastError();
}

cudaError_t launch_alpha_locprior(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s) {
  alpha_lp_global_kernel<<<1, kLpBlock, 0, s>>>(d_chain);
  alpha_lp_loc_kernel<<<h.nloc, kLpBlock, 0, s>>>(d_chain);
  return cudaGetLastError();
}

}  // namespace st
