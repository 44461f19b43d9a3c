// st_grad.cu -- ln P(D|Q,P) with Z marginalised, and its gradient with
// respect to the softmax logits of Q (per individual, over K) and of P (per
// locus and population, over the two alleles), on the biallelic 2-bit layout.
//
// This is the likelihood the reference evaluates per individual in
// CalcLikeInd (src/CalcLike.c:75-133), summed over individuals and taken
// without its underflow clamps:
//   ll = sum_i sum_l sum_copy log S,   S = sum_k Q_ik P_lk,a(copy)
//   g^Q_ik  = sum_l sum_copy P_lk,a / S        (dll/dQ)
//   g^P_lka = sum_i sum_copy [a(copy) = a] Q_ik / S
//   dll/dlogit = p * (g - <p, g>)               (softmax Jacobian)
// The reference has no gradient; this serves the optional Langevin move on Q.
//
// Two passes, each free of cross-lane reductions:
//   individual pass: thread = individual, walks a chunk of loci (P of a
//     32-locus stage in shared memory, genotype words staged beside it);
//     accumulates g^Q and ll in registers -> partials [lchunk][N][K].
//   locus pass: thread = locus, walks a chunk of individuals (Q rows of a
//     64-individual stage in shared memory); accumulates g^P in registers ->
//     partials [ichunk][L][K][2].
// Both recompute S (2K FMA per genotype) instead of exchanging it.  Finishing
// kernels sum the partials in a fixed order and apply the softmax Jacobian.
#include <cuda_runtime.h>

#include <algorithm>

#include <cstdint>

#include "st_device.cuh"
#include "st_kernels.h"

namespace st {
namespace {

constexpr int kGradBlock = 256;
constexpr int kLB = 32;   // loci per shared-memory stage (individual pass)
constexpr int kIB = 64;   // individuals per shared-memory stage (locus pass)

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c) { return fma(a, b, c); }

// Q = softmax(qlog) per individual (K), P = softmax(plog) per (l, k) over 2.
template <typename T>
__global__ void grad_softmax_kernel(GradArgs a) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int K = a.K;
  const T* ql = static_cast<const T*>(a.qlog);
  const T* pl = static_cast<const T*>(a.plog);
  T* Q = static_cast<T*>(a.Q);
  T* P = static_cast<T*>(a.P);
  if (t < (size_t)a.N) {
    const T* x = ql + t * K;
    T m = x[0];
    for (int k = 1; k < K; k++) m = x[k] > m ? x[k] : m;
    T s = 0;
    for (int k = 0; k < K; k++) s += exp(x[k] - m);
    for (int k = 0; k < K; k++) Q[t * K + k] = exp(x[k] - m) / s;
  }
  const size_t lk = (size_t)a.L * K;
  if (t < lk) {
    const T x0 = pl[2 * t], x1 = pl[2 * t + 1];
    const T m = x0 > x1 ? x0 : x1;
    const T e0 = exp(x0 - m), e1 = exp(x1 - m);
    P[2 * t] = e0 / (e0 + e1);
    P[2 * t + 1] = e1 / (e0 + e1);
  }
}

// FP32 uses the hardware reciprocal and logarithm (a few ulp; the gradient
// is checked to 2e-4 of its largest entry); FP64 keeps IEEE division and log.
__device__ __forceinline__ float div_t(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double div_t(double a, double b) { return a / b; }
__device__ __forceinline__ float log_t(float a) { return __logf(a); }
__device__ __forceinline__ double log_t(double a) { return log(a); }

// Weights of one genotype: copies of allele 0 / S0 and of allele 1 / S1, and
// its log-likelihood terms.  gt: 0 = 0/0, 1 = 0/1, 2 = 1/1, 3 = missing (all
// zero, so callers need no branch).
template <typename T>
__device__ __forceinline__ void genotype_terms(uint32_t gt, T s0, T s1, T& w0, T& w1, T& ll) {
  const T c0 = gt == 0u ? T(2) : (gt == 1u ? T(1) : T(0));
  const T c1 = gt == 2u ? T(2) : (gt == 1u ? T(1) : T(0));
  w0 = c0 > T(0) ? div_t(c0, s0) : T(0);
  w1 = c1 > T(0) ? div_t(c1, s1) : T(0);
  ll = (c0 > T(0) ? c0 * log_t(s0) : T(0)) + (c1 > T(0) ? c1 * log_t(s1) : T(0));
}

template <typename T, int KT>
__global__ void __launch_bounds__(kGradBlock) grad_ind_kernel(GradArgs a) {
  __shared__ T sP[kLB][KT][2];
  __shared__ uint32_t sW[kLB][kGradBlock / 16];
  const int N = a.N, L = a.L, K = a.K;
  const int i = blockIdx.x * kGradBlock + threadIdx.x;
  const bool valid = i < N;
  const T* Q = static_cast<const T*>(a.Q);
  const T* P = static_cast<const T*>(a.P);
  T q[KT], g[KT];
#pragma unroll
  for (int k = 0; k < KT; k++) {
    q[k] = (valid && k < K) ? Q[(size_t)i * K + k] : T(0);
    g[k] = T(0);
  }
  double ll = 0.0;
  const int l0 = blockIdx.y * a.lchunk_len;
  const int l1 = min(L, l0 + a.lchunk_len);
  const int wcol0 = (blockIdx.x * kGradBlock) >> 4;        // first word column of the CTA
  const int ncol = min(kGradBlock / 16, a.wpr - wcol0);
  const int sh = 2 * (i & 15), myc = (threadIdx.x >> 4);
  for (int lb = l0; lb < l1; lb += kLB) {
    const int nj = min(kLB, l1 - lb);
    __syncthreads();
    for (int idx = threadIdx.x; idx < kLB * KT * 2; idx += kGradBlock) {
      const int j = idx / (KT * 2), r = idx - j * (KT * 2), k = r >> 1, al = r & 1;
      sP[j][k][al] = (j < nj && k < K) ? P[((size_t)(lb + j) * K + k) * 2 + al] : T(0);
    }
    for (int idx = threadIdx.x; idx < kLB * (kGradBlock / 16); idx += kGradBlock) {
      const int j = idx / (kGradBlock / 16), c = idx - j * (kGradBlock / 16);
      sW[j][c] = (j < nj && c < ncol) ? __ldg(a.g2 + (size_t)(lb + j) * a.wpr + wcol0 + c)
                                      : 0xFFFFFFFFu;
    }
    __syncthreads();
    if (valid) {
      T llb = T(0);
#pragma unroll 4
      for (int j = 0; j < nj; j++) {
        const uint32_t gt = (sW[j][myc] >> sh) & 3u;
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int k = 0; k < KT; k++) {
          s0 = fma_t(q[k], sP[j][k][0], s0);
          s1 = fma_t(q[k], sP[j][k][1], s1);
        }
        T w0, w1, lt;
        genotype_terms(gt, s0, s1, w0, w1, lt);
        llb += lt;
#pragma unroll
        for (int k = 0; k < KT; k++) g[k] = fma_t(w0, sP[j][k][0], fma_t(w1, sP[j][k][1], g[k]));
      }
      ll += (double)llb;
    }
  }
  if (valid) {
    T* gq = static_cast<T*>(a.gqpart) + ((size_t)blockIdx.y * N + i) * K;
#pragma unroll
    for (int k = 0; k < KT; k++)
      if (k < K) gq[k] = g[k];
    a.llpart[(size_t)blockIdx.y * N + i] = ll;
  }
}

template <typename T, int KT>
__global__ void __launch_bounds__(kGradBlock) grad_loc_kernel(GradArgs a) {
  __shared__ T sQ[kIB][KT];
  const int N = a.N, L = a.L, K = a.K;
  const int l = blockIdx.x * kGradBlock + threadIdx.x;
  const bool valid = l < L;
  const T* Q = static_cast<const T*>(a.Q);
  const T* P = static_cast<const T*>(a.P);
  T p0[KT], p1[KT], g0[KT], g1[KT];
#pragma unroll
  for (int k = 0; k < KT; k++) {
    const bool in = valid && k < K;
    p0[k] = in ? P[((size_t)l * K + k) * 2] : T(0);
    p1[k] = in ? P[((size_t)l * K + k) * 2 + 1] : T(0);
    g0[k] = g1[k] = T(0);
  }
  const int i0 = blockIdx.y * a.ichunk_len;   // a multiple of 16
  const int i1 = min(N, i0 + a.ichunk_len);
  const uint32_t* row = a.g2 + (size_t)(valid ? l : 0) * a.wpr;
  for (int ib = i0; ib < i1; ib += kIB) {
    const int ni = min(kIB, i1 - ib);
    __syncthreads();
    for (int idx = threadIdx.x; idx < kIB * KT; idx += kGradBlock) {
      const int r = idx / KT, k = idx - r * KT;
      sQ[r][k] = (r < ni && k < K) ? Q[(size_t)(ib + r) * K + k] : T(0);
    }
    __syncthreads();
    if (!valid) continue;
    for (int wj = 0; wj < ni; wj += 16) {
      const uint32_t w = __ldg(row + ((ib + wj) >> 4));
      const int nh = min(16, ni - wj);
#pragma unroll 4
      for (int h = 0; h < nh; h++) {
        const uint32_t gt = (w >> (2 * h)) & 3u;
        const T* q = sQ[wj + h];
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int k = 0; k < KT; k++) {
          s0 = fma_t(q[k], p0[k], s0);
          s1 = fma_t(q[k], p1[k], s1);
        }
        T w0, w1, lt;
        genotype_terms(gt, s0, s1, w0, w1, lt);
#pragma unroll
        for (int k = 0; k < KT; k++) {
          g0[k] = fma_t(w0, q[k], g0[k]);
          g1[k] = fma_t(w1, q[k], g1[k]);
        }
      }
    }
  }
  if (valid) {
    T* gp = static_cast<T*>(a.gppart) + ((size_t)blockIdx.y * L + l) * K * 2;
#pragma unroll
    for (int k = 0; k < KT; k++)
      if (k < K) {
        gp[2 * k] = g0[k];
        gp[2 * k + 1] = g1[k];
      }
  }
}

// dll/dlogit of Q, per-individual ll, and one partial of the total per CTA.
template <typename T>
__global__ void __launch_bounds__(kGradBlock) grad_finish_q_kernel(GradArgs a) {
  __shared__ double sred[kGradBlock / 32];
  const int N = a.N, K = a.K;
  const int i = blockIdx.x * kGradBlock + threadIdx.x;
  double ll = 0.0;
  if (i < N) {
    const T* Q = static_cast<const T*>(a.Q) + (size_t)i * K;
    const T* gq = static_cast<const T*>(a.gqpart);
    T g[kGradMaxK];
    T s = T(0);
    for (int k = 0; k < K; k++) {
      T v = T(0);
      for (int c = 0; c < a.lchunks; c++) v += gq[((size_t)c * N + i) * K + k];
      g[k] = v;
      s = fma_t(Q[k], v, s);
    }
    T* dq = static_cast<T*>(a.dq) + (size_t)i * K;
    for (int k = 0; k < K; k++) dq[k] = Q[k] * (g[k] - s);
    for (int c = 0; c < a.lchunks; c++) ll += a.llpart[(size_t)c * N + i];
    if (a.ll_ind) a.ll_ind[i] = ll;
  }
  for (int off = 16; off > 0; off >>= 1) ll += __shfl_down_sync(0xffffffffu, ll, off);
  if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = ll;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kGradBlock / 32; w++) s += sred[w];
    a.blockpart[blockIdx.x] = s;
  }
}

template <typename T>
__global__ void __launch_bounds__(kGradBlock) grad_finish_p_kernel(GradArgs a) {
  const size_t lk = (size_t)a.L * a.K;
  const size_t t = (size_t)blockIdx.x * kGradBlock + threadIdx.x;
  if (t >= lk) return;
  const T* gp = static_cast<const T*>(a.gppart);
  T g0 = T(0), g1 = T(0);
  for (int c = 0; c < a.ichunks; c++) {
    g0 += gp[((size_t)c * lk + t) * 2];
    g1 += gp[((size_t)c * lk + t) * 2 + 1];
  }
  const T* P = static_cast<const T*>(a.P);
  const T q0 = P[2 * t], q1 = P[2 * t + 1];
  const T s = fma_t(q0, g0, q1 * g1);
  T* dp = static_cast<T*>(a.dp);
  dp[2 * t] = q0 * (g0 - s);
  dp[2 * t + 1] = q1 * (g1 - s);
}

// Total ln P(D): the per-CTA partials summed in order by one block.
__global__ void grad_total_kernel(const double* part, int n, double* out) {
  __shared__ double sred[kGradBlock / 32];
  double v = 0.0;
  for (int j = threadIdx.x; j < n; j += kGradBlock) v += part[j];
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kGradBlock / 32; w++) s += sred[w];
    *out = s;
  }
}

template <typename T, int KT>
cudaError_t launch_kt(const GradArgs& a) {
  const dim3 gi((a.N + kGradBlock - 1) / kGradBlock, a.lchunks);
  const dim3 gl((a.L + kGradBlock - 1) / kGradBlock, a.ichunks);
  grad_ind_kernel<T, KT><<<gi, kGradBlock, 0, a.stream>>>(a);
  grad_loc_kernel<T, KT><<<gl, kGradBlock, 0, a.stream>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_t(const GradArgs& a) {
  const size_t lk = (size_t)a.L * a.K;
  const size_t nsm = ((a.N > lk ? (size_t)a.N : lk) + kGradBlock - 1) / kGradBlock;
  grad_softmax_kernel<T><<<(unsigned)nsm, kGradBlock, 0, a.stream>>>(a);
  cudaError_t e = cudaSuccess;
  switch (grad_kclass(a.K)) {
    case 2: e = launch_kt<T, 2>(a); break;
    case 4: e = launch_kt<T, 4>(a); break;
    case 8: e = launch_kt<T, 8>(a); break;
    case 16: e = launch_kt<T, 16>(a); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  const unsigned nbq = (unsigned)((a.N + kGradBlock - 1) / kGradBlock);
  grad_finish_q_kernel<T><<<nbq, kGradBlock, 0, a.stream>>>(a);
  grad_finish_p_kernel<T><<<(unsigned)((lk + kGradBlock - 1) / kGradBlock), kGradBlock, 0,
                            a.stream>>>(a);
  if (a.loglik) grad_total_kernel<<<1, kGradBlock, 0, a.stream>>>(a.blockpart, (int)nbq, a.loglik);
  return cudaGetLastError();
}

template <int KT>
cudaError_t launch_q_kt(const GradArgs& a) {
  const dim3 gi((a.N + kGradBlock - 1) / kGradBlock, a.lchunks);
  grad_ind_kernel<float, KT><<<gi, kGradBlock, 0, a.stream>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Metropolis-adjusted Langevin move on Q_i, Z summed out, P fixed.
// Coordinates: theta_j = log Q_j - log Q_{K-1}, j < K-1 (the last logit is
// held at 0).  Target: ll_i(Q) + sum_k alpha_k log Q_k (the Dirichlet(alpha)
// prior times the Jacobian prod_k Q_k of the map theta -> Q).  Its gradient
// in theta_j is dll/dlogit_j + alpha_j - Q_j sum_k alpha_k.
// Proposal theta' = theta + eps^2/2 grad + eps xi, xi ~ N(0, I); accepted
// with the Metropolis-Hastings ratio of the Langevin proposal densities.
// Random draws: Philox stream kSMala, counter (i, 1 + j) for xi_j and
// (i, 0) for the acceptance uniform.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double normal_ab(uint32_t a, uint32_t b, uint32_t rep, uint32_t key) {
  const U4 w = philox_s(a, b, rep, kSMala, key);
  const double u1 = u01(w.x, w.y), u2 = u01(w.z, w.w);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

__device__ __forceinline__ double alpha_of(const ChainDev& ch, int k) {
  return ch.popalphas ? ch.alpha[k] : ch.alpha[0];
}

__global__ void __launch_bounds__(kGradBlock) mala_propose_kernel(const ChainDev* __restrict__ chp) {
  const ChainDev& ch = *chp;
  const int i = blockIdx.x * kGradBlock + threadIdx.x;
  if (i >= ch.N) return;
  const int K = ch.K;
  const uint32_t rep = (uint32_t)*ch.rep;
  double A = 0.0;
  for (int k = 0; k < K; k++) A += alpha_of(ch, k);
  const float* lq = ch.logQ + (size_t)i * K;
  const float* q = ch.Q + (size_t)i * K;
  const float* g = ch.mG + (size_t)i * K;
  double* th = ch.mTh + (size_t)i * K;
  double* thp = ch.mThp + (size_t)i * K;
  const double eps = ch.mEps[i];
  const double base = lq[K - 1];
  double m = 0.0;
  for (int j = 0; j < K - 1; j++) {
    const double t = (double)lq[j] - base;
    const double grad = (double)g[j] + alpha_of(ch, j) - (double)q[j] * A;
    const double tp = t + 0.5 * eps * eps * grad + eps * normal_ab((uint32_t)i, 1u + j, rep, ch.key);
    th[j] = t;
    thp[j] = tp;
    m = tp > m ? tp : m;
  }
  th[K - 1] = thp[K - 1] = 0.0;
  double s = 0.0;
  for (int k = 0; k < K; k++) s += exp(thp[k] - m);
  float* qp = ch.mQp + (size_t)i * K;
  for (int k = 0; k < K; k++) qp[k] = (float)(exp(thp[k] - m) / s);
}

__global__ void __launch_bounds__(kGradBlock) mala_accept_kernel(const ChainDev* __restrict__ chp) {
  const ChainDev& ch = *chp;
  const int i = blockIdx.x * kGradBlock + threadIdx.x;
  const int K = ch.K;
  int acc = 0;
  const bool valid = i < ch.N;
  if (valid) {
    const int rep = *ch.rep;
    double A = 0.0;
    for (int k = 0; k < K; k++) A += alpha_of(ch, k);
    const double* th = ch.mTh + (size_t)i * K;
    const double* thp = ch.mThp + (size_t)i * K;
    const float* q = ch.Q + (size_t)i * K;
    const float* qp = ch.mQp + (size_t)i * K;
    const float* g = ch.mG + (size_t)i * K;
    const float* gp = ch.mGp + (size_t)i * K;
    double m0 = 0.0, m1 = 0.0;
    for (int k = 0; k < K; k++) {
      m0 = th[k] > m0 ? th[k] : m0;
      m1 = thp[k] > m1 ? thp[k] : m1;
    }
    double s0 = 0.0, s1 = 0.0;
    for (int k = 0; k < K; k++) {
      s0 += exp(th[k] - m0);
      s1 += exp(thp[k] - m1);
    }
    const double lse0 = m0 + log(s0), lse1 = m1 + log(s1);
    double lp0 = ch.mLL[i], lp1 = ch.mLLp[i];
    for (int k = 0; k < K; k++) {
      lp0 += alpha_of(ch, k) * (th[k] - lse0);
      lp1 += alpha_of(ch, k) * (thp[k] - lse1);
    }
    const double eps = ch.mEps[i], h = 0.5 * eps * eps;
    double fwd = 0.0, bwd = 0.0;
    for (int j = 0; j < K - 1; j++) {
      const double g0 = (double)g[j] + alpha_of(ch, j) - (double)q[j] * A;
      const double g1 = (double)gp[j] + alpha_of(ch, j) - (double)qp[j] * A;
      const double df = thp[j] - th[j] - h * g0;
      const double db = th[j] - thp[j] - h * g1;
      fwd += df * df;
      bwd += db * db;
    }
    const double logr = lp1 - lp0 - (bwd - fwd) / (2.0 * eps * eps);
    const U4 w = philox_s((uint32_t)i, 0u, (uint32_t)rep, kSMala, ch.key);
    acc = log(u01(w.x, w.y)) < logr ? 1 : 0;
    if (acc) {
      float* qd = ch.Q + (size_t)i * K;
      float* lqd = ch.logQ + (size_t)i * K;
      for (int k = 0; k < K; k++) {
        qd[k] = qp[k];
        lqd[k] = (float)(thp[k] - lse1);
      }
    }
    if (rep < ch.burnin) {
      // Robbins-Monro adaptation toward the target acceptance (burn-in only)
      const double pa = logr >= 0.0 ? 1.0 : (logr == logr ? exp(logr) : 0.0);
      double e = eps * exp(pow((double)rep + 1.0, -0.6) * (pa - (double)ch.mala_target));
      e = e < 1e-6 ? 1e-6 : (e > 10.0 ? 10.0 : e);
      ch.mEps[i] = (float)e;
    }
  }
  // acceptance count: one atomic per warp
  const unsigned bal = __ballot_sync(0xffffffffu, acc);
  const unsigned tries = __ballot_sync(0xffffffffu, valid);
  if ((threadIdx.x & 31) == 0 && tries) {
    atomicAdd(&ch.stats[kStMalaAcc], (double)__popc(bal));
    atomicAdd(&ch.stats[kStMalaTries], (double)__popc(tries));
  }
}

}  // namespace

cudaError_t launch_mala_step(const GradArgs& cur, const GradArgs& prop, const ChainDev* d_chain) {
  const unsigned nb = (unsigned)((cur.N + kGradBlock - 1) / kGradBlock);
  cudaError_t e = launch_grad_q(cur);
  if (e != cudaSuccess) return e;
  mala_propose_kernel<<<nb, kGradBlock, 0, cur.stream>>>(d_chain);
  e = launch_grad_q(prop);
  if (e != cudaSuccess) return e;
  mala_accept_kernel<<<nb, kGradBlock, 0, cur.stream>>>(d_chain);
  return cudaGetLastError();
}

// ll_i and dll/dlogit of Q only (FP32; P given directly, no softmax of P).
cudaError_t launch_grad_q(const GradArgs& a) {
  cudaError_t e = cudaSuccess;
  switch (grad_kclass(a.K)) {
    case 2: e = launch_q_kt<2>(a); break;
    case 4: e = launch_q_kt<4>(a); break;
    case 8: e = launch_q_kt<8>(a); break;
    case 16: e = launch_q_kt<16>(a); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  grad_finish_q_kernel<float><<<(unsigned)((a.N + kGradBlock - 1) / kGradBlock), kGradBlock, 0,
                                a.stream>>>(a);
  return cudaGetLastError();
}

int grad_kclass(int K) {
  if (K < 1 || K > kGradMaxK) return 0;
  return K <= 2 ? 2 : K <= 4 ? 4 : K <= 8 ? 8 : 16;
}

// Chunks per pass: the smallest count c (1..cmax) whose grid takes at most
// 5 % more waves per unit of work, ceil(tiles * c / wave) / c, than perfect
// packing (tiles / wave), else the count with the fewest.  A grid just above
// a whole number of waves (600 CTAs on 592 slots) would run a nearly empty
// last wave as long as a full one; few chunks keep the partials small.
int wave_chunks(int tiles, int wave, int cmax) {
  const double ideal = (double)tiles / wave;
  int best = 1;
  double best_t = 1e300;
  for (int c = 1; c <= cmax; c++) {
    const double t = (double)((tiles * (long long)c + wave - 1) / wave) / c;
    if (t <= 1.05 * ideal) return c;
    if (t < best_t) {
      best_t = t;
      best = c;
    }
  }
  return best;
}

// Chunking: each pass's grid sized against one wave of 4 CTAs per SM on 148
// SMs (64 registers x 256 threads per CTA), chunks of at least 64 loci or
// individuals so the partials stay small.
void grad_plan(int N, int L, GradArgs* a) {
  const int tiles_i = (N + kGradBlock - 1) / kGradBlock;
  const int tiles_l = (L + kGradBlock - 1) / kGradBlock;
  const int wave = 148 * 4;
  const int lch = wave_chunks(tiles_i, wave, std::max(1, std::min(64, L / 64)));
  const int llen = std::max(64, (L + lch - 1) / lch);
  a->lchunk_len = llen;
  a->lchunks = (L + llen - 1) / llen;
  const int ich = wave_chunks(tiles_l, wave, std::max(1, std::min(64, N / 64)));
  int ilen = (N + ich - 1) / ich;
  ilen = ((ilen + 15) / 16) * 16;
  if (ilen < 64) ilen = 64;
  a->ichunk_len = ilen;
  a->ichunks = (N + ilen - 1) / ilen;
  a->nblocks_q = tiles_i;
}

cudaError_t launch_loglik_grad(const GradArgs& a, bool fp64) {
  return fp64 ? launch_t<double>(a) : launch_t<float>(a);
}

}  // namespace st
