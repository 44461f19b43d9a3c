// st_kernels.h -- host-side launchers of the sweep kernels.
#pragma once
#include <cuda_runtime.h>
#include "st_types.h"

namespace st {

// Chains covered by one launch: a device table of ChainDev and, per launch
// kind, the exclusive prefix of CTA counts (device array, nchains entries).
struct LaunchSet {
  ChainDev* chains;      // device pointer
  const int* prefix;     // device pointer
  int nchains;
  int total_ctas;
  cudaStream_t stream;
};

// Z-pass modes.
enum ZMode : int { kZNormal = 0, kZInit = 1, kZRecount = 2, kZMetro = 3, kZLike = 4 };
// Z-pass flags.
enum : int {
  kZfLikeIfCollect = 0x1,  // compute ln P(D) when the sweep collects
  kZfLikeAlways = 0x2,     // compute ln P(D) regardless
  kZfStoreZ = 0x4,         // write Z bytes
  kZfCollect = 0x8,        // fold ln P(D) into sumlikes/sumsqlikes when collecting
  kZfAdvance = 0x10,       // bump the device sweep counter at the end
  kZfF64 = 0x20,           // generic path: FP64 arithmetic (reference bit-parity)
  kZfInjected = 0x40,      // generic path: uniforms from the injected array
  kZfInterleave = 0x80     // fast path: the launch's chains share one data set and
                           // tile, and block b runs tile b / nchains of chain
                           // b % nchains, so the chains' CTAs over the same loci run
                           // together and read the genotype words once from DRAM
};

// Locus-kernel stages.
enum : int { kLocP = 0x1, kLocEps = 0x2, kLocFst = 0x4, kLocCollect = 0x8 };
// Individual-kernel modes and stages.
enum : int { kIndGibbs = 0, kIndPropose = 1, kIndAccept = 2, kIndNone = 3 };
enum : int { kIndAlpha = 0x1, kIndCollect = 0x2 };

size_t zpass_b2g_smem(int KT, int K, int T, int W, int mode);
// The default Z-pass tile (T individuals, W warps, R locus blocks) of a chain
// of this shape (st_api.cu choose_tile).
void default_zpass_tile(int N, int L, int K, int* T, int* W, int* R);
int zpass_b2g_width(int KT);   // CTA width (warps) of the fast path for a K class
cudaError_t launch_zpass_b2g(const LaunchSet& ls, int KT, int W, int mode, int flags,
                             size_t smem);
cudaError_t launch_zpass_u8(const LaunchSet& ls, int mode, int flags);
cudaError_t launch_locus(const LaunchSet& ls, int stages, int block);
cudaError_t launch_ind(const LaunchSet& ls, int G, int mode, int stages, int block);
cudaError_t launch_collect(const LaunchSet& ls, int block);
cudaError_t launch_lambda(const LaunchSet& ls, int block);
// NOADMIX: per-individual population log likelihoods and the one-hot pick
void noadmix_plan(int N, int L, int* lchunks, int* lchunk_len);
cudaError_t launch_noadmix(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s);
// USEPOPINFO: migrant-model Q of individuals with prior population information
void popinfo_plan(int N, int L, int* lchunks, int* lchunk_len);
cudaError_t launch_popinfo(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s);

// LOCPRIOR (st_locprior.cu): UpdateLocPrior (r, and nu / gamma without
// admixture; also adds the LocPrior sums when collecting) and
// UpdateAlphaLocPrior (global and location alphas, with their sums).
cudaError_t launch_locprior(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s);
cudaError_t launch_alpha_locprior(const ChainDev& h, const ChainDev* d_chain, cudaStream_t s);
// Injected-array parity modes (st_injected.cu): UpdateP and the proposal and
// accept steps of UpdateQMetro with the reference's own samplers.
cudaError_t launch_inj_p(const ChainDev& h, ChainDev* d_chain, const double* uni, cudaStream_t s);
cudaError_t launch_inj_metro_propose(const ChainDev& h, ChainDev* d_chain, const double* uni,
                                     int* taken, cudaStream_t s);
cudaError_t launch_inj_metro_accept(const ChainDev& h, ChainDev* d_chain, const double* uni,
                                    const int* taken, cudaStream_t s);
cudaError_t launch_pack_u8(const int32_t* geno, uint8_t* g8, size_t n, cudaStream_t s);
cudaError_t launch_clear_counts(const ChainDev* d_table, int nchains, cudaStream_t s);
cudaError_t launch_init_chain(const ChainDev& h, ChainDev* d_chain, int* d_prefix,
                              const double* eps0, int arows, float q0, float lq0, double f0,
                              double alpha0, double lambda0, cudaStream_t s);

// CTA counts per chain for each launch kind (host-side mirror of the tiling).
int ctas_zpass_b2g(const ChainDev& c);
int ctas_zpass_u8(const ChainDev& c, int block);
int ctas_locus(const ChainDev& c, int block);
int locus_lanes(int L, int K, int A);
int ctas_ind(const ChainDev& c, int block);
int ctas_collect(const ChainDev& c, int block);
int ctas_lambda(const ChainDev& c, int block);

// Gradient of ln P(D|Q,P) (Z marginalised) w.r.t. softmax logits, biallelic
// 2-bit data.  T = float or double in every T buffer.
constexpr int kGradMaxK = 16;
struct GradArgs {
  int N, L, K, wpr;
  const uint32_t* g2;
  const void* qlog;       // T [N][K]
  const void* plog;       // T [L][K][2]
  void* Q;                // T [N][K]    softmax workspace
  void* P;                // T [L][K][2] softmax workspace
  void* gqpart;           // T [lchunks][N][K]
  double* llpart;         // [lchunks][N]
  void* gppart;           // T [ichunks][L][K][2]
  void* dq;               // T [N][K]
  void* dp;               // T [L][K][2]
  double* ll_ind;         // [N] or null
  double* loglik;         // scalar or null
  double* blockpart;      // [nblocks_q]
  int lchunks, lchunk_len, ichunks, ichunk_len, nblocks_q;
  cudaStream_t stream;
};
int grad_kclass(int K);                        // 0 if K is out of range
void grad_plan(int N, int L, GradArgs* a);     // chunk sizes and counts
cudaError_t launch_loglik_grad(const GradArgs& a, bool fp64);
cudaError_t launch_grad_q(const GradArgs& a);   // ll_i and dll/dlogit(Q) only, FP32
// One Langevin move on every Q_i of a chain: cur.Q = chain Q, prop.Q = mQp.
cudaError_t launch_mala_step(const GradArgs& cur, const GradArgs& prop, const ChainDev* d_chain);

}  // namespace st
