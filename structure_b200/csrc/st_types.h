// st_types.h -- device-resident chain descriptor and the constants shared by
// the sweep kernels and the C-ABI layer.
#pragma once
#include <cstdint>

namespace st {

constexpr int kMaxPops = 32;          // K limit of the fused kernels
constexpr int kMaxAlleles = 64;       // per-locus allele limit (register arrays)
constexpr uint32_t kGammaMaxBlocks = 64;
constexpr int kUnassigned = -9;       // structure.h:8
constexpr uint8_t kZMissing = 0xFF;   // Z byte for a missing copy
constexpr uint8_t kG8Missing = 0xFF;  // U8 genotype byte for a missing copy

// Philox stream ids (counter word 3 = id << 24).
enum Stream : uint32_t {
  kSInitZ = 1, kSZ = 2, kSP = 3, kSQG = 4, kSQM = 5, kSQMA = 6,
  kSAlpha = 7, kSEps = 8, kSFst = 9, kSMala = 10, kSLambda = 11, kSNoAdmix = 12,
  kSPopInfo = 13, kSLocPrior = 14, kSLocAlpha = 15
};

// Device error word bits.
enum : int {
  kErrGammaCap = 0x1,    // gamma rejection loop hit its attempt cap
  kErrNaN = 0x2,         // non-finite value produced
  kErrBounds = 0x4,      // out-of-range index caught and skipped
  kErrFallThrough = 0x8  // categorical draw fell through (clamped)
};

// Genotype layouts on the device.
enum Layout : int {
  kLayoutU8 = 0,   // [N][2][L] bytes, allele code or 0xFF (reference order)
  kLayoutB2G = 1   // [L][wpr] uint32, 16 genotypes/word, 2 bits each:
                   // 0 = 0/0, 1 = 0/1, 2 = 1/1, 3 = missing
};

// Stats block (doubles) offsets.
enum : int {
  kStLike = 0, kStSumLikes = 1, kStSumSq = 2, kStNLike = 3, kStMetroHits = 4,
  kStEpsAcc = 5, kStAlphaT = 6, kStCopies = 7,
  kStAlphaS = 8,                       // K sums of log Q_ik
  kStFstDiff = kStAlphaS + kMaxPops,   // F likelihood differences
  kStFstNew = kStFstDiff + kMaxPops,   // F proposals
  kStAlphaLpd = kStFstNew + kMaxPops,  // alpha log acceptance ratios
  kStFstLpd = kStAlphaLpd + kMaxPops,  // F log acceptance ratios
  kStAlphaNew = kStFstLpd + kMaxPops,  // alpha proposals
  kStMalaAcc = kStAlphaNew + kMaxPops, // Langevin moves accepted
  kStMalaTries,                        // Langevin moves proposed
  kStLambdaLpd = kStMalaAcc + 2,       // lambda log acceptance ratios (K)
  kStSize = 256
};

// Done-counter slots of the last-CTA protocol.
enum : int { kCtrZ = 0, kCtrLocus = 1, kCtrInd = 2, kCtrMetro = 3, kCtrLambda = 4,
             kCtrCount = 8 };

struct ChainDev {
  // dimensions
  int N, L, K, A, G;        // G = power of two >= K (lanes per group)
  int layout, wpr;          // genotype layout, B2G words per locus row
  int Leff;                 // loci with at least one observed allele
  // model (mainparams / extraparams)
  int freqscorr, onefst, inferalpha, popalphas, unifprioralpha, inferlambda, popspecificlambda;
  int computeprob, pfrompopflagonly, ancestdist, numboxes, metrofreq, burnin;
  double alphamax, alphapropsd, alphapriora, alphapriorb;
  double fpriormean, fpriorsd, invsqrtnuminds;
  uint32_t key;             // seed32: low word of splitmix64(chain seed)
  int loc_tpl;              // locus kernel: lanes per locus (power of two, 1..32)
  // Z-pass tiling: T individuals per chunk, W warps, R locus blocks per CTA
  int tileT, tileW, tileR, nchunks, ngroups;
  // count histogram slices summed by the consumers (1: every producer adds
  // into slice 0); Metropolis log-ratio partials have ngroups slices
  int cnt_chunks, cnt_groups;
  // data
  const uint32_t* g2;
  const uint8_t* g8;
  const int32_t* numalleles;
  const int32_t* popflags;
  // state
  float *Q, *logQ, *TestQ, *logTestQ;   // N*K
  float *P, *logP;                      // L*K*A
  double *eps;                          // L*A
  double *F, *alpha, *lambda;           // K
  uint8_t* Z;                           // N*2*L (optional)
  int32_t* npart;                       // [K][A][L] allele counts
  int32_t* mpart;                       // [N][K] ancestry counts
  double* ldpart;                       // [groups][N]
  // accumulators
  double *QSum, *PSum, *SumEps, *FstSum, *sumAlpha, *sumlambda;
  int32_t* AncestDist;                  // N*K*numboxes
  double* stats;                        // kStSize
  double *likepart, *redpart;           // per-CTA partials
  unsigned* ctr;                        // kCtrCount
  int* rep;                             // device sweep counter
  int* err;                             // device error word
  const double* injected;               // parity uniforms (reference slots)
  // no-admixture model (NOADMIX): per-individual log likelihood of each
  // population, partial over locus chunks, then a categorical pick
  int noadmix, admburnin;
  double* napart;                       // [na_lchunks][N][K]
  int na_lchunks, na_lchunk_len;
  // USEPOPINFO: individuals flagged with a given population follow the
  // migrant model; the others the usual updates
  int usepopinfo, gensback;
  double migrprior;
  double alpha_n;                       // individuals the alpha update counts
  const int32_t* population;            // [N] given population, 1-based
  double* usepop;                       // [N][K][gensback+1] posterior sums
  double* pipart;                       // [pi_lchunks][N][K][gensback+1]
  int pi_lchunks, pi_lchunk_len;
  const int32_t* initpop;               // [N] initial Z population or -1, or null
  int noalpha;                          // USEPOPINFO with nobody unflagged: no alpha sums
  // LOCPRIOR: locations 0..nloc-1 (myloc), the reference's LocPrior array
  // locp ([0] r; no admixture: [1+k] nu, [1+K*(loc+1)+k] gamma) and, with
  // admixture, alpha rows [nloc+1][K] (global first, then per location)
  int locprior, lp_admix, updatelocprior, nloc, lp_len;
  double locpriorstep, maxlocprior;
  const int32_t* myloc;                 // [N]
  const int32_t* loc_start;             // [nloc+1] individuals of each location in
  const int32_t* loc_inds;              // [N]      loc_inds[loc_start[l] .. loc_start[l+1])
  double *locp, *sumlocp;               // [lp_len]
  // optional Langevin move on Q (Z summed out)
  int mala;
  float mala_target;
  float* mQp;                           // [N][K] proposed Q
  float *mG, *mGp;                      // [N][K] dll/dlogit at current / proposed Q
  double *mLL, *mLLp;                   // [N] ll_i at current / proposed Q
  double *mTh, *mThp;                   // [N][K] logits (last fixed at 0)
  float* mEps;                          // [N] step sizes
};

}  // namespace st
