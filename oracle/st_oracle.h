/*
 * st_oracle.h -- CPU restatement of the STRUCTURE per-sweep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the sm_100a
 * kernels in structure_b200/csrc: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it.  The product path never calls it.
 *
 * Every function restates one piece of the reference's CPU algorithm
 * (pmelsted/structure, STRUCTURE 2.3.4, src/...) with the random draws taken
 * from the same counter-based Philox4x32-10 streams the device uses, so that a
 * kernel and its restatement can be compared on identical inputs.  Each
 * function names the reference file:line it follows.
 *
 * Parity pins: the restatement is checked against the reference's own CPU
 * functions, compiled from the reference sources by oracle/Makefile into
 * oracle/_ref/libstref.so (see oracle/ref_driver.c), on shared inputs.
 */
#ifndef ST_ORACLE_H
#define ST_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_UNASSIGNED (-9)   /* structure.h:8 UNASSIGNED; also the recoded MISSING */

/* Philox stream identifiers: counter word 3 = stream << 24. */
enum {
    ORC_S_INITZ = 1, ORC_S_Z = 2, ORC_S_P = 3, ORC_S_QG = 4, ORC_S_QM = 5,
    ORC_S_QMA = 6, ORC_S_ALPHA = 7, ORC_S_EPS = 8, ORC_S_FST = 9, ORC_S_MALA = 10,
    ORC_S_LAMBDA = 11, ORC_S_NOADMIX = 12, ORC_S_POPINFO = 13, ORC_S_LOCPRIOR = 14,
    ORC_S_LOCALPHA = 15
};

/* Random123 Philox4x32-10 (Salmon et al., SC'11). */
void orc_philox(const uint32_t ctr[4], uint64_t key, uint32_t out[4]);
/* The streams of one chain: fixed key, ctr = {a, stream<<24 | b, sweep, seed32}. */
uint32_t orc_seed32(uint64_t seed);
void orc_stream(uint32_t a, uint32_t b, uint32_t rep, uint32_t stream, uint64_t seed,
                uint32_t out[4]);
double orc_u01(uint32_t hi, uint32_t lo);      /* 52-bit uniform in (0,1) */
double orc_rnd31_block(const uint32_t w[4]);  /* ran.c:152 rnd() on rand()=w>>1 */
double orc_normal(uint32_t idx, uint32_t rep, uint32_t stream, uint64_t key);

double orc_lgamma(double z);                   /* mymath.c:382 (Lanczos g=7, n=9) */
double orc_loggamma(double a, uint32_t e, uint32_t rep, uint32_t stream,
                    uint64_t key, int *err);
/* The FP32 draw of the Dirichlet of P, and its own ln and sin/cos of 2 pi u. */
float orc_loggamma_f32(float a, uint32_t e, uint32_t rep, uint32_t stream, uint64_t key,
                       int *err);
float orc_ln_f32(float x);
void orc_sincos_2pi_f32(float u, float *sn, float *cs);   /* log of a Gamma(a,1) draw */

/* --- Z (Updates/UpdateZ.c:13-56, mymath.c:105-129) --------------------- */
void orc_init_z(int N, int L, int K, const int32_t *geno, uint64_t key,
                int32_t *Z);
void orc_zupdate_f32(int N, int L, int K, int A, const int32_t *geno,
                     const float *Q, const float *P, uint64_t key, uint32_t rep,
                     int32_t *Z);
void orc_zupdate_f64_injected(int N, int L, int K, int A, const int32_t *geno,
                              const double *Q, const double *P,
                              const double *randomArr, int32_t *Z, int32_t *flags);
void orc_counts(int N, int L, int K, int A, const int32_t *geno, const int32_t *Z,
                int pfrompopflagonly, const int32_t *popflags,
                int32_t *n, int32_t *m);

/* --- P (Updates/UpdateP.c:106-199, ran.c:1248-1272) --------------------- */
void orc_update_p(int L, int K, int A, const int32_t *numalleles, const int32_t *n,
                  int freqscorr, const double *eps, const double *F,
                  const double *lambda, uint64_t key, uint32_t rep,
                  float *P, float *logP, int *err);

/* --- Q (Updates/UpdateQ.c:387-424 Gibbs, 199-307 Metro) ----------------- */
/* arow [N] (or NULL = row 0 for everyone): the row of alpha [rows][K] each
 * individual draws with (LOCPRIOR: 1 + its location, UpdateQ.c:255,409) */
void orc_update_q_gibbs(int N, int K, const int32_t *m, const double *alpha,
                        uint64_t key, uint32_t rep, float *Q, float *logQ, int *err,
                        const int32_t *arow);
void orc_metro_propose(int N, int K, const double *alpha, uint64_t key,
                       uint32_t rep, float *TestQ, float *logTestQ, int *err,
                       const int32_t *arow);
void orc_metro_logdiff(int N, int L, int K, int A, const int32_t *geno,
                       const float *Q, const float *TestQ, const float *P,
                       double *logdiff);
int  orc_metro_accept(int N, int K, const double *logdiff, uint64_t key,
                      uint32_t rep, float *Q, float *logQ, const float *TestQ,
                      const float *logTestQ, uint8_t *accepted);

/* --- alpha (Updates/UpdateAlpha.c:12-253) -------------------------------- */
typedef struct orc_alpha_params {
    int K, N, popalphas, unifprioralpha;
    double alphamax, alphapropsd, alphapriora, alphapriorb;
} orc_alpha_params;
void orc_alpha_sums(int N, int K, const float *logQ, double *S /* K */, double *T);
void orc_update_alpha(const orc_alpha_params *p, const double *S, double T,
                      double *alpha, uint64_t key, uint32_t rep, double *lpd_out);

/* --- epsilon (Updates/UpdateEpsilon.c:71-145) --------------------------- */
void orc_update_eps(int L, int K, int A, const int32_t *numalleles,
                    const float *logP, double *eps, const double *F,
                    double lambda0, double invsqrtnuminds, uint64_t key,
                    uint32_t rep, uint8_t *accepted);

/* --- F (Updates/UpdateFst.c:10-51, 142-204) ------------------------------ */
void orc_fst_diffs(int L, int K, int A, const int32_t *numalleles,
                   const float *logP, const double *eps, const double *F,
                   int onefst, double fpriorsd, uint64_t key, uint32_t rep,
                   double *newf, double *diff /* numfst */);
void orc_update_fst(int K, int onefst, double fpriormean, double fpriorsd,
                    int Leff, const double *diff, const double *newf,
                    double *F, uint64_t key, uint32_t rep, double *lpd_out);

/* --- NOADMIX Q (Updates/UpdateQ.c:310-383, mymath.c:80-100) -------------- */
/* ll_ik = sum over loci and copies of logP[l][k][allele] (FP64); pick k with
 * u*sum <= cumulative exp(ll - max), u = (w>>1)/2^31 of the Philox word at
 * (i, 0) of ORC_S_NOADMIX.  Q, logQ become one-hot (0 / -inf). */
/* LOCPRIOR (locp, myloc non-NULL): ll_ik starts at log gamma[myloc_i][k]. */
void orc_update_q_noadmix(int N, int L, int K, int A, const int32_t *geno, const float *logP,
                          uint64_t key, uint32_t rep, float *Q, float *logQ, int32_t *pick,
                          const double *locp, const int32_t *myloc);

/* --- USEPOPINFO Q (Updates/UpdateQ.c:499-706 UpdateQWithPops) ----------- */
/* For flagged individuals (popflags[i] != 0, population[i] in 1..K): the
 * migrant-model posterior over (gen, k), added to usepop [N][K][G+1] when
 * rep >= burnin, and Q/logQ from the pick (u = (w>>1)/2^31 at (i, 0) of
 * ORC_S_POPINFO).  P [L][K][A] as stored (float). */
void orc_update_q_withpops(int N, int L, int K, int A, const int32_t *geno, const float *P,
                           const int32_t *population, const int32_t *popflags, int gensback,
                           double migrprior, uint64_t key, uint32_t rep, int burnin, float *Q,
                           float *logQ, double *usepop);

/* --- lambda (Updates/UpdateLambda.c:8-102) ------------------------------- */
/* logP [L][K][A] (log P as stored), eps [L][A]; popspecific: one value per
 * population, else one shared value (from eps with freqscorr, else from P of
 * every population).  lpd_out [npop] receives the log acceptance ratios. */
void orc_update_lambda(int L, int K, int A, const int32_t *numalleles, const float *logP,
                       const double *eps, int freqscorr, int popspecific, double *lambda,
                       uint64_t key, uint32_t rep, double *lpd_out);

/* --- likelihood and bookkeeping (CalcLike.c:75-133,387-426; output.c) ---- */
double orc_calc_like(int N, int L, int K, int A, const int32_t *geno,
                     const double *Q, const double *P);
double orc_calc_like_f(int N, int L, int K, int A, const int32_t *geno,
                       const float *Q, const float *P);
void orc_init_eps(int N, int L, int A, const int32_t *geno,
                  const int32_t *numalleles, int freqscorr, double lambda,
                  double fpriormean, int K, double *eps, double *F);
double orc_est_logprob(double sumlikes, double sumsqlikes, int reps);

/* --- gradient of ln P(D|Q,P), Z marginalised, w.r.t. softmax logits --------
 * CalcLike.c:75-133 without the clamps; qlog [N][K], plog [L][K][A]; returns
 * ln P(D); dq, dp as the logits; ll_ind [N] (may be NULL). */
double orc_loglik_grad(int N, int L, int K, int A, const int32_t *geno,
                       const double *qlog, const double *plog,
                       double *dq, double *dp, double *ll_ind);

/* --- Langevin move on Q (no reference counterpart) -------------------------
 * One Metropolis-adjusted Langevin step per individual on the logits
 * theta_j = log Q_j - log Q_{K-1} (j < K-1), target ll_i + sum_k alpha_k log Q_k,
 * Z summed out, P fixed (P [L][K][2], biallelic).  Draws from the Philox
 * stream ORC_S_MALA: normals at (i, 1+j), the acceptance uniform at (i, 0).
 * Q, logQ are updated in place on acceptance; eps adapts when rep < burnin.
 * logr [N] and acc [N] receive the log acceptance ratios and decisions. */
void orc_mala_step(int N, int L, int K, const int32_t *geno, float *Q, float *logQ,
                   const float *P, const double *alpha, int popalphas, float *eps,
                   uint64_t key, uint32_t rep, int burnin, double target,
                   double *logr, uint8_t *acc);

/* --- LOCPRIOR (Updates/UpdateLocPrior.c, Updates/UpdateAlpha.c:257-305) --- */
/* The rand() words (w >> 1) and normals the reference would consume, in its
 * order, are appended to a trace when one is given (rw / nv sized by the
 * caller: 2 + 4 * (nloc + 1) words, (nloc + 1) * K normals are enough). */
typedef struct orc_trace {
    int32_t *rw;
    int32_t nr;
    double *nv;
    int32_t nn;
} orc_trace;
void orc_update_locprior(int N, int K, int nloc, int noadmix, const int32_t *myloc,
                         const float *Q, const double *alpha, double *locp,
                         double alphapropsd, double step, double maxlp, uint64_t key,
                         uint32_t rep, orc_trace *tr);
void orc_update_alpha_locprior(int N, int K, int nloc, const int32_t *myloc, const double *logQ,
                               double *alpha, double r, double alphapropsd, double alphamax,
                               uint64_t key, uint32_t rep, orc_trace *tr);

#ifdef __cplusplus
}
#endif
#endif
