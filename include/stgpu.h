/*
 * stgpu.h -- C ABI of the B200 STRUCTURE sweep engine (libstgpu.so).
 *
 * Drop-in boundary for the per-sweep MCMC hot path of STRUCTURE 2.3.4 as
 * shipped by pmelsted/structure.  In the reference each update is a pair of C
 * functions, a CPU twin and an OpenCL twin taking a leading CLDict*
 * (src/Updates/*.h); the device state lives in OpenCL buffers created by
 * src/Kernels.c:576-635 and is the source of truth between host reads.  This
 * header replaces that pair with one entry point per update on an opaque
 * chain handle whose state lives in HBM.
 *
 * Conventions
 *   - Every function returns an int status: ST_OK (0) or a negative ST_ERR_*.
 *     Nothing calls exit() (the reference's handleCLErr exits,
 *     src/Kernels.c:195-204).  st_last_error() gives the message.
 *   - Buffers passed in are caller-owned host memory; the library copies.
 *   - A context belongs to one host thread; chains of one context may be
 *     driven from that thread only.  There are no process globals (the
 *     reference keeps its model constants in globals, src/structure.h:70-121).
 *   - Genotypes use the reference's layout Geno[ind][line][loc]
 *     (src/structure.h:23 GenPos), alleles recoded to 0..k-1 and missing = -9
 *     as produced by CountAlleles (src/datain.c:824-904).
 */
#ifndef STGPU_H
#define STGPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define STGPU_VERSION 10000

enum st_status {
    ST_OK = 0,
    ST_ERR_ARG = -1,          /* invalid argument or size */
    ST_ERR_CUDA = -2,         /* CUDA runtime error */
    ST_ERR_NOMEM = -3,        /* allocation failed */
    ST_ERR_ADMISSION = -4,    /* would exceed the context's HBM budget */
    ST_ERR_STATE = -5,        /* operation not valid in the current state */
    ST_ERR_DEVICE = -6,       /* a kernel raised a bit in the device error word */
    ST_ERR_UNSUPPORTED = -7,  /* model option outside the implemented path */
    ST_ERR_NODEVICE = -8      /* no CUDA device / library built without one */
};

enum st_layout {
    ST_LAYOUT_AUTO = 0,       /* B2G when the data allow it, else U8 */
    ST_LAYOUT_U8 = 1,         /* one byte per allele copy, any allele count */
    ST_LAYOUT_B2G = 2         /* biallelic, 2 bits per genotype, locus-major */
};

/* Device error word bits (st_get_state ST_F_ERR). */
enum st_device_error {
    ST_DERR_GAMMA_CAP = 0x1,
    ST_DERR_NAN = 0x2,
    ST_DERR_BOUNDS = 0x4,
    ST_DERR_FALLTHROUGH = 0x8
};

typedef struct st_ctx st_ctx;
typedef struct st_data st_data;
typedef struct st_chain st_chain;
typedef struct st_batch st_batch;

/* ---- context -------------------------------------------------------------
 * Replaces InitCLDict / ReleaseCLDict (src/Kernels.c:641-751, Kernels.h:4-5).
 * hbm_budget = 0: free device memory at creation minus 2 GiB.              */
int st_version(void);
int st_ctx_create(int device, size_t hbm_budget, st_ctx **out);
int st_ctx_destroy(st_ctx *ctx);
const char *st_last_error(const st_ctx *ctx);
int st_ctx_memory(const st_ctx *ctx, size_t *in_use, size_t *budget);
/* Launch on the caller's cudaStream_t (passed as void*) instead of the
 * context's own stream; NULL restores the context stream.  The legacy default
 * stream is passed as cudaStreamLegacy ((void*)1).                          */
int st_ctx_set_stream(st_ctx *ctx, void *cuda_stream);

/* Per-kernel timing: when enabled, every launch is bracketed by CUDA events on
 * the launching stream.  st_ctx_profile_read synchronises, returns total
 * device milliseconds and launch counts per kind (ST_K_*), and clears them.
 * st_ctx_launches counts every kernel launched by the context.              */
enum st_kernel_kind { ST_K_LOCUS = 0, ST_K_IND = 1, ST_K_ZPASS = 2, ST_K_METRO = 3,
                      ST_K_OTHER = 4, ST_K_COUNT = 5 };
int st_ctx_profile(st_ctx *ctx, int enable);
int st_ctx_profile_read(st_ctx *ctx, double ms[ST_K_COUNT], int64_t launches[ST_K_COUNT]);
int64_t st_ctx_launches(const st_ctx *ctx);

/* ---- data ----------------------------------------------------------------
 * Replaces the Geno/NumAlleles/popflags uploads of src/structure.c:427-483.
 * Give either geno (reference layout, recoded) or packed (ST_LAYOUT_B2G
 * words [num_loci][ceil(num_inds/16)], 2 bits per individual: 0 = 0/0,
 * 1 = 0/1 (allele 0 on line 0), 2 = 1/1, 3 = missing).                      */
typedef struct st_data_desc {
    int32_t num_inds;          /* NUMINDS */
    int32_t num_loci;          /* NUMLOCI */
    int32_t lines;             /* LINES; must be 2 */
    int32_t layout;            /* enum st_layout */
    const int32_t *geno;       /* [num_inds][lines][num_loci] or NULL */
    const uint32_t *packed;    /* B2G words or NULL */
    const int32_t *num_alleles;/* [num_loci] NumAlleles */
    const int32_t *popflags;   /* [num_inds] Individual[].PopFlag or NULL */
    const int32_t *population; /* [num_inds] Individual[].Population (POPDATA) or NULL */
    const int32_t *location;   /* [num_inds] Individual[].Location (LOCDATA, or the
                                * population with LOCISPOP), >= 0, or NULL; locations
                                * are numbered 0.. in increasing order of these ids
                                * (src/Util.c:237-275 GetNumLocations)               */
} st_data_desc;

int st_data_upload(st_ctx *ctx, const st_data_desc *desc, st_data **out);
int st_data_destroy(st_data *data);
int st_data_layout(const st_data *data);

/* ---- model ---------------------------------------------------------------
 * The mainparams/extraparams keys the hot path reads (src/structure.h:70-121,
 * defaults of src/params.c:571-670 via st_model_defaults).                 */
typedef struct st_model {
    int32_t maxpops;           /* MAXPOPS (K), 1..32 */
    int32_t burnin, numreps;   /* BURNIN, NUMREPS */
    int32_t noadmix;           /* NOADMIX: each individual from one population */
    int32_t linkage;           /* LINKAGE: must be 0 */
    int32_t usepopinfo;        /* USEPOPINFO (needs population data) */
    int32_t locprior;          /* LOCPRIOR (needs location data; with NOADMIX, K >= 2) */
    int32_t freqscorr;         /* FREQSCORR */
    int32_t onefst;            /* ONEFST */
    int32_t inferalpha;        /* INFERALPHA */
    int32_t popalphas;         /* POPALPHAS */
    int32_t inferlambda;       /* INFERLAMBDA */
    int32_t popspecificlambda; /* POPSPECIFICLAMBDA */
    int32_t unifprioralpha;    /* UNIFPRIORALPHA */
    int32_t computeprob;       /* COMPUTEPROB */
    int32_t pfrompopflagonly;  /* PFROMPOPFLAGONLY */
    int32_t ancestdist;        /* ANCESTDIST */
    int32_t numboxes;          /* NUMBOXES */
    int32_t metrofreq;         /* METROFREQ */
    int32_t recessivealleles;  /* RECESSIVEALLELES: must be 0 */
    double alpha;              /* ALPHA (initial) */
    double alphamax;           /* ALPHAMAX */
    double alphapropsd;        /* ALPHAPROPSD */
    double alphapriora;        /* ALPHAPRIORA */
    double alphapriorb;        /* ALPHAPRIORB */
    double lambda;             /* LAMBDA */
    double fpriormean;         /* FPRIORMEAN */
    double fpriorsd;           /* FPRIORSD */
    int32_t store_z;           /* keep Z in HBM (needed for st_get_state ST_F_Z) */
    int32_t precision;         /* 0: FP32 Z/P/Q arithmetic; 1: FP64 Z (U8 data) */
    int32_t tile_t, tile_w, tile_r; /* Z-pass tile (0 = choose): individuals per chunk, warps, locus blocks per CTA */
    int32_t mala;              /* 1: a Metropolis-adjusted Langevin move on every Q_i
                                * after the Q update (Z summed out; biallelic
                                * 2-bit data, K <= 16).  No reference counterpart. */
    int32_t mala_target;       /* step-size adaptation target, acceptance x 1000
                                * (0 = 574); steps adapt during burn-in only */
    int32_t admburnin;         /* ADMBURNIN: NOADMIX chains use the admixture Q update
                                * (and update alpha) until this sweep */
    int32_t gensback;          /* GENSBACK (USEPOPINFO) */
    int32_t popflag_given;     /* 1: popflags in the data are POPFLAG values; 0: every
                                * individual with a population is flagged (POPFLAG=0) */
    int32_t updatelocprior;    /* UPDATELOCPRIOR (LOCPRIOR): 0 keeps r, nu, gamma fixed */
    int32_t startatpopinfo;    /* STARTATPOPINFO: initial Z at each individual's given
                                * population where it is in 1..K (needs population
                                * data; without it the start is random, as in
                                * src/Init.c:89-93) */
    double migrprior;          /* MIGRPRIOR (USEPOPINFO) */
    double locpriorinit;       /* LOCPRIORINIT: initial r */
    double maxlocprior;        /* MAXLOCPRIOR: upper bound of r */
    double locpriorstep;       /* LOCPRIORSTEP: half-width of the r proposal */
} st_model;

int st_model_defaults(st_model *m);

/* ---- chain ---------------------------------------------------------------
 * Creates device state and runs the reference's Initialization
 * (src/Init.c:329-444): alpha = ALPHA, lambda = LAMBDA, random Z
 * (InitializeZ, Init.c:125-169), epsilon/F (InitFreqPriors, Init.c:173-240),
 * Q = 1/K (src/structure.c:51-58), zeroed sums.  The initialization is
 * queued on the context's stream and the call returns without waiting for
 * it; an error on the device surfaces at the next call that synchronizes
 * (st_sync, st_get_state, ...).                                               */
int st_chain_create(st_ctx *ctx, st_data *data, const st_model *model,
                    uint64_t seed, st_chain **out);
int st_chain_destroy(st_chain *chain);

/* ---- per-update entry points: one per reference CL twin -------------------
 * Each reads the chain's current state and writes the updated state; random
 * draws come from Philox4x32-10 counters (seed, sweep, update, index).
 * The sweep index is ST_F_REP (st_set_state), advanced only by st_sweep.    */
int st_update_p(st_chain *c);      /* UpdatePCL      src/Updates/UpdateP.c:202-273 */
int st_update_q(st_chain *c);      /* UpdateQCL      src/Updates/UpdateQ.c:894-929 */
int st_update_z(st_chain *c);      /* UpdateZCL      src/Updates/UpdateZ.c:60-93   */
int st_update_alpha(st_chain *c);  /* UpdateAlphaCL  src/Updates/UpdateAlpha.c:307-393 */
int st_update_eps(st_chain *c);    /* UpdateEpsilonCL src/Updates/UpdateEpsilon.c:270-292 */
int st_update_fst(st_chain *c);    /* UpdateFstCL    src/Updates/UpdateFst.c:100-140 */
int st_collect(st_chain *c);       /* DataCollectionCL src/output.c:104-183         */
int st_calc_like(st_chain *c, double *like); /* CalcLike src/CalcLike.c:387-426:
                                      ln P(D|Q,P) of the current state (synchronous;
                                      no sums are touched)                          */
int st_update_lambda(st_chain *c); /* UpdateLambda / UpdatePopLambda (CPU only in the
                                      reference) src/Updates/UpdateLambda.c:8-102   */
int st_update_locprior(st_chain *c);/* UpdateLocPrior (CPU only in the reference)
                                      src/Updates/UpdateLocPrior.c:142-150; with
                                      LOCPRIOR and admixture st_update_alpha runs
                                      UpdateAlphaLocPrior (Updates/UpdateAlpha.c:257-305) */
/* One Metropolis-adjusted Langevin move on every Q_i with Z summed out and P
 * fixed (chains created with st_model.mala; st_sweep runs it after the Q
 * update).  No reference counterpart.                                        */
int st_update_q_mala(st_chain *c);
/* UpdateZ (src/Updates/UpdateZ.c:13-56) fed an explicit uniform array laid out
 * like the reference's randomArr: slot ind*L*2 + loc*2 + (draws so far at
 * that locus).  precision 64 reproduces the reference's FP64 arithmetic.
 * Needs U8 data.                                                             */
int st_update_z_injected(st_chain *c, const double *uniforms, size_t n, int precision);
/* UpdateP (src/Updates/UpdateP.c:106-199) fed an explicit uniform array laid
 * out like the reference's randomArr for it: for locus l and population k the
 * block of MAXALLELES*64 values at (l*K*MAXALLELES + k*MAXALLELES)*64, read in
 * order by the reference's own sampler (LogRDirichletDisc over RGammaDisc,
 * src/ran.c:1094-1188,1248-1272) in FP64; P from the chain's current counts
 * (ST_F_N), eps, F and lambda.  n = L*K*MAXALLELES*64.  A draw that needs more
 * than its block (the reference exits) sets ST_DERR_GAMMA_CAP.              */
int st_update_p_injected(st_chain *c, const double *uniforms, size_t n);
/* UpdateQMetro (src/Updates/UpdateQ.c:199-307) fed an explicit uniform array:
 * for individual i the block of 64 values at i*64, from which the reference's
 * RDirichletDisc (src/ran.c:1197-1210) draws TestQ from alpha and the next
 * value is the accept uniform (accept iff u < exp(logdiff)); logdiff is the
 * chain's Metropolis data pass (FP64 on ST_LAYOUT_U8 data).  n = N*64.       */
int st_update_q_metro_injected(st_chain *c, const double *uniforms, size_t n);

/* One Z update with its counts and ln P(D) that allocates no device memory.
 * No counterpart in the reference: it serves callers that own every device
 * allocation themselves (a pool allocator that forbids outside cudaMalloc, a
 * fixed device-memory budget, a path where an allocation would synchronise
 * the device) and so cannot create a chain.
 *   g2        device, B2G words [num_loci][wpr], wpr >= ceil(num_inds/16);
 *             padding individuals coded 3 (missing)
 *   Q         device, float [num_inds][maxpops]
 *   P         device, float [num_loci][maxpops][2]
 *   seed, rep the chain seed (as given to st_chain_create) and sweep index;
 *             the draws equal st_update_z's on a chain with that seed at ST_F_REP = rep
 *   n_out     device, int32 [num_loci][maxpops][2]  (ST_F_N after st_update_z)
 *   m_out     device, int32 [num_inds][maxpops]     (ST_F_M after st_update_z)
 *   like_out  device double, ln P(D|Q,P), or NULL to skip it
 *   err_out   device int32 error word (ST_DERR_* bits), or NULL
 *   scratch_bytes (host, may be NULL) receives the scratch the call needs.
 * The count partials live in one static device array of
 * ST_NOALLOC_SCRATCH_BYTES per GPU (held until exit); a call that needs more
 * returns ST_ERR_ADMISSION.  Calls are asynchronous on cuda_stream (NULL =
 * default stream) and share that array: calls that overlap on the GPU race.
 * The first call on a device looks the array up (and may load the library's
 * device code); make it before any stream capture.  The address it caches
 * belongs to the device's context: after a cudaDeviceReset the process must
 * load the library again before calling this entry point.                   */
#define ST_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int st_update_z_noalloc(int device, const uint32_t *g2, int32_t wpr, int32_t num_inds,
                        int32_t num_loci, int32_t maxpops, const float *Q, const float *P,
                        uint64_t seed, int32_t rep, int32_t *n_out, int32_t *m_out,
                        double *like_out, int32_t *err_out, void *cuda_stream,
                        size_t *scratch_bytes);

/* ---- sweeps ----------------------------------------------------------------
 * st_sweep: n sweeps in the order of src/structure.c:497-685 (P, Q, Z, alpha,
 * eps, F, DataCollection after burn-in), fused into 3-5 launches per sweep.
 * st_run: from the current sweep to BURNIN+NUMREPS.                          */
int st_sweep(st_chain *c, int nsweeps);
int st_run(st_chain *c);
int st_sync(st_chain *c);          /* wait; ST_ERR_DEVICE if the error word is set */

/* Many chains (any mix of data sets, N, L; same METROFREQ) advanced by one
 * launch per update step.                                                    */
int st_batch_create(st_ctx *ctx, st_chain **chains, int nchains, st_batch **out);
int st_batch_sweep(st_batch *b, int nsweeps);
int st_batch_destroy(st_batch *b);
/* Replay each kind of sweep (Gibbs, Metropolis) from a CUDA graph captured on
 * first use (default on).  Used only when profiling is off and the context's
 * stream is not the legacy default stream; otherwise launches are direct.
 * No reference counterpart (the reference enqueues every kernel per sweep,
 * src/structure.c:497-685).                                                  */
int st_batch_graphs(st_batch *b, int enable);
/* Z-pass tile autotuner (biallelic 2-bit path): for each K class of the
 * batch, times candidate tiles (individuals per chunk x locus blocks per CTA)
 * with `reps` Z passes each on the batch's own chains, keeps the fastest and
 * remembers it for batches of the same chain shapes created later in this
 * process (chains created with st_model.tile_t / tile_r set are left alone
 * then).  Draws and counts do not depend on the tile; the chain state is left
 * as it was.  Takes about a second on 20 chains of 2000 x 50,000.  No
 * reference counterpart.                                                     */
int st_batch_autotune(st_batch *b, int reps);

/* ---- gradient of ln P(D|Q,P) -----------------------------------------------
 * No reference counterpart (the reference evaluates the likelihood only,
 * src/CalcLike.c:75-133 CalcLikeInd).  With Z summed out,
 *   ln P(D|Q,P) = sum_i sum_l sum_copy log sum_k Q_ik P_lk,allele(copy),
 * taken without CalcLikeInd's underflow clamps, Q_i = softmax(q_logits_i)
 * over K and P_lk = softmax(p_logits_lk) over the two alleles.  Biallelic
 * 2-bit data (ST_LAYOUT_B2G), K = 1..16.  precision 32 (float buffers) or 64
 * (double buffers).  Every pointer is DEVICE memory owned by the caller:
 * q_logits, dq [N][K]; p_logits, dp [L][K][2]; loglik (double scalar) and
 * ll_ind (double [N], per individual) may be NULL.  Asynchronous on the
 * context's stream.                                                          */
typedef struct st_grad st_grad;
int st_grad_create(st_ctx *ctx, st_data *data, int maxpops, int precision, st_grad **out);
int st_grad_destroy(st_grad *g);
int st_loglik_grad(st_grad *g, const void *q_logits, const void *p_logits, void *dq, void *dp,
                   double *loglik, double *ll_ind);

/* ---- state ---------------------------------------------------------------- */
enum st_field {
    ST_F_Q = 1,        /* float [N][K] */
    ST_F_LOGQ,         /* float [N][K] */
    ST_F_TESTQ,        /* float [N][K] Metropolis proposal */
    ST_F_LOGTESTQ,     /* float [N][K] */
    ST_F_P,            /* float [L][K][A] */
    ST_F_LOGP,         /* float [L][K][A] */
    ST_F_EPS,          /* double [L][A] */
    ST_F_F,            /* double [K] */
    ST_F_ALPHA,        /* double [K]; LOCPRIOR with admixture [NUMLOCATIONS+1][K],
                        * the global row first (src/structure.h:45 AlphaPos) */
    ST_F_LAMBDA,       /* double [K] */
    ST_F_Z,            /* uint8 [N][2][L], 0xFF = missing (needs store_z) */
    ST_F_N,            /* int32 [L][K][A] allele counts from the last Z pass (get) */
    ST_F_M,            /* int32 [N][K] ancestry counts from the last Z pass (get) */
    ST_F_LOGDIFF,      /* double [N] last Metropolis log ratio (get) */
    ST_F_QSUM,         /* double [N][K] */
    ST_F_PSUM,         /* double [L][K][A] */
    ST_F_SUMEPS,       /* double [L][A] */
    ST_F_FSTSUM,       /* double [K] */
    ST_F_SUMALPHA,     /* double, as ST_F_ALPHA */
    ST_F_SUMLAMBDA,    /* double [K] */
    ST_F_ANCESTDIST,   /* int32 [N][K][NUMBOXES] */
    ST_F_STATS,        /* double [256]: like, sumlikes, sumsqlikes, ... */
    ST_F_REP,          /* int32: sweep counter */
    ST_F_ERR,          /* int32: device error word */
    ST_F_DIMS,         /* int32 [8]: N, L, K, A, layout, G, nchunks, ngroups */
    ST_F_MALA_EPS,     /* float [N]: Langevin step sizes (chains with st_model.mala) */
    ST_F_USEPOPPROBS,  /* double [N][K][GENSBACK+1]: USEPOPINFO posterior sums
                        * (the reference's UsePopProbs, from sweep BURNIN on) */
    ST_F_LOCPRIOR,     /* double: LOCPRIOR's LocPrior array, [1] = r with admixture,
                        * [1 + K*(NUMLOCATIONS+1)] = r, nu [K], gamma [NUMLOCATIONS][K]
                        * without (src/structure.c:354-365, structure.h:47) */
    ST_F_SUMLOCPRIOR,  /* double, as ST_F_LOCPRIOR: sums from sweep BURNIN on */
    ST_F_MYLOC         /* int32 [N]: each individual's location 0..NUMLOCATIONS-1 (get) */
};
int st_get_state(st_chain *c, int field, void *host, size_t bytes);
int st_set_state(st_chain *c, int field, const void *host, size_t bytes);
size_t st_field_bytes(st_chain *c, int field);

/* Checkpoint / resume; no counterpart in the reference.
 * st_chain_save writes every array of the chain, its sweep counter and its
 * random-stream key to a file; st_chain_load restores them into a chain
 * created on the same data with the same K, layout and options (seed
 * irrelevant; its Z-pass tile and NUMREPS may differ).  Draws are keyed by
 * (seed, sweep, update, element), so the loaded chain continues exactly as
 * the saved one would have.  A file of another shape, saved under other
 * st_model options, truncated or with trailing bytes returns ST_ERR_STATE
 * and leaves the chain unchanged (the file is read and checked whole before
 * any device memory is written).  Load before putting the chain in a batch:
 * a batch keeps its own copy of each chain's descriptor from
 * st_batch_create.                                                          */
int st_chain_save(st_chain *c, const char *path);
int st_chain_load(st_chain *c, const char *path);

/* Per-chain timing of the last st_sweep / st_batch_sweep call (ms). */
int st_get_timing(st_chain *c, double *ms_total);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
