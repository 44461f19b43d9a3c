/*
 * ref_driver.c -- harness around the reference's own CPU code.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the reference's CPU
 * translation units straight from the reference tree (every src/*.c except
 * structure.c and Kernels.c) together with this file into
 * oracle/_ref/libstref.so.  Nothing of the reference is copied here; this file
 * only
 *   - supplies no-op bodies for the OpenCL host helpers the CPU files link
 *     against (Kernels.c is not built: there is no OpenCL here),
 *   - feeds the reference's random calls from a controlled stream: the
 *     reference files are compiled with -Drand=stref_rand and ran.c with
 *     -DRNormal=stref_ref_RNormal, so rand() and RNormal() land here,
 *   - drives the CPU update functions in the order of the sweep loop in
 *     structure.c:497-685 (the CPU twins of each *CL update).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "structure.h"
#include "Kernels.h"
#include "ran.h"
#include "mymath.h"
#include "CalcLike.h"
#include "output.h"
#include "Init.h"
#include "datain.h"
#include "Updates/UpdateZ.h"
#include "Updates/UpdateP.h"
#include "Updates/UpdateQ.h"
#include "Updates/UpdateAlpha.h"
#include "Updates/UpdateEpsilon.h"
#include "Updates/UpdateFst.h"
#include "Updates/UpdateLambda.h"
#include "Updates/UpdateLocPrior.h"
#include "Util.h"

/* ---- OpenCL host helpers (Kernels.c) as no-ops ------------------------- */
int InitCLDict(CLDict *d) { (void)d; return EXIT_SUCCESS; }
void ReleaseCLDict(CLDict *d) { (void)d; }
void handleCLErr(cl_int e, CLDict *d, char *m) { (void)e; (void)d; (void)m; }
void runKernel(CLDict *d, enum KERNEL k, int n, size_t *g, char *m)
{ (void)d; (void)k; (void)n; (void)g; (void)m; }
void runTask(CLDict *d, enum KERNEL k, char *m) { (void)d; (void)k; (void)m; }
void setKernelArg(CLDict *d, enum KERNEL k, enum BUFFER b, int a)
{ (void)d; (void)k; (void)b; (void)a; }
void setKernelArgExplicit(CLDict *d, enum KERNEL k, size_t s, void *v, int a)
{ (void)d; (void)k; (void)s; (void)v; (void)a; }
void readBuffer(CLDict *d, void *p, size_t s, enum BUFFER b, char *m)
{ (void)d; (void)p; (void)s; (void)b; (void)m; }
void writeBuffer(CLDict *d, void *p, size_t s, enum BUFFER b, char *m)
{ (void)d; (void)p; (void)s; (void)b; (void)m; }
void finishCommands(CLDict *d, char *m) { (void)d; (void)m; }

/* ---- uniform-array cursor --------------------------------------------------
 * The CPU update functions read uniforms through a cursor over randomArr
 * (randGen.c:23-36).  The reference version ends the process when one slot
 * region is over-read; UpdateQMetro's gamma draws can do that with its
 * 64-value budget per individual.  This cursor keeps reading the following
 * values of the array and counts the overrun instead.                        */
#include "randGen.h"
static long g_guard_hits = 0;
long stref_guard_hits(void) { return g_guard_hits; }
double rndDisc(RndDiscState *s)
{
    double v = s->randomArr[s->baseOffset + s->randomValsTaken];
    s->randomValsTaken += 1;
    if (s->randomValsTaken > s->maxrandom) g_guard_hits++;
    return v;
}

/* ---- controlled random streams ------------------------------------------ */
static const int32_t *g_rq = NULL;
static long g_rq_n = -1, g_rq_pos = 0, g_rq_over = 0;
static const double *g_nq = NULL;
static long g_nq_n = -1, g_nq_pos = 0, g_nq_over = 0;
static uint64_t g_xs[2] = {0x9E3779B97F4A7C15ull, 0xD1B54A32D192ED03ull};

static uint64_t xs_next(void)
{
    uint64_t s1 = g_xs[0];
    const uint64_t s0 = g_xs[1];
    g_xs[0] = s0;
    s1 ^= s1 << 23;
    g_xs[1] = s1 ^ s0 ^ (s1 >> 18) ^ (s0 >> 5);
    return g_xs[1] + s0;
}

void stref_free_seed(uint64_t seed)
{
    g_xs[0] = seed ^ 0x9E3779B97F4A7C15ull;
    g_xs[1] = (seed * 0xBF58476D1CE4E5B9ull) ^ 0x94D049BB133111EBull;
    if (!g_xs[0] && !g_xs[1]) g_xs[0] = 1;
    for (int i = 0; i < 8; i++) xs_next();
}

/* n < 0: free mode (xorshift128+, 31-bit like glibc rand()). */
void stref_rand_queue(const int32_t *vals, long n)
{
    g_rq = vals; g_rq_n = n; g_rq_pos = 0; g_rq_over = 0;
}
long stref_rand_consumed(void) { return g_rq_pos; }
long stref_rand_overrun(void) { return g_rq_over; }

int stref_rand(void)
{
    if (g_rq_n >= 0) {
        if (g_rq_pos < g_rq_n) return g_rq[g_rq_pos++];
        g_rq_over++;
        return 1 << 30;
    }
    return (int)(xs_next() >> 33);
}
void stref_srand(unsigned s) { stref_free_seed(s); }

void stref_normal_queue(const double *vals, long n)
{
    g_nq = vals; g_nq_n = n; g_nq_pos = 0; g_nq_over = 0;
}
long stref_normal_consumed(void) { return g_nq_pos; }

extern double stref_ref_RNormal(double mu, double sd);   /* ran.c:686 RNormal */
double RNormal(double mu, double sd)
{
    if (g_nq_n >= 0) {
        if (g_nq_pos < g_nq_n) return mu + sd * g_nq[g_nq_pos++];
        g_nq_over++;
        return mu;
    }
    return stref_ref_RNormal(mu, sd);
}

/* ---- globals of structure.h -------------------------------------------- */
typedef struct stref_model {
    int N, L, K, maxalleles;
    int freqscorr, onefst, inferalpha, popalphas, unifprioralpha;
    int metrofreq, burnin, numreps, computeprob, pfrompopflagonly;
    int ancestdist, numboxes;
    double alpha, alphamax, alphapropsd, alphapriora, alphapriorb;
    double lambda, fpriormean, fpriorsd;
    int inferlambda, popspecificlambda;
    int noadmix, admburnin;
    int usepopinfo, gensback, popflag;
    double migrprior;
    int locprior, updatelocprior;
    double locpriorinit, maxlocprior, locpriorstep;
    int startatpopinfo;
} stref_model;

void stref_set_globals(const stref_model *m)
{
    NUMINDS = m->N; NUMLOCI = m->L; LINES = 2; MAXPOPS = m->K;
    MAXALLELES = m->maxalleles; MISSING = -9;
    FREQSCORR = m->freqscorr; ONEFST = m->onefst; INFERALPHA = m->inferalpha;
    POPALPHAS = m->popalphas; UNIFPRIORALPHA = m->unifprioralpha;
    ALPHA = m->alpha; ALPHAMAX = m->alphamax; ALPHAPROPSD = m->alphapropsd;
    ALPHAPRIORA = m->alphapriora; ALPHAPRIORB = m->alphapriorb;
    LAMBDA = m->lambda; FPRIORMEAN = m->fpriormean; FPRIORSD = m->fpriorsd;
    METROFREQ = m->metrofreq; BURNIN = m->burnin; NUMREPS = m->numreps;
    COMPUTEPROB = m->computeprob; PFROMPOPFLAGONLY = m->pfrompopflagonly;
    ANCESTDIST = m->ancestdist; NUMBOXES = m->numboxes > 0 ? m->numboxes : 1000;
    USEPOPINFO = m->usepopinfo; NOADMIX = m->noadmix; LOCPRIOR = m->locprior; LINKAGE = 0;
    UPDATELOCPRIOR = m->updatelocprior; LOCPRIORINIT = m->locpriorinit;
    MAXLOCPRIOR = m->maxlocprior; LOCPRIORSTEP = m->locpriorstep;
    RECESSIVEALLELES = 0;
    INFERLAMBDA = m->inferlambda; POPSPECIFICLAMBDA = m->popspecificlambda;
    STARTATPOPINFO = m->startatpopinfo;
    POPDATA = (m->usepopinfo || m->startatpopinfo) ? 1 : 0; POPFLAG = m->popflag;
    MIGRPRIOR = m->migrprior;
    INTERMEDSAVE = 0; REPORTHITRATE = 0; UPDATEFREQ = 1 << 30; ADMBURNIN = m->admburnin;
    NOALPHA = 0; PHASED = 0; PHASEINFO = 0; MARKOVPHASE = 0; NOQS = 0;
    LOCDATA = m->locprior ? 1 : 0; LOCISPOP = 0; PRINTQHAT = 0; ECHODATA = 0;
    GENSBACK = m->usepopinfo ? m->gensback : 2;
}

struct IND *stref_individuals(int N, const int32_t *popflags)
{
    struct IND *ind = calloc((size_t)N, sizeof(struct IND));
    for (int i = 0; i < N; i++) ind[i].PopFlag = popflags ? popflags[i] : 0;
    return ind;
}

/* individuals with a given population (1-based) as well */
struct IND *stref_individuals_pop(int N, const int32_t *popflags, const int32_t *population)
{
    struct IND *ind = stref_individuals(N, popflags);
    for (int i = 0; i < N; i++) ind[i].Population = population ? population[i] : 0;
    return ind;
}
void stref_free(void *p) { free(p); }

/* individuals with a location (LOCDATA) as well; src/Util.c:237-275
 * GetNumLocations sets NUMLOCATIONS and each myloc */
struct IND *stref_individuals_loc(int N, const int32_t *popflags, const int32_t *population,
                                  const int32_t *location)
{
    struct IND *ind = stref_individuals_pop(N, popflags, population);
    if (location) {
        for (int i = 0; i < N; i++) ind[i].Location = location[i];
        GetNumLocations(ind);
    }
    return ind;
}
int stref_numlocations(void) { return NUMLOCATIONS; }
void stref_set_numlocations(int n) { NUMLOCATIONS = n; }

/* ---- one reference chain, driven in structure.c order ------------------ */
typedef struct stref_chain {
    stref_model m;
    int *Geno, *Z, *Z1, *NumAlleles, *Translation, *AncestDist;
    double *Q, *P, *Eps, *SumEps, *Fst, *FstSum, *Alpha, *sumAlpha;
    double *lambda, *sumlambda, *PSum, *QSum, *R, *sumR, *varR;
    double *sumIndLikes, *indLikesNorm, *randomArr, *Phase, *UsePopProbs;
    double *LocPrior, *sumLocPrior;
    int LocPriorLen, numlocations;
    double like, sumlikes, sumsqlikes;
    size_t nrand;
    struct IND *Individual;
    int rep;
} stref_chain;

static void fill_uniform(double *a, size_t n)
{
    for (size_t j = 0; j < n; j++) a[j] = (double)(xs_next() >> 33) / 2147483648.0;
}

/* geno: raw int32 [N][2][L] with -9 missing; recoded in a private copy by the
 * reference's own Initialization -> CountAlleles. */
stref_chain *stref_chain_new(const stref_model *m, const int32_t *geno,
                             const int32_t *popflags, const int32_t *population,
                             const int32_t *location, uint64_t seed)
{
    stref_chain *c = calloc(1, sizeof(stref_chain));
    int N = m->N, L = m->L, K = m->K;
    c->m = *m;
    stref_set_globals(m);
    stref_free_seed(seed);
    stref_rand_queue(NULL, -1);
    stref_normal_queue(NULL, -1);
    size_t G = (size_t)N * 2 * L;
    c->Geno = malloc(sizeof(int) * G);
    memcpy(c->Geno, geno, sizeof(int) * G);
    MAXALLELES = FindMaxAlleles(c->Geno, NULL);
    c->m.maxalleles = MAXALLELES;
    int A = MAXALLELES;
    c->Z = calloc(G, sizeof(int));
    c->Z1 = calloc(G, sizeof(int));
    c->NumAlleles = calloc((size_t)L, sizeof(int));
    c->Translation = calloc((size_t)L * A, sizeof(int));
    c->Q = calloc((size_t)N * K, sizeof(double));
    c->QSum = calloc((size_t)N * K, sizeof(double));
    c->P = calloc((size_t)L * K * A, sizeof(double));
    c->PSum = calloc((size_t)L * K * A, sizeof(double));
    c->Eps = calloc((size_t)L * A, sizeof(double));
    c->SumEps = calloc((size_t)L * A, sizeof(double));
    c->Fst = calloc((size_t)K, sizeof(double));
    c->FstSum = calloc((size_t)K, sizeof(double));
    c->Individual = stref_individuals_loc(N, popflags, population,
                                          m->locprior ? location : NULL);
    c->numlocations = m->locprior ? NUMLOCATIONS : 0;
    /* src/structure.c:354-375: LocPrior = r (admixture) or r, nu, gamma
     * (no admixture); alpha global + one row per location (admixture) */
    size_t na = (m->locprior && !m->noadmix) ? (size_t)K * (c->numlocations + 1) : (size_t)K;
    c->Alpha = calloc(na, sizeof(double));
    c->sumAlpha = calloc(na, sizeof(double));
    if (m->locprior) {
        c->LocPriorLen = m->noadmix ? 1 + K * (c->numlocations + 1) : 1;
        c->LocPrior = calloc((size_t)c->LocPriorLen, sizeof(double));
        c->sumLocPrior = calloc((size_t)c->LocPriorLen, sizeof(double));
    }
    c->lambda = calloc((size_t)K, sizeof(double));
    c->sumlambda = calloc((size_t)K, sizeof(double));
    c->R = calloc((size_t)N, sizeof(double));
    c->sumR = calloc((size_t)N + 1, sizeof(double));
    c->varR = calloc((size_t)N + 1, sizeof(double));
    c->Phase = calloc((size_t)N * L, sizeof(double));
    c->sumIndLikes = calloc((size_t)N, sizeof(double));
    c->indLikesNorm = calloc((size_t)N, sizeof(double));
    if (m->ancestdist) c->AncestDist = calloc((size_t)N * K * NUMBOXES, sizeof(int));
    if (m->usepopinfo)
        c->UsePopProbs = calloc((size_t)N * K * (GENSBACK + 1), sizeof(double));
    size_t nr = (size_t)N * L * 2;
    size_t np = (size_t)L * K * A * MAXRANDOM;
    size_t nq = (size_t)N * MAXRANDOM;
    c->nrand = nr > np ? nr : np;
    if (nq > c->nrand) c->nrand = nq;
    c->randomArr = malloc(sizeof(double) * c->nrand);
    int savefreq = 0;
    CLDict dict;
    Initialization(c->Geno, NULL, c->Individual, c->Translation, c->NumAlleles,
                   c->Z, c->Z1, c->Eps, c->SumEps, c->Fst, c->PSum, c->Q, c->QSum,
                   c->FstSum, c->AncestDist, c->UsePopProbs, c->Alpha, c->sumAlpha, c->sumR,
                   c->varR, &c->sumlikes, &c->sumsqlikes, &savefreq, c->R,
                   c->lambda, c->sumlambda, c->Phase, NULL, c->LocPrior, c->sumLocPrior,
                   c->LocPriorLen, c->sumIndLikes, c->indLikesNorm, &dict);
    c->rep = 0;
    return c;
}

/* structure.c:497-685 with the CPU twins (USEWORKINGCL=0 semantics). */
int stref_chain_sweeps(stref_chain *c, int nsweeps)
{
    stref_set_globals(&c->m);
    MAXALLELES = c->m.maxalleles;
    NUMLOCATIONS = c->numlocations;
    int N = c->m.N, L = c->m.L, K = c->m.K, A = MAXALLELES;
    for (int s = 0; s < nsweeps; s++, c->rep++) {
        int rep = c->rep;
        fill_uniform(c->randomArr, (size_t)L * K * A * MAXRANDOM);
        UpdateP(c->P, c->Eps, c->Fst, c->NumAlleles, c->Geno, c->Z, c->lambda,
                c->Individual, c->randomArr);
        if (METROFREQ > 0 && rep % METROFREQ == 0)
            fill_uniform(c->randomArr, (size_t)N * MAXRANDOM);
        UpdateQ(c->Geno, NULL, c->Q, c->P, c->Z, c->Alpha, rep, c->Individual,
                c->UsePopProbs, NULL, c->LocPrior, c->randomArr);
        if (LOCPRIOR && UPDATELOCPRIOR)     /* structure.c:535-537 */
            UpdateLocPrior(c->Q, c->LocPrior, c->Alpha, c->Individual);
        fill_uniform(c->randomArr, (size_t)N * L * 2);
        UpdateZ(c->Z, c->Q, c->P, c->Geno, c->randomArr);
        if (LOCPRIOR && NOADMIX == 0)       /* structure.c:577-590 */
            UpdateAlphaLocPrior(c->Q, c->Alpha, c->LocPrior, c->Individual);
        else if (INFERALPHA)
            UpdateAlpha(c->Q, c->Alpha, c->Individual, rep);
        if (INFERLAMBDA) {       /* structure.c:586-593 */
            if (POPSPECIFICLAMBDA) UpdatePopLambda(c->P, c->lambda, c->NumAlleles);
            else UpdateLambda(c->P, c->Eps, c->lambda, c->NumAlleles);
        }
        if (FREQSCORR) {
            UpdateEpsilon(c->P, c->Eps, c->Fst, c->NumAlleles, c->lambda[0]);
            UpdateFst(c->Eps, c->Fst, c->P, c->NumAlleles);
        }
        if (rep + 1 > BURNIN)
            DataCollection(c->Geno, NULL, c->Q, c->QSum, c->Z, c->Z1, c->P, c->PSum,
                           c->Fst, c->FstSum, c->NumAlleles, c->AncestDist, c->Alpha,
                           c->sumAlpha, c->sumR, c->varR, &c->like, &c->sumlikes,
                           &c->sumsqlikes, c->R, c->Eps, c->SumEps, 0.0, c->lambda,
                           c->sumlambda, NULL, c->LocPrior, c->sumLocPrior,
                           c->LocPriorLen, c->sumIndLikes, c->indLikesNorm, rep);
    }
    return c->rep;
}

typedef struct stref_view {
    int *Geno, *Z, *NumAlleles, *Translation, *AncestDist;
    double *Q, *P, *Eps, *SumEps, *Fst, *FstSum, *Alpha, *sumAlpha;
    double *PSum, *QSum, *like, *sumlikes, *sumsqlikes;
    int maxalleles, rep;
    double *lambda, *sumlambda, *UsePopProbs;
    double *LocPrior, *sumLocPrior;
    int LocPriorLen, numlocations;
} stref_view;

void stref_chain_view(stref_chain *c, stref_view *v)
{
    v->Geno = c->Geno; v->Z = c->Z; v->NumAlleles = c->NumAlleles;
    v->Translation = c->Translation; v->AncestDist = c->AncestDist;
    v->Q = c->Q; v->P = c->P; v->Eps = c->Eps; v->SumEps = c->SumEps;
    v->Fst = c->Fst; v->FstSum = c->FstSum; v->Alpha = c->Alpha;
    v->sumAlpha = c->sumAlpha; v->PSum = c->PSum; v->QSum = c->QSum;
    v->like = &c->like; v->sumlikes = &c->sumlikes; v->sumsqlikes = &c->sumsqlikes;
    v->maxalleles = c->m.maxalleles; v->rep = c->rep;
    v->lambda = c->lambda; v->sumlambda = c->sumlambda; v->UsePopProbs = c->UsePopProbs;
    v->LocPrior = c->LocPrior; v->sumLocPrior = c->sumLocPrior;
    v->LocPriorLen = c->LocPriorLen; v->numlocations = c->numlocations;
}

void stref_chain_free(stref_chain *c)
{
    void *ps[] = {c->Geno, c->Z, c->Z1, c->NumAlleles, c->Translation, c->AncestDist,
                  c->Q, c->P, c->Eps, c->SumEps, c->Fst, c->FstSum, c->Alpha,
                  c->sumAlpha, c->lambda, c->sumlambda, c->PSum, c->QSum, c->R,
                  c->sumR, c->varR, c->sumIndLikes, c->indLikesNorm, c->randomArr,
                  c->Phase, c->Individual, c->UsePopProbs, c->LocPrior, c->sumLocPrior};
    for (size_t j = 0; j < sizeof(ps) / sizeof(ps[0]); j++) free(ps[j]);
    free(c);
}

/* ---- thin entry points for single-function parity checks ---------------- */
double stref_LogProbQ(double *Q, double onealpha, struct IND *ind);
double stref_FlikeFreqs(double f, double *Eps, double *P, int *NumAlleles, int pop);
extern double LogProbQ(double *Q, double onealpha, struct IND *Individual);
extern double LogProbQonepop(double *Q, double alpha, double alphasum,
                             struct IND *Individual, int pop);
extern double AlphaPriorDiff(double newalpha, double oldalpha);
extern double FlikeFreqs(double f, double *Epsilon, double *P, int *NumAlleles, int pop);
extern double FPriorDiff(double newf, double oldf);
extern void GetNumFromPops(int *NumAFromPops, int *Geno, int *Z, int *NumAlleles,
                           struct IND *Individual);
extern void GetNumLociPop(int *NumLociPop, int *Z, int ind);
extern void InitializeZ(int *Geno, struct IND *Individual, int *Z);
extern void InitFreqPriors(double *Epsilon, double *Fst, int *Geno, int *NumAlleles);
extern double EstLogProb(double sumlikes, double sumsqlikes, int reps);
extern void UpdateSums(double *Q, double *QSum, int *Z, double *P, double *PSum,
                       double *Fst, double *FstSum, int *NumAlleles, int *AncestDist,
                       double *Epsilon, double *SumEpsilon, double *lambda,
                       double *sumlambda, double *LocPrior, double *sumLocPrior,
                       int LocPriorLen);

double stref_LogProbQ(double *Q, double onealpha, struct IND *ind)
{ return LogProbQ(Q, onealpha, ind); }
double stref_FlikeFreqs(double f, double *Eps, double *P, int *NumAlleles, int pop)
{ return FlikeFreqs(f, Eps, P, NumAlleles, pop); }
