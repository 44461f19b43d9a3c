/*
 * st_oracle.c -- CPU restatement of the STRUCTURE per-sweep hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): loaded by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg.  Built with
 * -ffp-contract=off so that every a*b+c is two roundings unless written as
 * fma()/fmaf(), exactly like the device code built with -fmad=false.
 *
 * Reference = pmelsted/structure (STRUCTURE 2.3.4 CPU code under src/).
 * Random draws come from Philox4x32-10 counters (the device convention):
 *   fixed key, ctr = {index, (stream << 24) | sub-index, sweep, seed32}.
 */
#include "st_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LOG_UNDERFLO_D   (-230.25850929940458)   /* log(1e-100): ran.c:1262 patch */
#define SQRT_UNDERFLO    1e-50                   /* sqrt(UNDERFLO), CalcLike.c:107 */
#define TWO_PI           6.283185307179586
#define GAMMA_MAX_BLOCKS 64
#define ERR_GAMMA_CAP    0x8

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                            */
/* ------------------------------------------------------------------------ */
void orc_philox(const uint32_t ctr[4], uint64_t key, uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Stream layout shared with the device: a fixed Philox key, and the counter
 *   {a, (stream << 24) | (b & 0xFFFFFF), sweep, seed32},
 * seed32 = low word of splitmix64(chain seed) (Steele, Lea & Flood 2014). */
#define ORC_KEY0 0xA511E9B3u
#define ORC_KEY1 0x3C6EF372u

uint32_t orc_seed32(uint64_t seed)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)z;
}

void orc_stream(uint32_t a, uint32_t b, uint32_t rep, uint32_t stream, uint64_t seed,
                uint32_t out[4])
{
    uint32_t c[4] = {a, (stream << 24) | (b & 0xFFFFFFu), rep, orc_seed32(seed)};
    orc_philox(c, ((uint64_t)ORC_KEY1 << 32) | ORC_KEY0, out);
}

static void philox4(uint32_t a, uint32_t b, uint32_t rep, uint32_t stream,
                    uint64_t key, uint32_t out[4])
{
    orc_stream(a, b, rep, stream, key, out);
}

double orc_u01(uint32_t hi, uint32_t lo)
{
    uint64_t x = ((uint64_t)(hi >> 6) << 26) | (uint64_t)(lo >> 6);   /* 52 bits */
    return ((double)x + 0.5) * (1.0 / 4503599627370496.0);
}

/* ran.c:128-161: RandomReal/rnd on rand() in [0, 2^31); rnd() redraws on 0. */
double orc_rnd31_block(const uint32_t w[4])
{
    for (int j = 0; j < 4; j++) {
        uint32_t v = w[j] >> 1;
        if (v != 0) return (double)v / 2147483648.0;
    }
    return 1.0 / 4294967296.0;
}

double orc_normal(uint32_t idx, uint32_t rep, uint32_t stream, uint64_t key)
{
    uint32_t w[4];
    philox4(idx, 0, rep, stream, key, w);
    double u1 = orc_u01(w[0], w[1]);
    double u2 = orc_u01(w[2], w[3]);
    return sqrt(-2.0 * log(u1)) * cos(TWO_PI * u2);
}

/* ------------------------------------------------------------------------ */
/* ln Gamma: Lanczos (1964) g=7, n=9 series with the coefficient set used    */
/* by mymath.c:382-429 (A. Miller 1988); same summation order.               */
/* ------------------------------------------------------------------------ */
double orc_lgamma(double z)
{
    static const double c[9] = {
        0.9999999999995183, 676.5203681218835, -1259.139216722289,
        771.3234287757674, -176.6150291498386, 12.50734324009056,
        -0.1385710331296526, 9.934937113930748e-6, 1.659470187408462e-7};
    double s = 0.0;
    double t = z + 7.0;
    for (int j = 8; j >= 1; j--) {
        s += c[j] / t;
        t -= 1.0;
    }
    s += c[0];
    return log(s) + 0.9189385332046727 - (z + 6.5) + (z - 0.5) * log(z + 6.5);
}

/* ------------------------------------------------------------------------ */
/* Marsaglia & Tsang (2000) gamma, returned as log(draw).                    */
/* Attempts come in pairs: block 2j gives two Box-Muller normals, block      */
/* 2j+1 the two acceptance uniforms.  Shape < 1 uses G(a) = G(a+1) U^(1/a)   */
/* with U from block 0xFFFFFF.                                               */
/* ------------------------------------------------------------------------ */
double orc_loggamma(double a, uint32_t e, uint32_t rep, uint32_t stream,
                    uint64_t key, int *err)
{
    double aa = a < 1.0 ? a + 1.0 : a;
    double d = aa - 1.0 / 3.0;
    double c = 1.0 / sqrt(9.0 * d);
    double lg = 0.0;
    int done = 0;
    for (uint32_t j = 0; j < GAMMA_MAX_BLOCKS && !done; j += 2) {
        uint32_t b0[4], b1[4];
        philox4(e, j, rep, stream, key, b0);
        philox4(e, j + 1, rep, stream, key, b1);
        double u1 = orc_u01(b0[0], b0[1]);
        double u2 = orc_u01(b0[2], b0[3]);
        double rad = sqrt(-2.0 * log(u1));
        double ang = TWO_PI * u2;
        double xs[2] = {rad * cos(ang), rad * sin(ang)};
        double vs[2] = {orc_u01(b1[0], b1[1]), orc_u01(b1[2], b1[3])};
        for (int h = 0; h < 2; h++) {
            double x = xs[h];
            double t = 1.0 + c * x;
            if (t <= 0.0) continue;
            double v = t * t * t;
            double x2 = x * x;
            double u = vs[h];
            if (u < 1.0 - 0.0331 * x2 * x2 ||
                log(u) < 0.5 * x2 + d * (1.0 - v + log(v))) {
                lg = log(d * v);
                done = 1;
                break;
            }
        }
    }
    if (!done) {
        if (err) *err |= ERR_GAMMA_CAP;
        lg = log(d);
    }
    if (a < 1.0) {
        uint32_t w[4];
        philox4(e, 0xFFFFFFu, rep, stream, key, w);
        lg += log(orc_u01(w[0], w[1])) / a;
    }
    return lg;
}

/* ------------------------------------------------------------------------ */
/* FP32 gamma draw for the Dirichlet of P: the device's log_gamma_draw_f32,  */
/* operation for operation (IEEE float add, multiply, fmaf, divide, sqrtf;  */
/* no contraction), so both give the same bits.  ln and sin/cos are series: */
/* ln m = 2 atanh((m-1)/(m+1)) for m in [sqrt(1/2), sqrt(2)) plus e ln 2 in  */
/* a Cody-Waite head and tail; sin and cos of theta in [-pi/4, pi/4] by      */
/* Taylor series to theta^9 / theta^10 after the quadrant reduction of 4u.  */
/* Marsaglia & Tsang (2000) with v - 1 = y (3 + y (3 + y)), y = c x, and     */
/* 1 - v + ln v = ln(1 + w) - w summed as a series when |w| < 1/8.          */
/* ------------------------------------------------------------------------ */
static float u23c_f32(uint32_t w)
{
    return (float)(((w >> 9) << 1) | 1u) * 5.9604644775390625e-8f;
}

static float ln_f32(float x)
{
    uint32_t b;
    memcpy(&b, &x, 4);
    int e = (int)((b >> 23) & 0xFFu) - 127;
    uint32_t mb = (b & 0x7FFFFFu) | 0x3F800000u;
    float m;
    memcpy(&m, &mb, 4);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    float sv = (m - 1.0f) / (m + 1.0f);
    float z = sv * sv;
    float q = fmaf(z, 1.0f / 11.0f, 1.0f / 9.0f);
    q = fmaf(z, q, 1.0f / 7.0f);
    q = fmaf(z, q, 1.0f / 5.0f);
    q = fmaf(z, q, 1.0f / 3.0f);
    float t = 2.0f * sv;
    float lm = fmaf(t * z, q, t);
    float fe = (float)e;
    return fe * 0.693145751953125f + fmaf(fe, 1.42860682e-6f, lm);
}

static void sincos_2pi_f32(float u, float *sn, float *cs)
{
    float q = u * 4.0f;
    int n = (int)(q + 0.5f);
    float r = q - (float)n;
    float th = r * 1.57079637f;
    float t2 = th * th;
    float ps = fmaf(t2, 1.0f / 362880.0f, -1.0f / 5040.0f);
    ps = fmaf(t2, ps, 1.0f / 120.0f);
    ps = fmaf(t2, ps, -1.0f / 6.0f);
    float sv = fmaf(th * t2, ps, th);
    float pc = fmaf(t2, -1.0f / 3628800.0f, 1.0f / 40320.0f);
    pc = fmaf(t2, pc, -1.0f / 720.0f);
    pc = fmaf(t2, pc, 1.0f / 24.0f);
    pc = fmaf(t2, pc, -0.5f);
    float cv = fmaf(t2, pc, 1.0f);
    switch (n & 3) {
    case 0: *sn = sv; *cs = cv; break;
    case 1: *sn = cv; *cs = -sv; break;
    case 2: *sn = -sv; *cs = -cv; break;
    default: *sn = -cv; *cs = sv; break;
    }
}

float orc_loggamma_f32(float a, uint32_t e, uint32_t rep, uint32_t stream, uint64_t key,
                       int *err)
{
    float aa = a < 1.0f ? a + 1.0f : a;
    float d = aa - 1.0f / 3.0f;
    float c = 1.0f / sqrtf(9.0f * d);
    float lg = 0.0f;
    int done = 0;
    for (uint32_t j = 0; j < GAMMA_MAX_BLOCKS && !done; j++) {
        uint32_t b[4];
        philox4(e, j, rep, stream, key, b);
        float sn, cs;
        sincos_2pi_f32(u23c_f32(b[1]), &sn, &cs);
        float rad = sqrtf(-2.0f * ln_f32(u23c_f32(b[0])));
        float xs[2] = {rad * cs, rad * sn};
        float us[2] = {u23c_f32(b[2]), u23c_f32(b[3])};
        for (int h = 0; h < 2 && !done; h++) {
            float x = xs[h];
            float y = c * x;
            if (!(1.0f + y > 0.0f)) continue;
            float w = y * fmaf(y, 3.0f + y, 3.0f);
            float v = 1.0f + w;
            if (!(v > 1e-30f)) continue;
            float x2 = x * x;
            float u = us[h];
            int acc = u < 1.0f - (0.0331f * x2) * x2;
            if (!acc) {
                float g;
                if (fabsf(w) < 0.125f) {
                    float p = fmaf(w, 1.0f / 9.0f, -0.125f);
                    p = fmaf(w, p, 1.0f / 7.0f);
                    p = fmaf(w, p, -1.0f / 6.0f);
                    p = fmaf(w, p, 0.2f);
                    p = fmaf(w, p, -0.25f);
                    p = fmaf(w, p, 1.0f / 3.0f);
                    p = fmaf(w, p, -0.5f);
                    g = (w * w) * p;
                } else {
                    g = ln_f32(v) - w;
                }
                acc = ln_f32(u) < fmaf(d, g, 0.5f * x2);
            }
            if (acc) {
                lg = ln_f32(d * v);
                done = 1;
            }
        }
    }
    if (!done) {
        if (err) *err |= ERR_GAMMA_CAP;
        lg = ln_f32(d);
    }
    if (a < 1.0f) {
        uint32_t w[4];
        philox4(e, 0xFFFFFFu, rep, stream, key, w);
        lg = lg + ln_f32(u23c_f32(w[0])) / a;
    }
    return lg;
}

float orc_ln_f32(float x) { return ln_f32(x); }

void orc_sincos_2pi_f32(float u, float *sn, float *cs) { sincos_2pi_f32(u, sn, cs); }

/* Pairwise tree over G (power of two) slots, the order of a xor-butterfly. */
static double tree_sum(double *v, int G)
{
    for (int off = 1; off < G; off <<= 1)
        for (int j = 0; j < G; j += 2 * off) v[j] = v[j] + v[j + off];
    return v[0];
}

static int pow2_at_least(int k)
{
    int g = 1;
    while (g < k) g <<= 1;
    return g;
}

/* ------------------------------------------------------------------------ */
/* Z                                                                        */
/* ------------------------------------------------------------------------ */
/* Init.c:125-169 InitializeZ: RandomInteger(0,K-1) = (int)(d*K), d = rand()/2^31 */
void orc_init_z(int N, int L, int K, const int32_t *geno, uint64_t key, int32_t *Z)
{
    for (int i = 0; i < N; i++)
        for (int l = 0; l < L; l++) {
            uint32_t w[4];
            philox4((uint32_t)l, (uint32_t)(i >> 1), 0, ORC_S_INITZ, key, w);
            for (int line = 0; line < 2; line++) {
                size_t pos = ((size_t)i * 2 + line) * L + l;
                if (geno[pos] < 0) {
                    Z[pos] = ORC_UNASSIGNED;
                } else {
                    uint64_t v = w[2 * (i & 1) + line] >> 1;
                    Z[pos] = (int32_t)((v * (uint64_t)K) >> 31);
                }
            }
        }
}

/* Updates/UpdateZ.c:13-56 + mymath.c:105-129 in FP32: cumsum by fmaf,
 * r = u*sum, z = first k with r <= cumsum_k  (= #{k<K-1 : cumsum_k < r}). */
void orc_zupdate_f32(int N, int L, int K, int A, const int32_t *geno,
                     const float *Q, const float *P, uint64_t key, uint32_t rep,
                     int32_t *Z)
{
    float C[64];
    for (int i = 0; i < N; i++) {
        const float *q = Q + (size_t)i * K;
        for (int l = 0; l < L; l++) {
            uint32_t w[4];
            philox4((uint32_t)l, (uint32_t)(i >> 1), rep, ORC_S_Z, key, w);
            for (int line = 0; line < 2; line++) {
                size_t pos = ((size_t)i * 2 + line) * L + l;
                int a = geno[pos];
                if (a < 0) { Z[pos] = ORC_UNASSIGNED; continue; }
                const float *p = P + (size_t)l * K * A + a;
                C[0] = q[0] * p[0];
                for (int k = 1; k < K; k++) C[k] = fmaf(q[k], p[(size_t)k * A], C[k - 1]);
                /* u = the word's low 23 bits / 2^23; r = RN(u * T) */
                float u = (float)(w[2 * (i & 1) + line] & 0x7FFFFFu) * (1.0f / 8388608.0f);
                float r = u * C[K - 1];
                int z = 0;
                for (int k = 0; k < K - 1; k++) z += (C[k] < r);
                Z[pos] = z;
            }
        }
    }
}

/* The reference's UpdateZ arithmetic verbatim in FP64 (no contraction),
 * reading uniforms from randomArr at slot i*L*2 + l*2 + (#draws so far).
 * flags bit 0: a fall-through (option == K) was clamped to K-1. */
void orc_zupdate_f64_injected(int N, int L, int K, int A, const int32_t *geno,
                              const double *Q, const double *P,
                              const double *randomArr, int32_t *Z, int32_t *flags)
{
    double W[64];
    *flags = 0;
    for (int i = 0; i < N; i++)
        for (int l = 0; l < L; l++) {
            int taken = 0;
            for (int line = 0; line < 2; line++) {
                size_t pos = ((size_t)i * 2 + line) * L + l;
                int a = geno[pos];
                if (a < 0) { Z[pos] = ORC_UNASSIGNED; continue; }
                double sum = 0.0;
                for (int k = 0; k < K; k++) {
                    W[k] = Q[(size_t)i * K + k] * P[((size_t)l * K + k) * A + a];
                    sum += W[k];
                }
                double u = randomArr[(size_t)i * L * 2 + (size_t)l * 2 + taken++];
                double r = 0.0 + u * (sum - 0.0);
                double so = 0.0;
                int k;
                for (k = 0; k < K; k++) {
                    so += W[k];
                    if (r <= so) break;
                }
                if (k == K) { k = K - 1; *flags |= 1; }
                Z[pos] = k;
            }
        }
}

/* Updates/UpdateP.c:60-99 GetNumFromPops and Updates/UpdateQ.c:17-35 GetNumLociPop */
void orc_counts(int N, int L, int K, int A, const int32_t *geno, const int32_t *Z,
                int pfrompopflagonly, const int32_t *popflags,
                int32_t *n, int32_t *m)
{
    memset(n, 0, sizeof(int32_t) * (size_t)L * K * A);
    memset(m, 0, sizeof(int32_t) * (size_t)N * K);
    for (int i = 0; i < N; i++)
        for (int line = 0; line < 2; line++)
            for (int l = 0; l < L; l++) {
                size_t pos = ((size_t)i * 2 + line) * L + l;
                int z = Z[pos], a = geno[pos];
                if (z == ORC_UNASSIGNED) continue;
                m[(size_t)i * K + z]++;
                if (a >= 0 && (!pfrompopflagonly || popflags[i] == 1))
                    n[((size_t)l * K + z) * A + a]++;
            }
}

/* ------------------------------------------------------------------------ */
/* Dirichlet from log-gamma draws (ran.c:1248-1272 incl. the 1e-100 patch)   */
/* ------------------------------------------------------------------------ */
static void dirichlet_seq(const double *lg, int n, int patch, float *P, float *logP)
{
    double M = lg[0];
    for (int a = 1; a < n; a++) if (lg[a] > M) M = lg[a];
    double S = 0.0;
    for (int a = 0; a < n; a++) S += exp(lg[a] - M);
    double ls = M + log(S);
    if (patch && ls < LOG_UNDERFLO_D) {
        for (int a = 0; a < n; a++) {
            P[a] = (float)(1.0 / (double)n);
            logP[a] = (float)(-log((double)n));
        }
        return;
    }
    for (int a = 0; a < n; a++) {
        double lp = lg[a] - ls;
        logP[a] = (float)lp;
        P[a] = (float)exp(lp);
    }
}

void orc_update_p(int L, int K, int A, const int32_t *numalleles, const int32_t *n,
                  int freqscorr, const double *eps, const double *F,
                  const double *lambda, uint64_t key, uint32_t rep,
                  float *P, float *logP, int *err)
{
    double lg[256];
    for (int l = 0; l < L; l++) {
        int na = numalleles[l];
        for (int k = 0; k < K; k++) {
            size_t base = ((size_t)l * K + k) * A;
            for (int a = 0; a < na; a++) {
                double shape;
                if (freqscorr)
                    shape = eps[(size_t)l * A + a] * (1.0 - F[k]) / F[k] + (double)n[base + a];
                else
                    shape = lambda[k] + (double)n[base + a];
                lg[a] = (double)orc_loggamma_f32((float)shape, (uint32_t)(base + a), rep,
                                                 ORC_S_P, key, err);
            }
            if (na > 0) dirichlet_seq(lg, na, 1, P + base, logP + base);
        }
    }
}

/* Dirichlet over K populations with a G-lane butterfly normalisation. */
static void dirichlet_tree(const double *lg, int K, float *Q, float *logQ)
{
    double v[64];
    int G = pow2_at_least(K);
    double M = lg[0];
    for (int k = 1; k < K; k++) if (lg[k] > M) M = lg[k];
    for (int k = 0; k < G; k++) v[k] = k < K ? exp(lg[k] - M) : 0.0;
    double ls = M + log(tree_sum(v, G));
    for (int k = 0; k < K; k++) {
        double lq = lg[k] - ls;
        logQ[k] = (float)lq;
        Q[k] = (float)exp(lq);
    }
}

void orc_update_q_gibbs(int N, int K, const int32_t *m, const double *alpha,
                        uint64_t key, uint32_t rep, float *Q, float *logQ, int *err,
                        const int32_t *arow)
{
    double lg[64];
    for (int i = 0; i < N; i++) {
        /* LOCPRIOR: the individual's location row of alpha (UpdateQ.c:409-413) */
        const double *al = alpha + (arow ? (size_t)arow[i] * K : 0);
        for (int k = 0; k < K; k++)
            lg[k] = orc_loggamma(al[k] + (double)m[(size_t)i * K + k],
                                 (uint32_t)(i * K + k), rep, ORC_S_QG, key, err);
        dirichlet_tree(lg, K, Q + (size_t)i * K, logQ + (size_t)i * K);
    }
}

void orc_metro_propose(int N, int K, const double *alpha, uint64_t key,
                       uint32_t rep, float *TestQ, float *logTestQ, int *err,
                       const int32_t *arow)
{
    double lg[64];
    for (int i = 0; i < N; i++) {
        const double *al = alpha + (arow ? (size_t)arow[i] * K : 0);   /* UpdateQ.c:255-257 */
        for (int k = 0; k < K; k++)
            lg[k] = orc_loggamma(al[k], (uint32_t)(i * K + k), rep, ORC_S_QM, key, err);
        dirichlet_tree(lg, K, TestQ + (size_t)i * K, logTestQ + (size_t)i * K);
    }
}

/* CalcLike.c:281-345 CalcLikeIndDiff, FP64, same loop order. */
void orc_metro_logdiff(int N, int L, int K, int A, const int32_t *geno,
                       const float *Q, const float *TestQ, const float *P,
                       double *logdiff)
{
    for (int i = 0; i < N; i++) {
        double lp = 0.0, lm = 0.0;
        for (int line = 0; line < 2; line++)
            for (int l = 0; l < L; l++) {
                int a = geno[((size_t)i * 2 + line) * L + l];
                if (a < 0) continue;
                double tp = 0.0, tm = 0.0;
                for (int k = 0; k < K; k++) {
                    double p = P[((size_t)l * K + k) * A + a];
                    tp += (double)TestQ[(size_t)i * K + k] * p;
                    tm += (double)Q[(size_t)i * K + k] * p;
                }
                lp += log(tp);
                lm += log(tm);
            }
        logdiff[i] = lp - lm;
    }
}

/* Updates/UpdateQ.c:278-289: accept if u < exp(logdiff). */
int orc_metro_accept(int N, int K, const double *logdiff, uint64_t key,
                     uint32_t rep, float *Q, float *logQ, const float *TestQ,
                     const float *logTestQ, uint8_t *accepted)
{
    int hits = 0;
    for (int i = 0; i < N; i++) {
        uint32_t w[4];
        philox4((uint32_t)i, 0, rep, ORC_S_QMA, key, w);
        double u = orc_u01(w[0], w[1]);
        int acc = u < exp(logdiff[i]);
        if (accepted) accepted[i] = (uint8_t)acc;
        if (acc) {
            hits++;
            for (int k = 0; k < K; k++) {
                Q[(size_t)i * K + k] = TestQ[(size_t)i * K + k];
                logQ[(size_t)i * K + k] = logTestQ[(size_t)i * K + k];
            }
        }
    }
    return hits;
}

/* ------------------------------------------------------------------------ */
/* alpha                                                                    */
/* ------------------------------------------------------------------------ */
/* S_k = sum_i log Q_ik (LogProbQonepop, UpdateAlpha.c:84-116, unclamped);
 * T = sum_ik log max(Q_ik, sqrt(UNDERFLO)) (LogProbQ, UpdateAlpha.c:144-186). */
void orc_alpha_sums(int N, int K, const float *logQ, double *S, double *T)
{
    const double lclamp = log(SQRT_UNDERFLO);
    *T = 0.0;
    for (int k = 0; k < K; k++) S[k] = 0.0;
    for (int i = 0; i < N; i++)
        for (int k = 0; k < K; k++) {
            double lq = (double)logQ[(size_t)i * K + k];
            S[k] += lq;
            *T += lq > lclamp ? lq : lclamp;
        }
}

/* Updates/UpdateAlpha.c:189-253, including its carry of logprobdiff from one
 * population to the next when UNIFPRIORALPHA=1 and POPALPHAS=1. */
void orc_update_alpha(const orc_alpha_params *p, const double *S, double T,
                      double *alpha, uint64_t key, uint32_t rep, double *lpd_out)
{
    int K = p->K;
    int numalphas = p->popalphas ? K : 1;
    double logprobdiff = 0.0;
    for (int pop = 0; pop < numalphas; pop++) {
        double newalpha = alpha[pop] + p->alphapropsd * orc_normal((uint32_t)pop, rep, ORC_S_ALPHA, key);
        if ((newalpha > 0) && ((newalpha < p->alphamax) || (!(p->unifprioralpha)))) {
            if (!(p->unifprioralpha))
                logprobdiff = (p->alphapriora - 1) * log(newalpha / alpha[pop]) +
                              (alpha[pop] - newalpha) / p->alphapriorb;
            if (p->popalphas) {
                double sumalphas = 0.0;
                for (int i = 0; i < K; i++) sumalphas += alpha[i];
                logprobdiff -= (alpha[pop] - 1.0) * S[pop] +
                               (orc_lgamma(sumalphas) - orc_lgamma(alpha[pop])) * p->N;
                sumalphas += newalpha - alpha[pop];
                logprobdiff += (newalpha - 1.0) * S[pop] +
                               (orc_lgamma(sumalphas) - orc_lgamma(newalpha)) * p->N;
            } else {
                logprobdiff += (newalpha - 1.0) * T +
                               (orc_lgamma(K * newalpha) - K * orc_lgamma(newalpha)) * p->N;
                logprobdiff -= (alpha[pop] - 1.0) * T +
                               (orc_lgamma(K * alpha[pop]) - K * orc_lgamma(alpha[pop])) * p->N;
            }
            uint32_t w[4];
            philox4((uint32_t)pop, 1, rep, ORC_S_ALPHA, key, w);
            double unifrv = orc_rnd31_block(w);
            if (lpd_out) lpd_out[pop] = logprobdiff;
            if (unifrv < exp(logprobdiff)) {
                alpha[pop] = newalpha;
                if (!(p->popalphas))
                    for (int q = 1; q < K; q++) alpha[q] = newalpha;
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* epsilon: Updates/UpdateEpsilon.c:71-145 NonIndependenceUpdateEpsilon      */
/* ------------------------------------------------------------------------ */
void orc_update_eps(int L, int K, int A, const int32_t *numalleles,
                    const float *logP, double *eps, const double *F,
                    double lambda0, double invsqrtnuminds, uint64_t key,
                    uint32_t rep, uint8_t *accepted)
{
    double t[64];
    int G = pow2_at_least(K);
    for (int l = 0; l < L; l++) {
        int na = numalleles[l];
        if (accepted) accepted[l] = 0;
        if (na <= 1) continue;
        uint32_t w[4];
        philox4((uint32_t)l, 0, rep, ORC_S_EPS, key, w);
        int a1 = (int)(((double)(w[0] >> 1) / 2147483648.0) * na);
        int a2 = (int)(((double)(w[1] >> 1) / 2147483648.0) * (na - 1));
        if (a2 >= a1) a2 += 1;
        double difference = 0.0 + ((double)(w[2] >> 1) / 2147483648.0) * (invsqrtnuminds - 0.0);
        double e1 = eps[(size_t)l * A + a1], e2 = eps[(size_t)l * A + a2];
        if (!((e1 + difference < 1.0) && (e2 - difference > 0.0))) continue;
        for (int k = 0; k < G; k++) {
            if (k >= K) { t[k] = 0.0; continue; }
            double frac = (1.0 - F[k]) / F[k];
            double lp1 = (double)logP[((size_t)l * K + k) * A + a1];
            double lp2 = (double)logP[((size_t)l * K + k) * A + a2];
            double s = orc_lgamma(frac * e1);
            s += orc_lgamma(frac * e2);
            s -= orc_lgamma(frac * (e1 + difference));
            s -= orc_lgamma(frac * (e2 - difference));
            s += frac * difference * lp1;
            s -= frac * difference * lp2;
            t[k] = s;
        }
        double sum = tree_sum(t, G);
        if (lambda0 != 1.0)
            sum += log(pow((e1 + difference) * (e2 - difference) / e1 / e2, lambda0 - 1.0));
        philox4((uint32_t)l, 1, rep, ORC_S_EPS, key, w);
        if (orc_rnd31_block(w) < exp(sum)) {
            eps[(size_t)l * A + a1] += difference;
            eps[(size_t)l * A + a2] -= difference;
            if (accepted) accepted[l] = 1;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* F: Updates/UpdateFst.c                                                    */
/* ------------------------------------------------------------------------ */
/* diff[j] = sum over loci/alleles of the FlikeFreqs(new)-FlikeFreqs(old)
 * terms for proposal j (UpdateFst.c:22-51), without the L*lgamma(frac) part. */
void orc_fst_diffs(int L, int K, int A, const int32_t *numalleles,
                   const float *logP, const double *eps, const double *F,
                   int onefst, double fpriorsd, uint64_t key, uint32_t rep,
                   double *newf, double *diff)
{
    int numfst = onefst ? 1 : K;
    for (int j = 0; j < numfst; j++) {
        newf[j] = F[j] + fpriorsd * orc_normal((uint32_t)j, rep, ORC_S_FST, key);
        diff[j] = 0.0;
        if (!(newf[j] > 0.0 && newf[j] < 1.0)) continue;
        double nfr = (1.0 - newf[j]) / newf[j];
        double ofr = (1.0 - F[j]) / F[j];
        int k0 = onefst ? 0 : j, k1 = onefst ? K : j + 1;
        for (int k = k0; k < k1; k++)
            for (int l = 0; l < L; l++)
                for (int a = 0; a < numalleles[l]; a++) {
                    double e = eps[(size_t)l * A + a];
                    double lp = (double)logP[((size_t)l * K + k) * A + a];
                    diff[j] += (nfr - ofr) * e * lp - (orc_lgamma(nfr * e) - orc_lgamma(ofr * e));
                }
    }
}

/* UpdateFst.c:142-204 with FPriorDiff (10-18). */
void orc_update_fst(int K, int onefst, double fpriormean, double fpriorsd,
                    int Leff, const double *diff, const double *newf,
                    double *F, uint64_t key, uint32_t rep, double *lpd_out)
{
    int numfst = onefst ? 1 : K;
    for (int j = 0; j < numfst; j++) {
        double oldf = F[j], nf = newf[j];
        if (!(nf > 0.0 && nf < 1.0)) continue;
        double logprobdiff = (fpriormean * fpriormean / (fpriorsd * fpriorsd) - 1) * log(nf / oldf) +
                             (oldf - nf) * fpriormean / (fpriorsd * fpriorsd);
        double nfr = (1.0 - nf) / nf, ofr = (1.0 - oldf) / oldf;
        int npops = onefst ? K : 1;
        logprobdiff += (double)Leff * npops * (orc_lgamma(nfr) - orc_lgamma(ofr)) + diff[j];
        if (lpd_out) lpd_out[j] = logprobdiff;
        int accept = 0;
        if (logprobdiff >= 0.0) {
            accept = 1;
        } else {
            uint32_t w[4];
            philox4((uint32_t)j, 1, rep, ORC_S_FST, key, w);
            if (orc_rnd31_block(w) < exp(logprobdiff)) accept = 1;
        }
        if (accept) {
            if (onefst) { for (int k = 0; k < K; k++) F[k] = nf; }
            else F[j] = nf;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* CalcLike.c:75-133 CalcLikeInd / 387-426 CalcLike (non-recessive branch)   */
/* ------------------------------------------------------------------------ */
double orc_calc_like(int N, int L, int K, int A, const int32_t *geno,
                     const double *Q, const double *P)
{
    double like = 0.0;
    for (int i = 0; i < N; i++) {
        double rt = 1.0, ll = 0.0;
        for (int line = 0; line < 2; line++)
            for (int l = 0; l < L; l++) {
                int a = geno[((size_t)i * 2 + line) * L + l];
                if (a < 0) continue;
                double term = 0.0;
                for (int k = 0; k < K; k++)
                    term += Q[(size_t)i * K + k] * P[((size_t)l * K + k) * A + a];
                rt *= term > SQRT_UNDERFLO ? term : SQRT_UNDERFLO;
                if (rt < SQRT_UNDERFLO) {
                    ll += log(rt);
                    rt = 1.0;
                }
            }
        ll += log(rt);
        like += ll;
    }
    return like;
}

double orc_calc_like_f(int N, int L, int K, int A, const int32_t *geno,
                       const float *Q, const float *P)
{
    size_t nq = (size_t)N * K, np = (size_t)L * K * A;
    double *q = (double *)malloc(sizeof(double) * nq);
    double *p = (double *)malloc(sizeof(double) * np);
    for (size_t j = 0; j < nq; j++) q[j] = Q[j];
    for (size_t j = 0; j < np; j++) p[j] = P[j];
    double r = orc_calc_like(N, L, K, A, geno, q, p);
    free(q);
    free(p);
    return r;
}

/* Init.c:173-240 InitFreqPriors */
void orc_init_eps(int N, int L, int A, const int32_t *geno,
                  const int32_t *numalleles, int freqscorr, double lambda,
                  double fpriormean, int K, double *eps, double *F)
{
    int cnt[256];
    for (int l = 0; l < L; l++) {
        int na = numalleles[l], total = 0;
        for (int a = 0; a < na; a++) cnt[a] = 0;
        if (freqscorr) {
            for (int i = 0; i < N; i++)
                for (int line = 0; line < 2; line++) {
                    int v = geno[((size_t)i * 2 + line) * L + l];
                    if (v >= 0) { total++; if (v < na) cnt[v]++; }
                }
        }
        for (int a = 0; a < na; a++)
            eps[(size_t)l * A + a] = freqscorr
                ? (((double)lambda + (double)cnt[a]) / ((double)na * (double)lambda + (double)total))
                : lambda;
    }
    for (int k = 0; k < K; k++) F[k] = freqscorr ? fpriormean : 0.5;
}

/* output.c:458-467 EstLogProb with mymath.c:52-62 SampleVar */
double orc_est_logprob(double sumlikes, double sumsqlikes, int reps)
{
    double mean = sumlikes / reps;
    double var = reps == 1 ? 0.0 : (sumsqlikes - sumlikes * sumlikes / reps) / (reps - 1);
    return mean - var / 2.0;
}

/* ------------------------------------------------------------------------ */
/* Gradient of the Z-marginalised log-likelihood (CalcLike.c:75-133          */
/* CalcLikeInd summed over individuals, without the underflow clamps) with   */
/* respect to softmax logits: Q_i = softmax(qlog_i) over K, P_lk =           */
/* softmax(plog_lk) over the A alleles.                                      */
/*   ll = sum_i sum_l sum_copy log S,  S = sum_k Q_ik P_lk,a(copy)            */
/*   dll/dQ_ik = sum_l sum_copy P_lk,a / S;  dll/dP_lka = sum_i sum_copy Q_ik/S */
/*   d/dlogit = p * (g - <p, g>)  (softmax Jacobian)                          */
/* ------------------------------------------------------------------------ */
static void softmax_rows(const double *x, double *y, size_t rows, int n)
{
    for (size_t r = 0; r < rows; r++) {
        const double *a = x + r * n;
        double *b = y + r * n, m = a[0], s = 0.0;
        for (int j = 1; j < n; j++) m = a[j] > m ? a[j] : m;
        for (int j = 0; j < n; j++) { b[j] = exp(a[j] - m); s += b[j]; }
        for (int j = 0; j < n; j++) b[j] /= s;
    }
}

double orc_loglik_grad(int N, int L, int K, int A, const int32_t *geno,
                       const double *qlog, const double *plog,
                       double *dq, double *dp, double *ll_ind)
{
    size_t nq = (size_t)N * K, np = (size_t)L * K * A;
    double *Q = (double *)malloc(sizeof(double) * nq);
    double *P = (double *)malloc(sizeof(double) * np);
    double *gq = (double *)calloc(nq, sizeof(double));
    double *gp = (double *)calloc(np, sizeof(double));
    softmax_rows(qlog, Q, (size_t)N, K);
    softmax_rows(plog, P, (size_t)L * K, A);
    double total = 0.0;
    for (int i = 0; i < N; i++) {
        double lli = 0.0;
        for (int line = 0; line < 2; line++)
            for (int l = 0; l < L; l++) {
                int a = geno[((size_t)i * 2 + line) * L + l];
                if (a < 0) continue;
                double S = 0.0;
                for (int k = 0; k < K; k++)
                    S += Q[(size_t)i * K + k] * P[((size_t)l * K + k) * A + a];
                lli += log(S);
                for (int k = 0; k < K; k++) {
                    gq[(size_t)i * K + k] += P[((size_t)l * K + k) * A + a] / S;
                    gp[((size_t)l * K + k) * A + a] += Q[(size_t)i * K + k] / S;
                }
            }
        if (ll_ind) ll_ind[i] = lli;
        total += lli;
    }
    for (int i = 0; i < N; i++) {
        double s = 0.0;
        for (int k = 0; k < K; k++) s += Q[(size_t)i * K + k] * gq[(size_t)i * K + k];
        for (int k = 0; k < K; k++)
            dq[(size_t)i * K + k] = Q[(size_t)i * K + k] * (gq[(size_t)i * K + k] - s);
    }
    for (size_t r = 0; r < (size_t)L * K; r++) {
        double s = 0.0;
        for (int a = 0; a < A; a++) s += P[r * A + a] * gp[r * A + a];
        for (int a = 0; a < A; a++) dp[r * A + a] = P[r * A + a] * (gp[r * A + a] - s);
    }
    free(Q); free(P); free(gq); free(gp);
    return total;
}

/* ll_i and dll/dQ_ik for one individual, Q and P given (P [L][K][2]). */
static double ind_loglik_dq(int L, int K, const int32_t *geno, int i, int N_unused,
                            const double *q, const float *P, double *g)
{
    (void)N_unused;
    double ll = 0.0;
    for (int k = 0; k < K; k++) g[k] = 0.0;
    for (int line = 0; line < 2; line++)
        for (int l = 0; l < L; l++) {
            int a = geno[((size_t)i * 2 + line) * L + l];
            if (a < 0) continue;
            double S = 0.0;
            for (int k = 0; k < K; k++) S += q[k] * (double)P[((size_t)l * K + k) * 2 + a];
            ll += log(S);
            for (int k = 0; k < K; k++) g[k] += (double)P[((size_t)l * K + k) * 2 + a] / S;
        }
    return ll;
}

void orc_mala_step(int N, int L, int K, const int32_t *geno, float *Q, float *logQ,
                   const float *P, const double *alpha, int popalphas, float *eps,
                   uint64_t key, uint32_t rep, int burnin, double target,
                   double *logr, uint8_t *acc)
{
    double q[64], qp[64], g[64], gp[64], th[64], thp[64], al[64];
    double A = 0.0;
    for (int k = 0; k < K; k++) { al[k] = popalphas ? alpha[k] : alpha[0]; A += al[k]; }
    for (int i = 0; i < N; i++) {
        if (K < 2) { logr[i] = 0.0; acc[i] = 0; continue; }
        float *Qi = Q + (size_t)i * K, *lQi = logQ + (size_t)i * K;
        for (int k = 0; k < K; k++) q[k] = Qi[k];
        double ll0 = ind_loglik_dq(L, K, geno, i, N, q, P, g);
        double s = 0.0;
        for (int k = 0; k < K; k++) s += q[k] * g[k];
        for (int k = 0; k < K; k++) g[k] = q[k] * (g[k] - s);     /* dll/dlogit */
        double e = eps[i], h = 0.5 * e * e, base = lQi[K - 1], m = 0.0;
        for (int j = 0; j < K - 1; j++) {
            uint32_t w[4];
            philox4((uint32_t)i, 1u + (uint32_t)j, rep, ORC_S_MALA, key, w);
            double xi = sqrt(-2.0 * log(orc_u01(w[0], w[1]))) * cos(TWO_PI * orc_u01(w[2], w[3]));
            th[j] = (double)lQi[j] - base;
            double grad = g[j] + al[j] - q[j] * A;
            thp[j] = th[j] + h * grad + e * xi;
            if (thp[j] > m) m = thp[j];
        }
        th[K - 1] = thp[K - 1] = 0.0;
        double ss = 0.0;
        for (int k = 0; k < K; k++) ss += exp(thp[k] - m);
        for (int k = 0; k < K; k++) qp[k] = (double)(float)(exp(thp[k] - m) / ss);
        double ll1 = ind_loglik_dq(L, K, geno, i, N, qp, P, gp);
        s = 0.0;
        for (int k = 0; k < K; k++) s += qp[k] * gp[k];
        for (int k = 0; k < K; k++) gp[k] = qp[k] * (gp[k] - s);
        double m0 = 0.0, m1 = 0.0, s0 = 0.0, s1 = 0.0;
        for (int k = 0; k < K; k++) { if (th[k] > m0) m0 = th[k]; if (thp[k] > m1) m1 = thp[k]; }
        for (int k = 0; k < K; k++) { s0 += exp(th[k] - m0); s1 += exp(thp[k] - m1); }
        double lse0 = m0 + log(s0), lse1 = m1 + log(s1);
        double lp0 = ll0, lp1 = ll1;
        for (int k = 0; k < K; k++) { lp0 += al[k] * (th[k] - lse0); lp1 += al[k] * (thp[k] - lse1); }
        double fwd = 0.0, bwd = 0.0;
        for (int j = 0; j < K - 1; j++) {
            double g0 = g[j] + al[j] - q[j] * A, g1 = gp[j] + al[j] - qp[j] * A;
            double df = thp[j] - th[j] - h * g0, db = th[j] - thp[j] - h * g1;
            fwd += df * df;
            bwd += db * db;
        }
        double lr = lp1 - lp0 - (bwd - fwd) / (2.0 * e * e);
        uint32_t w[4];
        philox4((uint32_t)i, 0u, rep, ORC_S_MALA, key, w);
        int a = log(orc_u01(w[0], w[1])) < lr;
        logr[i] = lr;
        acc[i] = (uint8_t)a;
        if (a)
            for (int k = 0; k < K; k++) { Qi[k] = (float)qp[k]; lQi[k] = (float)(thp[k] - lse1); }
        if ((int)rep < burnin) {
            double pa = lr >= 0.0 ? 1.0 : (lr == lr ? exp(lr) : 0.0);
            double en = e * exp(pow((double)rep + 1.0, -0.6) * (pa - target));
            en = en < 1e-6 ? 1e-6 : (en > 10.0 ? 10.0 : en);
            eps[i] = (float)en;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Updates/UpdateLambda.c:8-102 UpdatePopLambda / UpdateLambda: proposal      */
/* N(lambda, 0.3) inside (0, 10), log ratio over loci with >1 allele.         */
/* ------------------------------------------------------------------------ */
void orc_update_lambda(int L, int K, int A, const int32_t *numalleles, const float *logP,
                       const double *eps, int freqscorr, int popspecific, double *lambda,
                       uint64_t key, uint32_t rep, double *lpd_out)
{
    const double maxl = 10.0, sd = 0.3;
    int npop = popspecific ? K : 1;
    for (int q = 0; q < npop; q++) {
        double lam = lambda[q];
        double nw = lam + sd * orc_normal((uint32_t)q, rep, ORC_S_LAMBDA, key);
        if (lpd_out) lpd_out[q] = NAN;
        if (!(nw > 0.0 && nw < maxl)) continue;
        double reps = popspecific ? 1.0 : (freqscorr ? 1.0 : (double)K);
        double sum = 0.0;
        for (int l = 0; l < L; l++) {
            int na = numalleles[l];
            if (na <= 1) continue;
            sum += reps * orc_lgamma(na * nw);
            sum -= reps * orc_lgamma(na * lam);
            sum += reps * na * orc_lgamma(lam);
            sum -= reps * na * orc_lgamma(nw);
            double slog = 0.0;
            if (popspecific) {
                for (int a = 0; a < na; a++) slog += (double)logP[((size_t)l * K + q) * A + a];
            } else if (freqscorr) {
                for (int a = 0; a < na; a++) slog += log(eps[(size_t)l * A + a]);
            } else {
                for (int k = 0; k < K; k++)
                    for (int a = 0; a < na; a++) slog += (double)logP[((size_t)l * K + k) * A + a];
            }
            sum += (nw - lam) * slog;
        }
        if (lpd_out) lpd_out[q] = sum;
        uint32_t w[4];
        philox4((uint32_t)q, 1, rep, ORC_S_LAMBDA, key, w);
        if (orc_rnd31_block(w) < exp(sum)) {
            if (popspecific) lambda[q] = nw;
            else for (int k = 0; k < K; k++) lambda[k] = nw;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Updates/UpdateQ.c:310-383 UpdateQNoAdmix with mymath.c:80-100 PickAnOption */
/* ------------------------------------------------------------------------ */
void orc_update_q_noadmix(int N, int L, int K, int A, const int32_t *geno, const float *logP,
                          uint64_t key, uint32_t rep, float *Q, float *logQ, int32_t *pick,
                          const double *locp, const int32_t *myloc)
{
    double p[64];
    for (int i = 0; i < N; i++) {
        double mx = 0.0;
        for (int k = 0; k < K; k++) {
            /* LOCPRIOR: the product starts at gamma[myloc][k] (UpdateQ.c:339-345) */
            double s = locp ? log(locp[1 + (size_t)K * (myloc[i] + 1) + k]) : 0.0;
            for (int l = 0; l < L; l++)
                for (int line = 0; line < 2; line++) {
                    int a = geno[((size_t)i * 2 + line) * L + l];
                    if (a >= 0) s += (double)logP[((size_t)l * K + k) * A + a];
                }
            p[k] = s;
            if (k == 0 || s > mx) mx = s;
        }
        double sum = 0.0;
        for (int k = 0; k < K; k++) sum += (p[k] = exp(p[k] - mx));
        uint32_t w[4];
        philox4((uint32_t)i, 0, rep, ORC_S_NOADMIX, key, w);
        double r = (double)(w[0] >> 1) / 2147483648.0 * sum, cum = 0.0;
        int pk = K - 1;
        for (int k = 0; k < K; k++) {
            cum += p[k];
            if (r <= cum) { pk = k; break; }
        }
        if (pick) pick[i] = pk;
        for (int k = 0; k < K; k++) {
            Q[(size_t)i * K + k] = k == pk ? 1.0f : 0.0f;
            logQ[(size_t)i * K + k] = k == pk ? 0.0f : -INFINITY;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Updates/UpdateQ.c:499-706 UpdateQWithPops: migrant model for individuals  */
/* with prior population information.                                        */
/* ------------------------------------------------------------------------ */
void orc_update_q_withpops(int N, int L, int K, int A, const int32_t *geno, const float *P,
                           const int32_t *population, const int32_t *popflags, int gensback,
                           double migrprior, uint64_t key, uint32_t rep, int burnin, float *Q,
                           float *logQ, double *usepop)
{
    const int G = gensback + 1;
    double post[64 * 8], pri[8];
    double w = 0.5, sw = 0.0;
    for (int g = 0; g < G; g++) { w *= 2.0; pri[g] = w; sw += w * (K - 1); }
    for (int g = 0; g < G; g++) pri[g] = migrprior * pri[g] / sw;
    for (int i = 0; i < N; i++) {
        if (!popflags[i]) continue;
        const int home = population[i] - 1;
        double mx = 0.0;
        for (int k = 0; k < K; k++)
            for (int g = 0; g < G; g++) {
                const double p = g > 0 ? exp((g - 1) * log(0.5)) : 1.0;
                double s = 0.0;
                for (int l = 0; l < L; l++) {
                    const int a0 = geno[((size_t)i * 2) * L + l];
                    const int a1 = geno[((size_t)i * 2 + 1) * L + l];
                    const float *Pl = P + (size_t)l * K * A;
                    double like;
                    if (a0 >= 0 && a1 >= 0) {
                        double pk0 = Pl[k * A + a0], ph0 = Pl[home * A + a0];
                        double pk1 = Pl[k * A + a1], ph1 = Pl[home * A + a1];
                        like = g == 0 ? pk0 * pk1
                                      : 0.5 * p * pk0 * ph1 + 0.5 * p * ph0 * pk1 +
                                            (1.0 - p) * ph0 * ph1;
                    } else if (a0 >= 0) {
                        like = p * Pl[k * A + a0] + (1.0 - p) * Pl[home * A + a0];
                    } else if (a1 >= 0) {
                        like = p * Pl[home * A + a1] + (1.0 - p) * Pl[home * A + a1];
                    } else {
                        continue;
                    }
                    s += log(like > SQRT_UNDERFLO ? like : SQRT_UNDERFLO);
                }
                post[k * G + g] = s;
                if ((k == 0 && g == 0) || s > mx) mx = s;
            }
        double sum = 0.0;
        for (int g = 0; g < G; g++)
            for (int k = 0; k < K; k++) {
                double *v = &post[k * G + g];
                *v = exp(*v - mx);
                if (k == home) *v = g == 0 ? *v * (1.0 - migrprior) : 0.0;
                else *v *= pri[g];
                sum += *v;
            }
        if ((int)rep >= burnin)
            for (int j = 0; j < K * G; j++) usepop[(size_t)i * K * G + j] += post[j] / sum;
        uint32_t u[4];
        philox4((uint32_t)i, 0, rep, ORC_S_POPINFO, key, u);
        const double r = (double)(u[0] >> 1) / 2147483648.0 * sum;
        double cum = 0.0;
        int pk = home, pg = 0, done = 0;
        for (int g = 0; g < G && !done; g++)
            for (int k = 0; k < K; k++) {
                cum += post[k * G + g];
                if (r < cum) { pk = k; pg = g; done = 1; break; }
            }
        double q[64];
        for (int k = 0; k < K; k++) q[k] = 0.0;
        const double p = exp(pg * log(0.5));
        q[pk] = p;
        q[home] += 1.0 - p;
        for (int k = 0; k < K; k++) {
            Q[(size_t)i * K + k] = (float)q[k];
            logQ[(size_t)i * K + k] = q[k] > 0.0 ? (float)log(q[k]) : -INFINITY;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* LOCPRIOR                                                                 */
/* ------------------------------------------------------------------------ */
/* Uniform draws in the form of ran.c:128-147 RandomReal / RandomInteger on a
 * 31-bit rand() word (here w >> 1 of a Philox word); the words and normals
 * are appended to the trace in the order the reference consumes them. */
static double lp_real(uint32_t w, double lo, double hi, orc_trace *tr)
{
    uint32_t v = w >> 1;
    if (tr) tr->rw[tr->nr++] = (int32_t)v;
    double d = (double)v / 2147483648.0;
    return lo + d * (hi - lo);
}

static int lp_int(uint32_t w, int lo, int hi, orc_trace *tr)
{
    uint32_t v = w >> 1;
    if (tr) tr->rw[tr->nr++] = (int32_t)v;
    double d = (double)v / 2147483648.0;
    return lo + (int)(d * (hi - lo + 1));
}

static double lp_normal(uint32_t idx, uint32_t rep, uint64_t key, orc_trace *tr)
{
    double z = orc_normal(idx, rep, ORC_S_LOCALPHA, key);
    if (tr) tr->nv[tr->nn++] = z;
    return z;
}

/* Updates/UpdateLocPrior.c:12-140: UpdateLocPriorNoAdmix (r, nu, gamma) and
 * UpdateLocPriorAdmix (r only).  locp is the reference's LocPrior array:
 * [0] r, [1 + k] nu (eta), [1 + K*(loc+1) + k] gamma of location loc.
 * alpha [(nloc+1)][K]: the global row, then one row per location.
 * Draws: r at (0, 0) of ORC_S_LOCPRIOR (word 0 the proposal, word 1 the
 * acceptance), nu at (0, 1) (words: pop1, pop2, step, acceptance), gamma of
 * location loc at (loc, 2) (same words). */
void orc_update_locprior(int N, int K, int nloc, int noadmix, const int32_t *myloc,
                         const float *Q, const double *alpha, double *locp,
                         double alphapropsd, double step, double maxlp, uint64_t key,
                         uint32_t rep, orc_trace *tr)
{
    uint32_t w[4];
    const double cur = locp[0];
    philox4(0, 0, rep, ORC_S_LOCPRIOR, key, w);
    const double nw = lp_real(w[0], cur - step, cur + step, tr);
    if (!noadmix) {
        if (nw > 0.0 && nw < maxlp) {
            const double d = nw - cur;
            double diff = 0.0;
            for (int k = 0; k < K; k++) {
                const double ga = alpha[k];
                for (int loc = 0; loc < nloc; loc++) {
                    const double la = alpha[(size_t)K * (loc + 1) + k];
                    diff += ga * d * log(la) - d * la - orc_lgamma(ga * nw) +
                            orc_lgamma(ga * cur) + ga * nw * log(nw) - ga * cur * log(cur);
                }
            }
            if (diff > 0.0 || lp_real(w[1], 0.0, 1.0, tr) < exp(diff)) locp[0] = nw;
        }
        return;
    }
    double *eta = locp + 1;
    double *gam = locp + 1 + K;     /* gam[loc*K + k] */
    if (nw > 0.0 && nw < maxlp) {
        double ld = orc_lgamma(nw) - orc_lgamma(cur);
        for (int k = 0; k < K; k++) ld += orc_lgamma(cur * eta[k]) - orc_lgamma(nw * eta[k]);
        ld *= nloc;
        for (int loc = 0; loc < nloc; loc++)
            for (int k = 0; k < K; k++) ld += (nw - cur) * eta[k] * log(gam[(size_t)loc * K + k]);
        if (ld >= 0.0 || lp_real(w[1], 0.0, 1.0, tr) < exp(ld)) locp[0] = nw;
    }
    const double r = locp[0];
    philox4(0, 1, rep, ORC_S_LOCPRIOR, key, w);
    int p1 = lp_int(w[0], 0, K - 1, tr), p2 = lp_int(w[1], 0, K - 2, tr);
    if (p2 >= p1) p2++;
    double dd = lp_real(w[2], 0.0, alphapropsd, tr);
    double e1 = eta[p1] + dd, e2 = eta[p2] - dd;
    if (e1 < 1.0 && e2 > 0.0) {
        double ld = nloc * (orc_lgamma(r * eta[p1]) + orc_lgamma(r * eta[p2]) -
                            orc_lgamma(r * e1) - orc_lgamma(r * e2));
        for (int loc = 0; loc < nloc; loc++)
            ld += r * ((e1 - eta[p1]) * log(gam[(size_t)loc * K + p1]) +
                       (e2 - eta[p2]) * log(gam[(size_t)loc * K + p2]));
        if (ld >= 0.0 || lp_real(w[3], 0.0, 1.0, tr) < exp(ld)) {
            eta[p1] = e1;
            eta[p2] = e2;
        }
    }
    for (int loc = 0; loc < nloc; loc++) {
        double dc1, dc2;
        philox4((uint32_t)loc, 2, rep, ORC_S_LOCPRIOR, key, w);
        p1 = lp_int(w[0], 0, K - 1, tr);
        p2 = lp_int(w[1], 0, K - 2, tr);
        if (p2 >= p1) p2++;
        dd = lp_real(w[2], 0.0, alphapropsd, tr);
        double *gl = gam + (size_t)loc * K;
        const double g1 = gl[p1] + dd, g2 = gl[p2] - dd;
        if (!(g1 < 1.0 && g2 > 0.0)) continue;
        dc1 = dc2 = 0.0;    /* sum of Q over the location's individuals */
        for (int i = 0; i < N; i++)
            if (myloc[i] == loc) {
                dc1 += (double)Q[(size_t)i * K + p1];
                dc2 += (double)Q[(size_t)i * K + p2];
            }
        const double l1 = log(g1) - log(gl[p1]), l2 = log(g2) - log(gl[p2]);
        const double ld = (r * eta[p1] - 1.0) * l1 + (r * eta[p2] - 1.0) * l2 + dc1 * l1 + dc2 * l2;
        if (ld >= 0.0 || lp_real(w[3], 0.0, 1.0, tr) < exp(ld)) {
            gl[p1] = g1;
            gl[p2] = g2;
        }
    }
}

/* Updates/UpdateAlpha.c:118-139,257-305 UpdateAlphaLocPrior with
 * LogProbQ_LocPrior_loc: the global alphas (a normal step each, accepted on
 * the Gamma(alpha_k r, r) densities of the location alphas), then each
 * location's alphas in turn against Pr(Q of its individuals | alpha_loc).
 * logQ [N][K] in FP64.  Draws: the normal of global alpha k at (k, 0) of
 * ORC_S_LOCALPHA and its acceptance at (k, 1) word 0; location loc, pop k:
 * index K*(loc+1)+k likewise. */
static double lp_logprob_loc(int N, int K, const int32_t *myloc, const double *logQ,
                             const double *al, int loc)
{
    double like = 0.0, sa = 0.0, sg = 0.0;
    int n = 0;
    for (int i = 0; i < N; i++) {
        if (myloc[i] != loc) continue;
        for (int k = 0; k < K; k++) like += (al[k] - 1.0) * logQ[(size_t)i * K + k];
        n++;
    }
    for (int k = 0; k < K; k++) {
        sa += al[k];
        sg += orc_lgamma(al[k]);
    }
    return like + (orc_lgamma(sa) - sg) * (double)n;
}

void orc_update_alpha_locprior(int N, int K, int nloc, const int32_t *myloc, const double *logQ,
                               double *alpha, double r, double alphapropsd, double alphamax,
                               uint64_t key, uint32_t rep, orc_trace *tr)
{
    uint32_t w[4];
    for (int k = 0; k < K; k++) {
        const double old = alpha[k];
        const double nw = old + alphapropsd * lp_normal((uint32_t)k, rep, key, tr);
        if (nw >= alphamax || nw <= 0.0) continue;
        double diff = 0.0;
        for (int loc = 0; loc < nloc; loc++)
            diff += (nw - old) * r * log(alpha[(size_t)K * (loc + 1) + k]) - orc_lgamma(nw * r) +
                    orc_lgamma(old * r) + (nw - old) * r * log(r);
        philox4((uint32_t)k, 1, rep, ORC_S_LOCALPHA, key, w);
        if (diff > 0.0 || lp_real(w[0], 0.0, 1.0, tr) < exp(diff)) alpha[k] = nw;
    }
    for (int loc = 0; loc < nloc; loc++) {
        double *al = alpha + (size_t)K * (loc + 1);
        double lp = lp_logprob_loc(N, K, myloc, logQ, al, loc);
        for (int k = 0; k < K; k++) {
            const uint32_t idx = (uint32_t)(K * (loc + 1) + k);
            const double ga = alpha[k], old = al[k];
            const double nw = old + alphapropsd * lp_normal(idx, rep, key, tr);
            if (nw <= 0.0) continue;
            al[k] = nw;
            const double lpn = lp_logprob_loc(N, K, myloc, logQ, al, loc);
            const double diff = (ga * r - 1.0) * log(nw / old) - r * (nw - old) + lpn - lp;
            philox4(idx, 1, rep, ORC_S_LOCALPHA, key, w);
            if (diff >= 0.0 || lp_real(w[0], 0.0, 1.0, tr) < exp(diff)) lp = lpn;
            else al[k] = old;
        }
    }
}
