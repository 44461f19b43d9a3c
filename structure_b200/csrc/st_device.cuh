// st_device.cuh -- device-side building blocks shared by the sweep kernels:
// Philox4x32-10 counters, uniform/normal conversions, the Lanczos ln-Gamma,
// Marsaglia-Tsang log-gamma draws and warp-group reductions.
//
// Built with -fmad=false: every a*b+c below is two IEEE roundings unless it
// is written as an explicit fma intrinsic, so the host restatement of the same
// formulas (compiled with -ffp-contract=off) reproduces them exactly, up to
// the last-ulp differences of log/exp/sin/cos between CUDA and libm.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "st_types.h"

namespace st {

// Random123 Philox4x32-10 with a fixed key, so the ten round keys are
// compile-time immediates; a chain's identity is the counter word seed32.
// Streams: counter = {a, (stream << 24) | (b & 0xFFFFFF), sweep, seed32},
// seed32 = low word of splitmix64(chain seed).
struct U4 { uint32_t x, y, z, w; };

constexpr uint32_t kPhiloxKey0 = 0xA511E9B3u, kPhiloxKey1 = 0x3C6EF372u;

__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t k0 = kPhiloxKey0 + (uint32_t)r * 0x9E3779B9u;
    const uint32_t k1 = kPhiloxKey1 + (uint32_t)r * 0xBB67AE85u;
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;   // one 32x32->64 multiply each
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
  }
  return U4{c0, c1, c2, c3};
}

__device__ __forceinline__ U4 philox_s(uint32_t a, uint32_t b, uint32_t rep,
                                       uint32_t stream, uint32_t seed32) {
  return philox(a, (stream << 24) | (b & 0xFFFFFFu), rep, seed32);
}

// philox_s for a run of blocks that share a, rep, stream and seed32 and differ
// only in b (the data pass: one locus, one sweep, consecutive individual
// pairs).  The work of rounds 0-3 that does not depend on b is done once in
// the constructor; block(b) returns exactly philox_s(a, b, rep, stream, seed32)
// with 33 instead of 40 multiply/xor steps.  c0 after round 0 is
// head ^ (b & 0xFFFFFF), which the caller may form itself (block_r0).
struct PhiloxRun {
  uint32_t head;         // hi(M1 rep) ^ k0_0 ^ (stream << 24)
  uint32_t y1, z0, z2, w3;
  __device__ __forceinline__ PhiloxRun(uint32_t a, uint32_t rep, uint32_t stream,
                                       uint32_t seed32) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * a, p1 = (uint64_t)0xCD9E8D57u * rep;
    head = (uint32_t)(p1 >> 32) ^ kPhiloxKey0 ^ (stream << 24);
    const uint32_t a1 = (uint32_t)p1, a2 = (uint32_t)(p0 >> 32) ^ seed32 ^ kPhiloxKey1,
                   a3 = (uint32_t)p0;
    const uint64_t q1 = (uint64_t)0xCD9E8D57u * a2;                     // round 1, c2 fixed
    const uint32_t b0 = (uint32_t)(q1 >> 32) ^ a1 ^ (kPhiloxKey0 + 0x9E3779B9u);
    y1 = a3 ^ (kPhiloxKey1 + 0xBB67AE85u);
    z0 = (uint32_t)q1 ^ (kPhiloxKey0 + 2u * 0x9E3779B9u);
    const uint64_t q2 = (uint64_t)0xD2511F53u * b0;                     // round 2, c0 fixed
    z2 = (uint32_t)(q2 >> 32) ^ (kPhiloxKey1 + 2u * 0xBB67AE85u);
    w3 = (uint32_t)q2 ^ (kPhiloxKey1 + 3u * 0xBB67AE85u);
  }
  __device__ __forceinline__ U4 block_r0(uint32_t c0) const {
    const uint64_t r1 = (uint64_t)0xD2511F53u * c0;                     // round 1
    const uint32_t r1c2 = (uint32_t)(r1 >> 32) ^ y1, r1c3 = (uint32_t)r1;
    const uint64_t r2 = (uint64_t)0xCD9E8D57u * r1c2;                   // round 2
    const uint32_t r2c0 = (uint32_t)(r2 >> 32) ^ z0, r2c1 = (uint32_t)r2, r2c2 = r1c3 ^ z2;
    const uint64_t p0 = (uint64_t)0xD2511F53u * r2c0;                   // round 3
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * r2c2;
    uint32_t c0n = (uint32_t)(p1 >> 32) ^ r2c1 ^ (kPhiloxKey0 + 3u * 0x9E3779B9u);
    uint32_t c1n = (uint32_t)p1, c2n = (uint32_t)(p0 >> 32) ^ w3, c3n = (uint32_t)p0;
#pragma unroll
    for (int r = 4; r < 10; r++) {
      const uint32_t k0 = kPhiloxKey0 + (uint32_t)r * 0x9E3779B9u;
      const uint32_t k1 = kPhiloxKey1 + (uint32_t)r * 0xBB67AE85u;
      const uint64_t q0 = (uint64_t)0xD2511F53u * c0n;
      const uint64_t q1 = (uint64_t)0xCD9E8D57u * c2n;
      const uint32_t n0 = (uint32_t)(q1 >> 32) ^ c1n ^ k0;
      const uint32_t n2 = (uint32_t)(q0 >> 32) ^ c3n ^ k1;
      c0n = n0; c1n = (uint32_t)q1; c2n = n2; c3n = (uint32_t)q0;
    }
    return U4{c0n, c1n, c2n, c3n};
  }
  __device__ __forceinline__ U4 block(uint32_t b) const { return block_r0(head ^ (b & 0xFFFFFFu)); }
};

// 52-bit uniform in (0,1).
__device__ __forceinline__ double u01(uint32_t hi, uint32_t lo) {
  uint64_t x = ((uint64_t)(hi >> 6) << 26) | (uint64_t)(lo >> 6);
  return ((double)x + 0.5) * (1.0 / 4503599627370496.0);
}

// rnd() of ran.c:152 on a rand() stream w>>1 (31 bits), skipping zeros.
__device__ __forceinline__ double rnd31(U4 w) {
  uint32_t v[4] = {w.x >> 1, w.y >> 1, w.z >> 1, w.w >> 1};
#pragma unroll
  for (int j = 0; j < 4; j++)
    if (v[j] != 0) return (double)v[j] / 2147483648.0;
  return 1.0 / 4294967296.0;
}

// Uniform u in [0,1) for the categorical draw of Z: a Philox word's low 23
// bits over 2^23.  neg_one_plus_u23 builds -(1 + u) directly from those bits
// (exponent of -1, the bits as mantissa: exact), so that
// fma(-(1 + u), T, T) = RN(T - (1 + u) T) = RN(-u T) in one rounding, which is
// -RN(u T): the same threshold r = RN(u T) that u23(w) * T gives.
__device__ __forceinline__ float u23(uint32_t w) {
  return (float)(w & 0x7FFFFFu) * (1.0f / 8388608.0f);
}
__device__ __forceinline__ float neg_one_plus_u23(uint32_t w) {
  return __uint_as_float(0xBF800000u | (w & 0x7FFFFFu));
}

// Neumaier's compensated summation (the Kahan-Babuska form, which also holds
// when a term outweighs the running sum): s + c carries the sum of the terms
// added so far to about twice the working precision.  Additions only, so
// contraction flags do not change it.
struct CompSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

constexpr double kTwoPi = 6.283185307179586;

// Standard normal for MH proposals: Box-Muller on block {idx, 0, rep, stream}.
__device__ __forceinline__ double normal_draw(uint32_t idx, uint32_t rep,
                                              uint32_t stream, uint32_t key) {
  U4 w = philox_s(idx, 0, rep, stream, key);
  double u1 = u01(w.x, w.y), u2 = u01(w.z, w.w);
  return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
}

// ln Gamma(z), z > 0: Lanczos (1964) series, g = 7, nine terms, with the
// coefficient set and summation order of the reference's mylgamma.
__device__ __forceinline__ double lanczos_lgamma(double z) {
  const double c1 = 676.5203681218835, c2 = -1259.139216722289,
               c3 = 771.3234287757674, c4 = -176.6150291498386,
               c5 = 12.50734324009056, c6 = -0.1385710331296526,
               c7 = 9.934937113930748e-6, c8 = 1.659470187408462e-7;
  double s = 0.0, t = z + 7.0;
  s += c8 / t; t -= 1.0;
  s += c7 / t; t -= 1.0;
  s += c6 / t; t -= 1.0;
  s += c5 / t; t -= 1.0;
  s += c4 / t; t -= 1.0;
  s += c3 / t; t -= 1.0;
  s += c2 / t; t -= 1.0;
  s += c1 / t;
  s += 0.9999999999995183;
  return log(s) + 0.9189385332046727 - (z + 6.5) + (z - 0.5) * log(z + 6.5);
}

// The same series evaluated with one division: the fractions c_j/(z+j) are
// folded into one numerator/denominator pair from the innermost term out,
//   num/den <- (num*(z+j) + c_{j+1}*den) / (den*(z+j)),
// which has the condition number of the original sum (all z+j > 0) and costs
// one DDIV instead of eight.  Agrees with lanczos_lgamma to a few ulps.
__device__ __forceinline__ double lanczos_lgamma_fast(double z) {
  double num = 1.659470187408462e-7, den = z + 7.0, f;
  f = z + 6.0; num = num * f + 9.934937113930748e-6 * den; den *= f;
  f = z + 5.0; num = num * f + -0.1385710331296526 * den; den *= f;
  f = z + 4.0; num = num * f + 12.50734324009056 * den; den *= f;
  f = z + 3.0; num = num * f + -176.6150291498386 * den; den *= f;
  f = z + 2.0; num = num * f + 771.3234287757674 * den; den *= f;
  f = z + 1.0; num = num * f + -1259.139216722289 * den; den *= f;
  f = z;       num = num * f + 676.5203681218835 * den; den *= f;
  const double s = 0.9999999999995183 + num / den;
  return log(s) + 0.9189385332046727 - (z + 6.5) + (z - 0.5) * log(z + 6.5);
}

// log of a Gamma(a, 1) draw by Marsaglia & Tsang (2000), "A simple method for
// generating gamma variables", ACM TOMS 26(3).  Attempts come in pairs: block
// 2j yields two Box-Muller normals, block 2j+1 their acceptance uniforms.
// For a < 1, G(a) = G(a+1) * U^(1/a) (U from block 0xFFFFFF), in logs so that
// tiny shapes never underflow.
static __device__ __noinline__ double log_gamma_draw(double a, uint32_t e, uint32_t rep,
                                                 uint32_t stream, uint32_t key,
                                                 int* errbits) {
  double aa = a < 1.0 ? a + 1.0 : a;
  double d = aa - 1.0 / 3.0;
  double c = 1.0 / sqrt(9.0 * d);
  double lg = 0.0;
  bool done = false;
  for (uint32_t j = 0; j < kGammaMaxBlocks && !done; j += 2) {
    U4 b0 = philox_s(e, j, rep, stream, key);
    U4 b1 = philox_s(e, j + 1, rep, stream, key);
    double u1 = u01(b0.x, b0.y), u2 = u01(b0.z, b0.w);
    double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincos(kTwoPi * u2, &s, &co);
    double xs[2] = {rad * co, rad * s};
    double vs[2] = {u01(b1.x, b1.y), u01(b1.z, b1.w)};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (done) break;
      double x = xs[h];
      double t = 1.0 + c * x;
      if (t <= 0.0) continue;
      double v = t * t * t;
      double x2 = x * x;
      double u = vs[h];
      if (u < 1.0 - 0.0331 * x2 * x2 || log(u) < 0.5 * x2 + d * (1.0 - v + log(v))) {
        lg = log(d * v);
        done = true;
      }
    }
  }
  if (!done) {
    *errbits |= kErrGammaCap;
    lg = log(d);
  }
  if (a < 1.0) {
    U4 w = philox_s(e, 0xFFFFFFu, rep, stream, key);
    lg += log(u01(w.x, w.y)) / a;
  }
  return lg;
}

// ---------------------------------------------------------------------------
// FP32 gamma draws for the Dirichlet of P.  Every operation below is an
// IEEE-rounded add, multiply, fma, divide or square root written as an
// explicit _rn intrinsic (never contracted, whatever -fmad says), so the
// oracle's C restatement of the same sequence gives the same bits.  log and
// sin/cos are this file's own: the atanh series of the logarithm and the
// Taylor series of sine and cosine, after exact range reductions.
// ---------------------------------------------------------------------------
// Uniform in (0,1) from a word's top 23 bits k: (2k + 1) / 2^24, exact in
// FP32 (the odd integer has at most 24 bits).
__device__ __forceinline__ float u23c_f32(uint32_t w) {
  return __fmul_rn((float)(((w >> 9) << 1) | 1u), 5.9604644775390625e-8f);
}

// ln x for a positive normal float: x = 2^e m with m in [sqrt(1/2), sqrt(2)),
// s = (m - 1) / (m + 1) (m - 1 exact), ln m = 2 atanh s = 2s (1 + s^2/3 +
// s^4/5 + ... + s^10/11) (|s| < 0.172, the next term below 2e-9 relative),
// and e ln 2 split into a 15-bit head (e ln2_hi exact for |e| < 256) and a
// tail (Cody and Waite's reduction).
__device__ __forceinline__ float ln_f32(float x) {
  const uint32_t b = __float_as_uint(x);
  int e = (int)((b >> 23) & 0xFFu) - 127;
  float m = __uint_as_float((b & 0x7FFFFFu) | 0x3F800000u);
  if (m > 1.41421356f) {
    m = __fmul_rn(m, 0.5f);
    e += 1;
  }
  const float sv = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
  const float z = __fmul_rn(sv, sv);
  float q = __fmaf_rn(z, 1.0f / 11.0f, 1.0f / 9.0f);
  q = __fmaf_rn(z, q, 1.0f / 7.0f);
  q = __fmaf_rn(z, q, 1.0f / 5.0f);
  q = __fmaf_rn(z, q, 1.0f / 3.0f);
  const float t = __fmul_rn(2.0f, sv);
  const float lm = __fmaf_rn(__fmul_rn(t, z), q, t);
  const float fe = (float)e;
  return __fadd_rn(__fmul_rn(fe, 0.693145751953125f), __fmaf_rn(fe, 1.42860682e-6f, lm));
}

// sin and cos of 2 pi u for u in [0,1): q = 4u (exact), n = nearest integer,
// r = q - n in [-1/2, 1/2] (exact), theta = r pi/2 in [-pi/4, pi/4], Taylor
// series to theta^9 (sine) and theta^10 (cosine), then the quadrant n.
__device__ __forceinline__ void sincos_2pi_f32(float u, float* sn, float* cs) {
  const float q = __fmul_rn(u, 4.0f);
  const int n = (int)__fadd_rn(q, 0.5f);
  const float r = __fsub_rn(q, (float)n);
  const float th = __fmul_rn(r, 1.57079637f);
  const float t2 = __fmul_rn(th, th);
  float ps = __fmaf_rn(t2, 1.0f / 362880.0f, -1.0f / 5040.0f);
  ps = __fmaf_rn(t2, ps, 1.0f / 120.0f);
  ps = __fmaf_rn(t2, ps, -1.0f / 6.0f);
  const float sv = __fmaf_rn(__fmul_rn(th, t2), ps, th);
  float pc = __fmaf_rn(t2, -1.0f / 3628800.0f, 1.0f / 40320.0f);
  pc = __fmaf_rn(t2, pc, -1.0f / 720.0f);
  pc = __fmaf_rn(t2, pc, 1.0f / 24.0f);
  pc = __fmaf_rn(t2, pc, -0.5f);
  const float cv = __fmaf_rn(t2, pc, 1.0f);
  switch (n & 3) {
    case 0: *sn = sv; *cs = cv; break;
    case 1: *sn = cv; *cs = -sv; break;
    case 2: *sn = -sv; *cs = -cv; break;
    default: *sn = -cv; *cs = sv; break;
  }
}

// ln of a Gamma(a, 1) draw in FP32 (Marsaglia and Tsang 2000).  Attempt pair
// j takes Philox block j: words x, y give two Box-Muller normals, z and w the
// two acceptance uniforms.  With y = c x, v - 1 = y (3 + y (3 + y)) is formed
// without cancellation and 1 - v + ln v = ln(1 + w) - w by its series when
// |w| < 1/8 (to w^9/9; the next term is below 3e-8 of the sum): at the
// shapes of large counts the direct form would lose ~1e-4 of the test's
// log density to cancellation.  Shape < 1: G(a) = G(a + 1) U^(1/a), U from
// block 0xFFFFFF.
static __device__ __noinline__ float log_gamma_draw_f32(float a, uint32_t e, uint32_t rep,
                                                    uint32_t stream, uint32_t key,
                                                    int* errbits) {
  const float aa = a < 1.0f ? __fadd_rn(a, 1.0f) : a;
  const float d = __fsub_rn(aa, 1.0f / 3.0f);
  const float c = __fdiv_rn(1.0f, __fsqrt_rn(__fmul_rn(9.0f, d)));
  float lg = 0.0f;
  bool done = false;
  for (uint32_t j = 0; j < kGammaMaxBlocks && !done; j++) {
    const U4 b = philox_s(e, j, rep, stream, key);
    float sn, cs;
    sincos_2pi_f32(u23c_f32(b.y), &sn, &cs);
    const float rad = __fsqrt_rn(__fmul_rn(-2.0f, ln_f32(u23c_f32(b.x))));
    const float xs[2] = {__fmul_rn(rad, cs), __fmul_rn(rad, sn)};
    const float us[2] = {u23c_f32(b.z), u23c_f32(b.w)};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (done) break;
      const float x = xs[h];
      const float y = __fmul_rn(c, x);
      if (!(__fadd_rn(1.0f, y) > 0.0f)) continue;
      const float w = __fmul_rn(y, __fmaf_rn(y, __fadd_rn(3.0f, y), 3.0f));
      const float v = __fadd_rn(1.0f, w);
      if (!(v > 1e-30f)) continue;
      const float x2 = __fmul_rn(x, x);
      const float u = us[h];
      bool acc = u < __fsub_rn(1.0f, __fmul_rn(__fmul_rn(0.0331f, x2), x2));
      if (!acc) {
        float g;
        if (fabsf(w) < 0.125f) {
          float p = __fmaf_rn(w, 1.0f / 9.0f, -0.125f);
          p = __fmaf_rn(w, p, 1.0f / 7.0f);
          p = __fmaf_rn(w, p, -1.0f / 6.0f);
          p = __fmaf_rn(w, p, 0.2f);
          p = __fmaf_rn(w, p, -0.25f);
          p = __fmaf_rn(w, p, 1.0f / 3.0f);
          p = __fmaf_rn(w, p, -0.5f);
          g = __fmul_rn(__fmul_rn(w, w), p);
        } else {
          g = __fsub_rn(ln_f32(v), w);
        }
        acc = ln_f32(u) < __fmaf_rn(d, g, __fmul_rn(0.5f, x2));
      }
      if (acc) {
        lg = ln_f32(__fmul_rn(d, v));
        done = true;
      }
    }
  }
  if (!done) {
    *errbits |= kErrGammaCap;
    lg = ln_f32(d);
  }
  if (a < 1.0f) {
    const U4 w = philox_s(e, 0xFFFFFFu, rep, stream, key);
    lg = __fadd_rn(lg, __fdiv_rn(ln_f32(u23c_f32(w.x)), a));
  }
  return lg;
}

// Butterfly over G lanes (G a power of two, width-G shuffles): every lane of
// the group ends with the same pairwise-tree value.
template <typename T>
__device__ __forceinline__ T group_sum(T v, int G) {
  for (int off = 1; off < G; off <<= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off, G);
  return v;
}
template <typename T>
__device__ __forceinline__ T group_max(T v, int G) {
  for (int off = 1; off < G; off <<= 1) {
    T o = __shfl_xor_sync(0xffffffffu, v, off, G);
    v = o > v ? o : v;
  }
  return v;
}

// Packed FP32x2 (sm_100) multiply / add / fma with explicit round-to-nearest,
// issued as PTX so the code generator never contracts a mul+add pair into an
// fma: the categorical draw needs r = round(u*T) and then C - r exactly.
__device__ __forceinline__ unsigned long long f2_bits(float2 v) {
  return ((unsigned long long)__float_as_uint(v.y) << 32) | __float_as_uint(v.x);
}
__device__ __forceinline__ float2 bits_f2(unsigned long long b) {
  return make_float2(__uint_as_float((uint32_t)b), __uint_as_float((uint32_t)(b >> 32)));
}
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(r);
}
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(r);
}
__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return bits_f2(r);
}

__device__ __forceinline__ void set_err(int* err, int bits) {
  if (bits) atomicOr(err, bits);
}

// "Last CTA" protocol for per-chain reductions: each CTA writes its partial,
// fences, and bumps a counter; the CTA that observes count == total-1 owns the
// finalisation and resets the counter for the next launch.  No spinning.
__device__ __forceinline__ bool last_cta_arrive(unsigned* ctr, unsigned total) {
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicAdd(ctr, 1u);
    s_last = (prev == total - 1) ? 1u : 0u;
    if (s_last) *ctr = 0u;
  }
  __syncthreads();
  bool last = s_last != 0u;
  if (last) __threadfence();
  return last;
}

// Binary search of the owning chain for a flat tile index.
__device__ __forceinline__ int find_chain(const int* prefix, int nchains, int t) {
  int lo = 0, hi = nchains - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace st
