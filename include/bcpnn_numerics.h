/*
 * bcpnn_numerics.h -- the numerics contract shared by the sm_100a kernels and
 * by any CPU code that must replay them bit for bit.
 *
 * Two things live here:
 *
 *  1. Philox4x32-10, the counter-based generator of Salmon, Moraes, Dror and
 *     Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11), and the
 *     fixed map from (seed, population, stream, tick, MCU) to the uniform and
 *     normal numbers that replace gsbn's `Random` class
 *     (src/gsbn/Random.cpp:27-63, seeded from std::random_device and so never
 *     replayable).
 *
 *  2. bx_expf / bx_logf: float exp and log written with IEEE-754 basic
 *     operations only (+, -, *, /, exact conversions and bit moves).  Every
 *     such operation is correctly rounded on x86-64 SSE and on the GPU, so a
 *     host and a device evaluation of the same expression give the same bits,
 *     provided no fused multiply-add is formed (compile host code with
 *     -ffp-contract=off and device code with -fmad=false).  gsbn evaluates
 *     std::exp(float)/std::log(float) (glibc expf/logf) on the CPU and CUDA
 *     expf/logf on the GPU; those two differ in the last bit and make CPU and
 *     GPU spike trains diverge.  These are evaluated in float (they sit on
 *     the per-cell path of the kernels) and stay within 2 ulp of the
 *     correctly rounded result (tests/test_numerics.py measures it).
 *     Double-precision versions (bx_exp_d, bx_log_d) serve host-side
 *     initial values and the Box-Muller transform.
 *
 *     Methods (textbook, no vendor code):
 *       exp: Cody & Waite additive range reduction x = k ln2 + r with a
 *            two-part ln2, |r| <= ln2/2, Taylor polynomial of e^r in Horner
 *            form, exact scaling by 2^k in two steps (W. J. Cody, W. Waite,
 *            "Software Manual for the Elementary Functions", 1980, ch. 6).
 *       log: x = 2^e m with m in [sqrt(2)/2, sqrt(2)), log m = 2 atanh(s),
 *            s = (m-1)/(m+1), odd power series of atanh (Abramowitz &
 *            Stegun 4.1.27 / 4.6.22), e ln2 added with a two-part ln2.
 *       cos(2 pi u): reduction to [-pi/2, pi/2] by symmetry and an even
 *            Taylor series to x^26.
 *     All coefficients are exact values of 1/n!, 2/(2n+1) and 1/(2n+1)
 *     rounded to the working precision, written as hexadecimal literals.
 */
#ifndef BCPNN_NUMERICS_H
#define BCPNN_NUMERICS_H

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define BX_HD __host__ __device__ __forceinline__
#else
#define BX_HD static inline
#endif

#ifdef __cplusplus
extern "C++" {
#endif

/* ------------------------------------------------------------------------ */
/* bit moves                                                                 */
/* ------------------------------------------------------------------------ */

BX_HD uint64_t bx_dbits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  union { double d; uint64_t u; } v; v.d = x; return v.u;
#endif
}

BX_HD double bx_bitsd(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  union { double d; uint64_t u; } v; v.u = u; return v.d;
#endif
}

BX_HD uint32_t bx_fbits(float x) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)__float_as_uint(x);
#else
  union { float f; uint32_t u; } v; v.f = x; return v.u;
#endif
}

BX_HD float bx_bitsf(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  union { float f; uint32_t u; } v; v.u = u; return v.f;
#endif
}

/* floor of a double known to be in (-2^52, 2^52), from exact operations.  */
BX_HD double bx_floor_d(double x) {
  /* truncation toward zero by an exact conversion, then step down for
     negative non-integers */
  double t = (double)(long long)x;
  return (t > x) ? t - 1.0 : t;
}

/* ------------------------------------------------------------------------ */
/* exp                                                                       */
/* ------------------------------------------------------------------------ */

/* e^x for |x| <= ~745, evaluated in double; caller guarantees the range.   */
BX_HD double bx_exp_d(double x) {
  const double INV_LN2 = 0x1.71547652b82fep+0;
  const double LN2_HI = 0x1.62e42fee00000p-1; /* 31 significant bits: k*LN2_HI exact for |k| < 2^22 */
  const double LN2_LO = 0x1.a39ef35793c76p-33;
  double kd = bx_floor_d(x * INV_LN2 + 0.5);
  double r = (x - kd * LN2_HI) - kd * LN2_LO;
  /* Taylor series of e^r, |r| <= 0.3466 + tiny; truncation error < 3e-19 */
  double p = 0x1.93974a8c07c9dp-37;          /* 1/14! */
  p = p * r + 0x1.6124613a86d09p-33;         /* 1/13! */
  p = p * r + 0x1.1eed8eff8d898p-29;         /* 1/12! */
  p = p * r + 0x1.ae64567f544e4p-26;         /* 1/11! */
  p = p * r + 0x1.27e4fb7789f5cp-22;         /* 1/10! */
  p = p * r + 0x1.71de3a556c734p-19;         /* 1/9!  */
  p = p * r + 0x1.a01a01a01a01ap-16;         /* 1/8!  */
  p = p * r + 0x1.a01a01a01a01ap-13;         /* 1/7!  */
  p = p * r + 0x1.6c16c16c16c17p-10;         /* 1/6!  */
  p = p * r + 0x1.1111111111111p-7;          /* 1/5!  */
  p = p * r + 0x1.5555555555555p-5;          /* 1/4!  */
  p = p * r + 0x1.5555555555555p-3;          /* 1/3!  */
  p = p * r + 0.5;                           /* 1/2!  */
  p = p * r + 1.0;
  p = p * r + 1.0;
  /* scale by 2^k in two exact steps so that k down to -1074 stays normal
     until the last multiplication */
  long long k = (long long)kd;
  long long k1 = k / 2, k2 = k - k1;
  double s1 = bx_bitsd((uint64_t)(k1 + 1023) << 52);
  double s2 = bx_bitsd((uint64_t)(k2 + 1023) << 52);
  return (p * s1) * s2;
}

/* float exp (see header comment): e^x = 2^k e^r, k = rint(x log2 e).
   Branch-free: out-of-range inputs are clamped for the computation and the
   special results selected at the end, so independent calls can overlap. */
BX_HD float bx_expf(float x) {
  const float LOG2E = 0x1.715476p+0f;
  const float LN2_HI = 0x1.62e4p-1f;                 /* 16 significant bits: k*LN2_HI exact for |k| <= 256 */
  const float LN2_LO = 0x1.7f7d1cp-20f;
  const float SHIFT = 0x1.8p23f;                     /* adding and removing it rounds to an integer */
  float xc = x < -104.0f ? -104.0f : x;
  xc = xc > 89.0f ? 89.0f : xc;
  xc = (x != x) ? 0.0f : xc;
  float t = xc * LOG2E + SHIFT;
  float kf = t - SHIFT;
  float r = (xc - kf * LN2_HI) - kf * LN2_LO;        /* |r| <= ln2/2 + 2^-20 */
  float p = 0x1.a01a02p-16f;                         /* 1/8! */
  p = p * r + 0x1.a01a02p-13f;                       /* 1/7! */
  p = p * r + 0x1.6c16c2p-10f;                       /* 1/6! */
  p = p * r + 0x1.111112p-7f;                        /* 1/5! */
  p = p * r + 0x1.555556p-5f;                        /* 1/4! */
  p = p * r + 0x1.555556p-3f;                        /* 1/3! */
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  int k = (int)(bx_fbits(t) - 0x4B400000u);          /* kf as an integer, in [-151, 129] */
  int k1 = k >> 1, k2 = k - k1;                      /* both in [-76, 65]: normal powers of two */
  float s1 = bx_bitsf((uint32_t)(k1 + 127) << 23);
  float s2 = bx_bitsf((uint32_t)(k2 + 127) << 23);
  float res = (p * s1) * s2;                         /* exact, then one rounding (subnormal or overflow) */
  res = x > 89.0f ? bx_bitsf(0x7f800000u) : res;     /* +inf */
  res = x < -104.0f ? 0.0f : res;                    /* below half the least subnormal */
  return (x != x) ? x : res;                         /* NaN */
}

/* ------------------------------------------------------------------------ */
/* log                                                                       */
/* ------------------------------------------------------------------------ */

/* natural log of a positive, finite, normal double. */
BX_HD double bx_log_d(double x) {
  const double LN2_HI = 0x1.62e42fee00000p-1;
  const double LN2_LO = 0x1.a39ef35793c76p-33;
  const double SQRT2 = 0x1.6a09e667f3bcdp+0;
  uint64_t b = bx_dbits(x);
  long long e = (long long)((b >> 52) & 0x7ff) - 1023;
  double m = bx_bitsd((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull); /* [1,2) */
  if (m > SQRT2) { m = m * 0.5; e = e + 1; }
  double s = (m - 1.0) / (m + 1.0);
  double z = s * s;
  double p = 0x1.2f684bda12f68p-5;           /* 1/27 */
  p = p * z + 0x1.47ae147ae147bp-5;          /* 1/25 */
  p = p * z + 0x1.642c8590b2164p-5;          /* 1/23 */
  p = p * z + 0x1.8618618618618p-5;          /* 1/21 */
  p = p * z + 0x1.af286bca1af28p-5;          /* 1/19 */
  p = p * z + 0x1.e1e1e1e1e1e1ep-5;          /* 1/17 */
  p = p * z + 0x1.1111111111111p-4;          /* 1/15 */
  p = p * z + 0x1.3b13b13b13b14p-4;          /* 1/13 */
  p = p * z + 0x1.745d1745d1746p-4;          /* 1/11 */
  p = p * z + 0x1.c71c71c71c71cp-4;          /* 1/9  */
  p = p * z + 0x1.2492492492492p-3;          /* 1/7  */
  p = p * z + 0x1.999999999999ap-3;          /* 1/5  */
  p = p * z + 0x1.5555555555555p-2;          /* 1/3  */
  double lm = (2.0 * s) + (2.0 * s) * (z * p);
  double ed = (double)e;
  return ed * LN2_HI + (ed * LN2_LO + lm);
}

/* float log (see header comment).  Branch-free like bx_expf. */
BX_HD float bx_logf(float x) {
  const float LN2_HI = 0x1.62e4p-1f;
  const float LN2_LO = 0x1.7f7d1cp-20f;
  const float SQRT2 = 0x1.6a09e6p+0f;
  const bool sub = x < 0x1p-126f;                           /* subnormal (or non-positive) */
  float xs = sub ? x * 0x1p23f : x;                          /* scale subnormals into the normal range */
  uint32_t b = bx_fbits(xs);
  int e = (int)((b >> 23) & 0xffu) - 127 - (sub ? 23 : 0);
  float m = bx_bitsf((b & 0x007fffffu) | 0x3f800000u);      /* [1, 2) */
  const bool hi = m > SQRT2;
  m = hi ? m * 0.5f : m;
  e = hi ? e + 1 : e;
  float s = (m - 1.0f) / (m + 1.0f);                         /* |s| <= 0.1716 */
  float z = s * s;
  float p = 0x1.745d18p-3f;                                  /* 2/11 */
  p = p * z + 0x1.c71c72p-3f;                                /* 2/9 */
  p = p * z + 0x1.24924ap-2f;                                /* 2/7 */
  p = p * z + 0x1.99999ap-2f;                                /* 2/5 */
  p = p * z + 0x1.555556p-1f;                                /* 2/3 */
  float lm = (s + s) + (s * z) * p;
  float ef = (float)e;
  float res = ef * LN2_HI + (ef * LN2_LO + lm);
  res = (bx_fbits(x) == 0x7f800000u) ? x : res;              /* +inf */
  res = (x == 0.0f) ? bx_bitsf(0xff800000u) : res;           /* -inf */
  res = (x < 0.0f) ? bx_bitsf(0x7fc00000u) : res;            /* NaN */
  return (x != x) ? x : res;                                 /* NaN */
}

/* ------------------------------------------------------------------------ */
/* cos(2 pi u) for Box-Muller                                                */
/* ------------------------------------------------------------------------ */

BX_HD double bx_cos2pi_d(double u) {
  const double TWO_PI = 0x1.921fb54442d18p+2;
  double a = u - bx_floor_d(u + 0.5);       /* [-0.5, 0.5) , cos even */
  if (a < 0.0) a = -a;                      /* [0, 0.5] */
  double sign = 1.0;
  if (a > 0.25) { a = 0.5 - a; sign = -1.0; } /* cos(pi - y) = -cos(y) */
  double x = a * TWO_PI;                    /* [0, pi/2] */
  double z = x * x;
  /* cos x = sum (-1)^n x^(2n)/(2n)!, to x^26, Horner in z = x^2 */
  double p = -0x1.88e85fc6a4e5ap-89;         /* -1/26! */
  p = p * z + 0x1.f2cf01972f578p-80;         /*  1/24! */
  p = p * z - 0x1.0ce396db7f853p-70;         /* -1/22! */
  p = p * z + 0x1.e542ba4020225p-62;         /*  1/20! */
  p = p * z - 0x1.6827863b97d97p-53;         /* -1/18! */
  p = p * z + 0x1.ae7f3e733b81fp-45;         /*  1/16! */
  p = p * z - 0x1.93974a8c07c9dp-37;         /* -1/14! */
  p = p * z + 0x1.1eed8eff8d898p-29;         /*  1/12! */
  p = p * z - 0x1.27e4fb7789f5cp-22;         /* -1/10! */
  p = p * z + 0x1.a01a01a01a01ap-16;         /*  1/8!  */
  p = p * z - 0x1.6c16c16c16c17p-10;         /* -1/6!  */
  p = p * z + 0x1.5555555555555p-5;          /*  1/4!  */
  p = p * z - 0.5;                           /* -1/2!  */
  double r = 1.0 + z * p;
  return sign * r;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                             */
/* ------------------------------------------------------------------------ */

typedef struct { uint32_t v[4]; } bx_u32x4;

BX_HD void bx_mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds: counter c[0..3], key k0, k1 (SC'11, table 2:
   multipliers 0xD2511F53, 0xCD9E8D57; Weyl key increments 0x9E3779B9,
   0xBB67AE85). */
BX_HD bx_u32x4 bx_philox4x32_10(bx_u32x4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint32_t hi0, lo0, hi1, lo1;
    bx_mulhilo32(0xD2511F53u, c.v[0], &hi0, &lo0);
    bx_mulhilo32(0xCD9E8D57u, c.v[2], &hi1, &lo1);
    bx_u32x4 o;
    o.v[0] = hi1 ^ c.v[1] ^ k0;
    o.v[1] = lo1;
    o.v[2] = hi0 ^ c.v[3] ^ k1;
    o.v[3] = lo0;
    c = o;
  }
  return c;
}

/* Stream identifiers (key word 1 = pop_id * 16 + stream). */
enum {
  BX_STREAM_UNIFORM = 0, /* spike sampling u < act * maxfq * dt            */
  BX_STREAM_NORMAL = 1,  /* support noise N(0, snoise), Box-Muller          */
  BX_STREAM_POISSON = 2  /* project-defined Poisson input noise spikes      */
};

/* Raw 32-bit lane for (seed, pop, stream, tick, mcu, block).  One Philox call
   covers four consecutive MCUs; lane = mcu & 3.                             */
BX_HD uint32_t bx_rng_lane(uint32_t seed, uint32_t pop, uint32_t stream,
                           uint32_t tick, uint32_t mcu, uint32_t block) {
  bx_u32x4 c;
  c.v[0] = mcu >> 2;
  c.v[1] = tick;
  c.v[2] = block;
  c.v[3] = 0u;
  bx_u32x4 o = bx_philox4x32_10(c, seed, pop * 16u + stream);
  return o.v[mcu & 3u];
}

/* Uniform float in [0, 1): top 24 bits times 2^-24 (exact). */
BX_HD float bx_u01(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

/* Uniform for spike sampling of MCU `mcu` of population `pop` at `tick`. */
BX_HD float bx_uniform01(uint32_t seed, uint32_t pop, uint32_t tick, uint32_t mcu) {
  return bx_u01(bx_rng_lane(seed, pop, BX_STREAM_UNIFORM, tick, mcu, 0u));
}

/* Uniform for the Poisson input-noise spike of MCU `mcu`. */
BX_HD float bx_uniform01_poisson(uint32_t seed, uint32_t pop, uint32_t tick, uint32_t mcu) {
  return bx_u01(bx_rng_lane(seed, pop, BX_STREAM_POISSON, tick, mcu, 0u));
}

/* Standard normal by Box-Muller from two lanes (blocks 0 and 1):
   u1 in (0, 1], u2 in [0, 1), z = sqrt(-2 ln u1) cos(2 pi u2), rounded to
   float once. */
BX_HD float bx_normal01(uint32_t seed, uint32_t pop, uint32_t tick, uint32_t mcu) {
  uint32_t a = bx_rng_lane(seed, pop, BX_STREAM_NORMAL, tick, mcu, 0u);
  uint32_t b = bx_rng_lane(seed, pop, BX_STREAM_NORMAL, tick, mcu, 1u);
  double u1 = (double)((a >> 8) + 1u) * 0x1p-24;
  double u2 = (double)(b >> 8) * 0x1p-24;
  double rr = -2.0 * bx_log_d(u1);
#if defined(__CUDA_ARCH__)
  double rad = __dsqrt_rn(rr);
#else
  double rad = __builtin_sqrt(rr);
#endif
  return (float)(rad * bx_cos2pi_d(u2));
}

/* ------------------------------------------------------------------------ */
/* ProcExtGen's stimulus values                                              */
/* ------------------------------------------------------------------------ */

/* log(1+eps) and log(0+eps), the two lginp values (ProcExtGen.cpp:130-144).
   gsbn computes them on the host with the C library's float log in every
   mode, so host code here calls the same function and the stimulus rows are
   gsbn's bit for bit.  Host only. */
#if defined(__CUDACC__)
static inline __host__ float bx_extgen_logf(float x) { return logf(x); }
#else
static inline float bx_extgen_logf(float x) { return logf(x); }
#endif

#ifdef __cplusplus
}
#endif

#endif /* BCPNN_NUMERICS_H */
