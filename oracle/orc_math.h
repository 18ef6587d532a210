/*
 * Oracle-side elementary functions (test infrastructure, never shipped).
 *
 * The SIFT kernels of the reference call CUDA's expf/__expf/atan2f/cosf/sinf
 * (pysift/core.py:266-268, 757-769) and CuPy's float32 log2 for the entropy
 * threshold (pysift/core.py:1143-1146).  Their last-bit behaviour is not
 * reproducible on a CPU, so the canonical definition used by this oracle and
 * by the CUDA product is a set of elementary functions written from their
 * mathematical definitions:
 *
 *   exp   : Cody-Waite reduction x = n*ln2 + r (ln2 split in two parts),
 *           Taylor series of exp(r) to degree 8 in Horner form (fmaf),
 *           exact scaling by 2^n.
 *   atan2 : t = min(|x|,|y|)/max(|x|,|y|) in [0,1], atan(t) = t*P(t^2)
 *           with P a degree-9 polynomial (coefficients from a Chebyshev
 *           interpolation of atan(sqrt(s))/sqrt(s) on [0,1], rounded to
 *           float32; max error ~1.5 ulp), then octant/quadrant fix-up.
 *   sincos: Cody-Waite reduction by pi/2 (three float parts), Taylor series
 *           of sin (to r^9) and cos (to r^10), quadrant rotation.
 *   log2d : (double) m*2^e split with m in [sqrt(1/2), sqrt(2)),
 *           ln(m) = 2*atanh((m-1)/(m+1)) by its series to s^29.
 *
 * The CUDA side (pysift_b200/csrc/sift_math.cuh) implements the same
 * operation sequences; the oracle keeps its own copy so that a slip in either
 * shows up as a parity failure.  Compiled with -ffp-contract=off: every
 * operator below is a single IEEE-754 operation, fmaf() is an explicit fused
 * multiply-add.
 */
#ifndef ORC_MATH_H
#define ORC_MATH_H
#include <math.h>
#include <stdint.h>
#include <string.h>

static inline float orc_bits2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t orc_f2bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline double orc_bits2d(uint64_t u) { double f; memcpy(&f, &u, 8); return f; }
static inline uint64_t orc_d2bits(double f) { uint64_t u; memcpy(&u, &f, 8); return u; }

/* 2^n as a float scale, exact multiply for n >= -126, two-step below. */
static inline float orc_scale2(float p, int n) {
    if (n > 127) n = 127 + (n > 127);  /* unreachable for the SIFT weights */
    if (n >= -126) return p * orc_bits2f((uint32_t)(n + 127) << 23);
    return (p * orc_bits2f((uint32_t)(n + 64 + 127) << 23)) * orc_bits2f((uint32_t)(127 - 64) << 23);
}

static inline float orc_expf(float x) {
    if (x < -104.0f) return 0.0f;
    if (x > 88.0f) x = 88.0f;
    const float LOG2E = 1.44269504088896341f;
    const float LN2_HI = 0.693145751953125f;          /* 16 significant bits */
    const float LN2_LO = 1.42860682030941723212e-06f; /* ln2 - LN2_HI        */
    float n = rintf(x * LOG2E);
    float r = fmaf(-n, LN2_HI, x);
    r = fmaf(-n, LN2_LO, r);
    float p = 2.48015873015873015873e-05f;      /* 1/8! */
    p = fmaf(p, r, 1.98412698412698412698e-04f); /* 1/7! */
    p = fmaf(p, r, 1.38888888888888888889e-03f); /* 1/6! */
    p = fmaf(p, r, 8.33333333333333333333e-03f); /* 1/5! */
    p = fmaf(p, r, 4.16666666666666666667e-02f); /* 1/4! */
    p = fmaf(p, r, 1.66666666666666666667e-01f); /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return orc_scale2(p, (int)n);
}

#define ORC_PI_F   3.14159265358979323846f
#define ORC_PIO2_F 1.57079632679489661923f
#define ORC_PIO4_F 0.78539816339744830962f

static inline float orc_atan2f(float y, float x) {
    float ax = fabsf(x), ay = fabsf(y);
    if (ax == 0.0f && ay == 0.0f) {
        float a = signbit(x) ? ORC_PI_F : 0.0f;
        return signbit(y) ? -a : a;
    }
    int swap = ay > ax;
    float mn = swap ? ax : ay;
    float mx = swap ? ay : ax;
    float t = mn / mx;
    float s = t * t;
    float p = -0x1.c919cep-10f;
    p = fmaf(p, s, 0x1.5dfc5ep-7f);
    p = fmaf(p, s, -0x1.f74692p-6f);
    p = fmaf(p, s, 0x1.d6bdd0p-5f);
    p = fmaf(p, s, -0x1.56eb74p-4f);
    p = fmaf(p, s, 0x1.c01c4cp-4f);
    p = fmaf(p, s, -0x1.2413b8p-3f);
    p = fmaf(p, s, 0x1.999052p-3f);
    p = fmaf(p, s, -0x1.555534p-2f);
    p = fmaf(p, s, 0x1.000000p+0f);
    float a = t * p;
    if (swap) a = ORC_PIO2_F - a;
    if (signbit(x)) a = ORC_PI_F - a;
    if (signbit(y)) a = -a;
    return a;
}

static inline void orc_sincosf(float x, float* s, float* c) {
    const float TWO_OVER_PI = 0.636619772367581343076f;
    const float P1 = 1.5703125f;                          /* 8 significant bits  */
    const float P2 = 4.83751296997070312500e-04f;         /* next 17 bits        */
    const float P3 = 7.54978995489188216e-08f;            /* remainder of pi/2   */
    float j = rintf(x * TWO_OVER_PI);
    float r = fmaf(-j, P1, x);
    r = fmaf(-j, P2, r);
    r = fmaf(-j, P3, r);
    float r2 = r * r;
    float ps = 2.75573192239858906526e-06f;           /*  1/9!  */
    ps = fmaf(ps, r2, -1.98412698412698412698e-04f);  /* -1/7!  */
    ps = fmaf(ps, r2, 8.33333333333333333333e-03f);   /*  1/5!  */
    ps = fmaf(ps, r2, -1.66666666666666666667e-01f);  /* -1/3!  */
    float sr = fmaf(r * r2, ps, r);
    float pc = -2.75573192239858906526e-07f;          /* -1/10! */
    pc = fmaf(pc, r2, 2.48015873015873015873e-05f);   /*  1/8!  */
    pc = fmaf(pc, r2, -1.38888888888888888889e-03f);  /* -1/6!  */
    pc = fmaf(pc, r2, 4.16666666666666666667e-02f);   /*  1/4!  */
    pc = fmaf(pc, r2, -0.5f);
    float cr = fmaf(r2, pc, 1.0f);
    int q = ((int)j) & 3;
    switch (q) {
        case 0: *s = sr;  *c = cr;  break;
        case 1: *s = cr;  *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

/* log2 of a positive normal double. */
static inline double orc_log2d(double p) {
    uint64_t b = orc_d2bits(p);
    int e = (int)((b >> 52) & 0x7ff) - 1022;            /* p = m * 2^e, m in [0.5,1) */
    double m = orc_bits2d((b & 0x000fffffffffffffULL) | 0x3fe0000000000000ULL);
    if (m < 0.70710678118654752440) { m = m * 2.0; e = e - 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    double t = 1.0 / 29.0;
    for (int k = 27; k >= 3; k -= 2) t = t * s2 + 1.0 / (double)k;
    t = t * s2 + 1.0;
    double ln_m = 2.0 * (s * t);
    return (double)e + ln_m * 1.44269504088896340736;
}

#endif
