// Device elementary functions for the SIFT kernels.
//
// The reference's kernels call CUDA's atan2f/expf/__expf/cosf/sinf
// (pysift/core.py:266-268, 757-769) and CuPy's float32 log2
// (pysift/core.py:1143-1146).  To make every stage reproducible bit for bit
// by a CPU restatement, this library defines its own elementary functions
// from their mathematical definitions:
//
//   sm_expf   Cody-Waite reduction x = n*ln2 + r (ln2 split in a 16-bit head
//             and a tail), Taylor series of exp(r) to degree 8 (Horner/fmaf),
//             exact power-of-two scaling.
//   sm_atan2f t = min(|x|,|y|)/max(|x|,|y|) in [0,1], atan(t) = t*P(t^2) with
//             P of degree 9 (coefficients from a Chebyshev interpolation of
//             atan(sqrt(s))/sqrt(s) on [0,1], rounded to float32; max error
//             ~1.5 ulp), then octant/quadrant fix-up from the operand signs.
//   sm_sincosf Cody-Waite reduction by pi/2 in three float parts (the split
//             used by the Cephes library), Taylor series of sin to r^9 and
//             cos to r^10, quadrant rotation.
//   sm_log2d  (double) m*2^e with m in [sqrt(1/2), sqrt(2)),
//             ln m = 2 atanh((m-1)/(m+1)) by its series to s^29.
//
// The library is compiled with --fmad=false, so every operator below is one
// IEEE-754 operation and fmaf() is the only fused multiply-add.
#pragma once
#include <cstdint>

namespace sm {

__device__ __forceinline__ float scale2(float p, int n) {
    if (n >= -126) return p * __uint_as_float((uint32_t)(n + 127) << 23);
    return (p * __uint_as_float((uint32_t)(n + 64 + 127) << 23)) * __uint_as_float((uint32_t)(127 - 64) << 23);
}

__device__ __forceinline__ float expf_(float x) {
    if (x < -104.0f) return 0.0f;
    if (x > 88.0f) x = 88.0f;
    const float LOG2E = 1.44269504088896341f;
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860682030941723212e-06f;
    float n = rintf(x * LOG2E);
    float r = fmaf(-n, LN2_HI, x);
    r = fmaf(-n, LN2_LO, r);
    float p = 2.48015873015873015873e-05f;
    p = fmaf(p, r, 1.98412698412698412698e-04f);
    p = fmaf(p, r, 1.38888888888888888889e-03f);
    p = fmaf(p, r, 8.33333333333333333333e-03f);
    p = fmaf(p, r, 4.16666666666666666667e-02f);
    p = fmaf(p, r, 1.66666666666666666667e-01f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return scale2(p, (int)n);
}

constexpr float PI_F = 3.14159265358979323846f;
constexpr float PIO2_F = 1.57079632679489661923f;
constexpr float PIO4_F = 0.78539816339744830962f;

__device__ __forceinline__ float atan2f_(float y, float x) {
    float ax = fabsf(x), ay = fabsf(y);
    if (ax == 0.0f && ay == 0.0f) {
        float a = signbit(x) ? PI_F : 0.0f;
        return signbit(y) ? -a : a;
    }
    const bool swap = ay > ax;
    const float mn = swap ? ax : ay;
    const float mx = swap ? ay : ax;
    const float t = mn / mx;
    const float s = t * t;
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
    if (swap) a = PIO2_F - a;
    if (signbit(x)) a = PI_F - a;
    if (signbit(y)) a = -a;
    return a;
}

__device__ __forceinline__ void sincosf_(float x, float* s, float* c) {
    const float TWO_OVER_PI = 0.636619772367581343076f;
    const float P1 = 1.5703125f;
    const float P2 = 4.83751296997070312500e-04f;
    const float P3 = 7.54978995489188216e-08f;
    float j = rintf(x * TWO_OVER_PI);
    float r = fmaf(-j, P1, x);
    r = fmaf(-j, P2, r);
    r = fmaf(-j, P3, r);
    float r2 = r * r;
    float ps = 2.75573192239858906526e-06f;
    ps = fmaf(ps, r2, -1.98412698412698412698e-04f);
    ps = fmaf(ps, r2, 8.33333333333333333333e-03f);
    ps = fmaf(ps, r2, -1.66666666666666666667e-01f);
    float sr = fmaf(r * r2, ps, r);
    float pc = -2.75573192239858906526e-07f;
    pc = fmaf(pc, r2, 2.48015873015873015873e-05f);
    pc = fmaf(pc, r2, -1.38888888888888888889e-03f);
    pc = fmaf(pc, r2, 4.16666666666666666667e-02f);
    pc = fmaf(pc, r2, -0.5f);
    float cr = fmaf(r2, pc, 1.0f);
    int q = ((int)j) & 3;
    if (q == 0) { *s = sr; *c = cr; }
    else if (q == 1) { *s = cr; *c = -sr; }
    else if (q == 2) { *s = -sr; *c = -cr; }
    else { *s = -cr; *c = sr; }
}

__device__ __forceinline__ double log2d_(double p) {
    uint64_t b = (uint64_t)__double_as_longlong(p);
    int e = (int)((b >> 52) & 0x7ff) - 1022;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffULL) | 0x3fe0000000000000ULL));
    if (m < 0.70710678118654752440) { m = m * 2.0; e = e - 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    double t = 1.0 / 29.0;
    for (int k = 27; k >= 3; k -= 2) t = t * s2 + 1.0 / (double)k;
    t = t * s2 + 1.0;
    double ln_m = 2.0 * (s * t);
    return (double)e + ln_m * 1.44269504088896340736;
}

}  // namespace sm
