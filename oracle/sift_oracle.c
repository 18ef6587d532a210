/*
 * sift_oracle.c -- CPU restatement of PySIFT's SIFT hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this file; the parity tests, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py use it as the checker.
 *
 * Every routine cites the reference code it restates (paths relative to the
 * reference project).  Where the reference is order-dependent or uses
 * approximate arithmetic, the canonical choice shared with the CUDA product
 * is stated in the routine's comment:
 *   - no implicit FMA contraction (compiled with -ffp-contract=off); the
 *     separable blur keeps the reference's FMA chain explicitly (fmaf);
 *   - IEEE division / sqrt where the reference uses fast-math or rsqrtf;
 *   - elementary functions from orc_math.h;
 *   - candidate order (octave, s, r, c) instead of atomic-slot order;
 *   - orientation and descriptor histograms summed exactly in 64-bit fixed
 *     point (2^-40 units), independent of summation order, instead of the
 *     reference's per-lane float sums / shared-memory float atomics.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "orc_math.h"

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* A1: entropy-adaptive contrast threshold (pysift/core.py:1129-1148).   */
/* Canonical: float64 entropy summed in bin order with orc_log2d.        */
/* ------------------------------------------------------------------ */
EXPORT double orc_contrast_thresh(const uint8_t* img, long n, double base) {
    long hist[256];
    memset(hist, 0, sizeof(hist));
    for (long i = 0; i < n; ++i) hist[img[i]]++;
    double total = (double)n;
    double ent = 0.0;
    for (int b = 0; b < 256; ++b) {
        if (hist[b] == 0) continue;
        double p = (double)hist[b] / total;
        ent = ent + p * orc_log2d(p);
    }
    ent = -ent;
    double scale = 0.8 + ent / 40.0;
    if (scale > 1.0) scale = 1.0;
    return base * scale;
}

/* ------------------------------------------------------------------ */
/* A2: u8 -> float base image (pysift/core.py:1248-1261): u/255 in f32. */
/* ------------------------------------------------------------------ */
EXPORT void orc_u8_to_f32(const uint8_t* img, long n, float* out) {
    for (long i = 0; i < n; ++i) out[i] = (float)img[i] / 255.0f;
}

/* ------------------------------------------------------------------ */
/* A3: 2x cubic B-spline zoom, scipy.ndimage.zoom(order=3,               */
/* mode='constant', grid_mode=False) semantics as called through cupyx   */
/* at pysift/core.py:1270-1275.  Prefilter in float64 with mirror        */
/* boundary (pole sqrt(3)-2, gain 6), interpolation in float64, output  */
/* rounded to float32.                                                   */
/* ------------------------------------------------------------------ */
/* B-spline direct transform as a symmetric FIR: the impulse response of the
 * cubic-spline prefilter on the mirror-extended line is
 * h[k] = (-6 z / (1 - z^2)) z^|k|, z = sqrt(3) - 2 (h[0] = sqrt(3)); it is
 * truncated at |k| <= 30 (|z|^31 < 2e-18).  Taps are applied k = -30..30 in
 * order with one fma each, over whole-sample-symmetric (mirror) extension. */
#define ORC_SPL_K 30
static void spline_taps(double h[2 * ORC_SPL_K + 1]) {
    const double z = sqrt(3.0) - 2.0;
    const double c0 = -6.0 * z / (1.0 - z * z);
    for (int k = -ORC_SPL_K; k <= ORC_SPL_K; ++k) {
        int a = k < 0 ? -k : k;
        double zk = 1.0;
        for (int i = 0; i < a; ++i) zk = zk * z;
        h[k + ORC_SPL_K] = c0 * zk;
    }
}

static long mirror_index(long idx, long len);

static void spline_prefilter_1d(const double* in, double* out, long n, long stride, const double* h) {
    for (long i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int k = -ORC_SPL_K; k <= ORC_SPL_K; ++k)
            acc = fma(h[k + ORC_SPL_K], in[mirror_index(i + k, n) * stride], acc);
        out[i * stride] = acc;
    }
}

EXPORT void orc_spline_prefilter_2d(double* c, int H, int W) {
    /* axis 0 (along columns) first, then axis 1 (along rows), as scipy */
    double h[2 * ORC_SPL_K + 1];
    spline_taps(h);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)H * W);
    #pragma omp parallel for schedule(static)
    for (int x = 0; x < W; ++x) spline_prefilter_1d(c + x, tmp + x, H, W, h);
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < H; ++r) spline_prefilter_1d(tmp + (long)r * W, c + (long)r * W, W, 1, h);
    free(tmp);
}

static void cubic_weights(double t, double w[4]) {
    /* t in [0,1): distance from the support point floor(x) */
    double y = t;
    double z = 1.0 - y;
    w[0] = z * z * z / 6.0;
    w[1] = (y * y * (y - 2.0) * 3.0 + 4.0) / 6.0;
    double y1 = 1.0 - y;
    w[2] = (y1 * y1 * (y1 - 2.0) * 3.0 + 4.0) / 6.0;
    w[3] = 1.0 - w[0] - w[1] - w[2];
}

static long mirror_index(long idx, long len) {
    if (len <= 1) return 0;
    long s2 = 2 * len - 2;
    if (idx < 0) {
        idx = s2 * (long)(-idx / s2) + idx;
        idx = idx <= 1 - len ? idx + s2 : -idx;
    } else if (idx >= len) {
        idx -= s2 * (long)(idx / s2);
        if (idx >= len) idx = s2 - idx;
    }
    return idx;
}

/* Coordinate setup for one axis: start index (mirror-mapped support) and
 * weights; valid=0 marks coordinates outside [0, len-1] (cval = 0). */
EXPORT void orc_zoom_axis(long in_len, long out_len, long* idx4, double* w4, int* valid) {
    double zoom = (out_len > 1) ? (double)(in_len - 1) / (double)(out_len - 1) : 1.0;
    for (long k = 0; k < out_len; ++k) {
        double cc = (double)k * zoom;
        if (cc < 0.0 || cc > (double)(in_len - 1)) { valid[k] = 0; continue; }
        valid[k] = 1;
        double fl = floor(cc);
        long start = (long)fl - 1;
        cubic_weights(cc - fl, w4 + 4 * k);
        for (int h = 0; h < 4; ++h) idx4[4 * k + h] = mirror_index(start + h, in_len);
    }
}

EXPORT void orc_zoom2x(const float* in, int H, int W, float* out) {
    int OH = 2 * H, OW = 2 * W;
    double* c = (double*)malloc(sizeof(double) * (size_t)H * W);
    for (long i = 0; i < (long)H * W; ++i) c[i] = (double)in[i];
    orc_spline_prefilter_2d(c, H, W);
    long* iy = (long*)malloc(sizeof(long) * 4 * OH);
    long* ix = (long*)malloc(sizeof(long) * 4 * OW);
    double* wy = (double*)malloc(sizeof(double) * 4 * OH);
    double* wx = (double*)malloc(sizeof(double) * 4 * OW);
    int* vy = (int*)malloc(sizeof(int) * OH);
    int* vx = (int*)malloc(sizeof(int) * OW);
    orc_zoom_axis(H, OH, iy, wy, vy);
    orc_zoom_axis(W, OW, ix, wx, vx);
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < OH; ++r) {
        for (int x = 0; x < OW; ++x) {
            if (!vy[r] || !vx[x]) { out[(long)r * OW + x] = 0.0f; continue; }
            double t = 0.0;
            for (int i = 0; i < 4; ++i) {
                const double* row = c + iy[4 * r + i] * (long)W;
                for (int j = 0; j < 4; ++j) {
                    double coeff = row[ix[4 * x + j]];
                    coeff *= wy[4 * r + i];
                    coeff *= wx[4 * x + j];
                    t += coeff;
                }
            }
            out[(long)r * OW + x] = (float)t;
        }
    }
    free(c); free(iy); free(ix); free(wy); free(wx); free(vy); free(vx);
}

/* ------------------------------------------------------------------ */
/* A4: separable Gaussian blur (pysift/core.py:475-608).                 */
/* Horizontal pass then vertical pass, each a sequential FMA chain over  */
/* k = 0..2r starting from 0 (the reference's `sum += tile*kern` as nvcc */
/* contracts it), half-sample-symmetric reflect boundary.                */
/* ------------------------------------------------------------------ */
static inline int reflect_idx(int i, int n) {
    int p = 2 * n;
    i = i % p;
    if (i < 0) i += p;
    if (i >= n) i = 2 * n - 1 - i;
    return i;
}

EXPORT void orc_gauss_blur(const float* in, float* out, int H, int W, const float* kern, int radius) {
    float* tmp = (float*)malloc(sizeof(float) * (size_t)H * W);
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < H; ++r) {
        for (int c = 0; c < W; ++c) {
            float sum = 0.0f;
            for (int k = 0; k <= 2 * radius; ++k)
                sum = fmaf(in[(long)r * W + reflect_idx(c - radius + k, W)], kern[k], sum);
            tmp[(long)r * W + c] = sum;
        }
    }
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < H; ++r) {
        for (int c = 0; c < W; ++c) {
            float sum = 0.0f;
            for (int k = 0; k <= 2 * radius; ++k)
                sum = fmaf(tmp[(long)reflect_idx(r - radius + k, H) * W + c], kern[k], sum);
            out[(long)r * W + c] = sum;
        }
    }
    free(tmp);
}

/* ------------------------------------------------------------------ */
/* A7: 26-neighbour extrema with contrast gate (pysift/core.py:176-217,  */
/* 1367-1460).  dog is (S2,H,W).  Canonical order (s, r, c); the first   */
/* max_cands are kept (the reference keeps the first by atomic slot).    */
/* Returns the number of extrema found (before truncation).              */
/* ------------------------------------------------------------------ */
EXPORT long orc_find_extrema(const float* dog, int S2, int H, int W, float thresh, int border,
                             int max_cands, int* coords) {
    long found = 0;
    long HW = (long)H * W;
    for (int s = 1; s < S2 - 1; ++s) {
        for (int r = border; r < H - border; ++r) {
            for (int c = border; c < W - border; ++c) {
                float v = dog[s * HW + (long)r * W + c];
                if (fabsf(v) <= thresh) continue;
                int is_max = 1, is_min = 1;
                for (int ds = -1; ds <= 1 && (is_max || is_min); ++ds)
                    for (int dr = -1; dr <= 1; ++dr)
                        for (int dc = -1; dc <= 1; ++dc) {
                            if (ds == 0 && dr == 0 && dc == 0) continue;
                            float nb = dog[(s + ds) * HW + (long)(r + dr) * W + (c + dc)];
                            is_max = is_max && (v >= nb);
                            is_min = is_min && (v <= nb);
                        }
                if (is_max || is_min) {
                    if (found < max_cands) {
                        coords[found * 3 + 0] = s;
                        coords[found * 3 + 1] = r;
                        coords[found * 3 + 2] = c;
                    }
                    found++;
                }
            }
        }
    }
    return found;
}

/* ------------------------------------------------------------------ */
/* A8: Taylor refinement + contrast + edge test (pysift/core.py:343-463, */
/* 1462-1523).  One octave: dog (S2,H,W), candidates (n,3) = (s,r,c).    */
/* Canonical: IEEE division (the reference compiles --use_fast_math),    */
/* no contraction, expression trees as written in the reference.         */
/* out: valid[n], ri[n], ci[n], si[n], resp[n].                          */
/* ------------------------------------------------------------------ */
EXPORT void orc_refine(const float* dog, int S2, int H, int W, const int* cands, long n,
                       int n_scales, int border, float cthr, float edge_score,
                       int* valid, float* out_ri, float* out_ci, int* out_si, float* out_resp) {
    long HW = (long)H * W;
    int S = n_scales;
    (void)S2;
    #pragma omp parallel for schedule(static)
    for (long idx = 0; idx < n; ++idx) {
        int si = cands[idx * 3 + 0], row = cands[idx * 3 + 1], col = cands[idx * 3 + 2];
        float ox = 0.0f, oy = 0.0f, os_ = 0.0f;
        int converged = 0;
        for (int iter = 0; iter < 5; ++iter) {
            if (si < 1 || si > S || row < border || row >= H - border || col < border || col >= W - border) break;
            const float* cr = dog + si * HW + (long)row * W;
            const float* cr1 = dog + si * HW + (long)(row + 1) * W;
            const float* crm = dog + si * HW + (long)(row - 1) * W;
            const float* pr = dog + (si + 1) * HW + (long)row * W;
            const float* pr1 = dog + (si + 1) * HW + (long)(row + 1) * W;
            const float* prm = dog + (si + 1) * HW + (long)(row - 1) * W;
            const float* mr = dog + (si - 1) * HW + (long)row * W;
            const float* mr1 = dog + (si - 1) * HW + (long)(row + 1) * W;
            const float* mrm = dog + (si - 1) * HW + (long)(row - 1) * W;
            float cval = cr[col];
            float dx = (cr[col + 1] - cr[col - 1]) * 0.5f;
            float dy = (cr1[col] - crm[col]) * 0.5f;
            float ds = (pr[col] - mr[col]) * 0.5f;
            float dxx = cr[col + 1] - 2.0f * cval + cr[col - 1];
            float dyy = cr1[col] - 2.0f * cval + crm[col];
            float dss = pr[col] - 2.0f * cval + mr[col];
            float dxy = (cr1[col + 1] - cr1[col - 1] - crm[col + 1] + crm[col - 1]) * 0.25f;
            float dxs = (pr[col + 1] - pr[col - 1] - mr[col + 1] + mr[col - 1]) * 0.25f;
            float dys = (pr1[col] - prm[col] - mr1[col] + mrm[col]) * 0.25f;
            float det = dxx * (dyy * dss - dys * dys) - dxy * (dxy * dss - dys * dxs) + dxs * (dxy * dys - dyy * dxs);
            if (fabsf(det) < 1e-12f) break;
            float inv_det = 1.0f / det;
            float p = -dx, q = -dy, rv = -ds;
            ox = (p * (dyy * dss - dys * dys) - dxy * (q * dss - dys * rv) + dxs * (q * dys - dyy * rv)) * inv_det;
            oy = (dxx * (q * dss - dys * rv) - p * (dxy * dss - dys * dxs) + dxs * (dxy * rv - q * dxs)) * inv_det;
            os_ = (dxx * (dyy * rv - q * dys) - dxy * (dxy * rv - q * dxs) + p * (dxy * dys - dyy * dxs)) * inv_det;
            if (fabsf(ox) < 0.5f && fabsf(oy) < 0.5f && fabsf(os_) < 0.5f) { converged = 1; break; }
            col += (ox >= 0.0f) ? (int)(ox + 0.5f) : (int)(ox - 0.5f);
            row += (oy >= 0.0f) ? (int)(oy + 0.5f) : (int)(oy - 0.5f);
            si += (os_ >= 0.0f) ? (int)(os_ + 0.5f) : (int)(os_ - 0.5f);
        }
        valid[idx] = 0;
        if (!converged) continue;
        if (si < 1 || si > S || row < border || row >= H - border || col < border || col >= W - border) continue;
        const float* cr = dog + si * HW + (long)row * W;
        const float* cr1 = dog + si * HW + (long)(row + 1) * W;
        const float* crm = dog + si * HW + (long)(row - 1) * W;
        const float* pr = dog + (si + 1) * HW + (long)row * W;
        const float* mr = dog + (si - 1) * HW + (long)row * W;
        float cval = cr[col];
        float dx_ = (cr[col + 1] - cr[col - 1]) * 0.5f;
        float dy_ = (cr1[col] - crm[col]) * 0.5f;
        float ds_ = (pr[col] - mr[col]) * 0.5f;
        float response = fabsf(cval + 0.5f * (dx_ * ox + dy_ * oy + ds_ * os_));
        if (response < cthr) continue;
        float dxx = cr[col + 1] - 2.0f * cval + cr[col - 1];
        float dyy = cr1[col] - 2.0f * cval + crm[col];
        float dxy = (cr1[col + 1] - cr1[col - 1] - crm[col + 1] + crm[col - 1]) * 0.25f;
        float trace = dxx + dyy;
        float det2d = dxx * dyy - dxy * dxy;
        if (det2d <= 0.0f || (trace * trace / det2d) >= edge_score) continue;
        valid[idx] = 1;
        out_ri[idx] = (float)row + oy;
        out_ci[idx] = (float)col + ox;
        out_si[idx] = si;
        out_resp[idx] = response;
    }
}

/* ------------------------------------------------------------------ */
/* A10: orientation histogram (pysift/core.py:228-333).  gauss is       */
/* (L,H,W); kpts (N,4) = [ri, ci, sigma, si].  36 bins with linear bin  */
/* split, 2x [.25,.5,.25] circular smoothing, peaks >= 0.8*max and >=    */
/* both neighbours, parabolic refinement, up to 4 angles (-1 = none).   */
/* Canonical: orc_expf for __expf, orc_atan2f for atan2f; the histogram */
/* is an exact fixed-point sum (orc_fix) instead of per-lane float sums */
/* merged by a warp tree, so its value does not depend on the order in  */
/* which pixels are visited.                                            */
/* ------------------------------------------------------------------ */
/* Exact, order-independent histogram accumulation: every non-negative
 * float32 contribution is rounded to a multiple of 2^-40 (round to nearest
 * even) and summed as a 64-bit integer; the bin value is the sum rounded to
 * float32 and scaled back.  Contributions are below 2.2 (gradient
 * magnitudes of pyramid values in [-0.28, 1.28]), so the sums stay far below
 * 2^63 for any patch these kernels visit. */
static inline long long orc_fix(float c) { return llrintf(c * 0x1p40f); }
static inline float orc_unfix(long long s) { return (float)s * 0x1p-40f; }
/* The descriptor's bins use a quantum of 2^-24 (same rounding, same
 * integer sum): the kernel keeps them in 32-bit shared words folded into
 * 64-bit totals, so the sum is the same exact integer. */
static inline long long orc_fix24(float c) { return llrintf(c * 0x1p24f); }
static inline float orc_unfix24(long long s) { return (float)s * 0x1p-24f; }

static float tree32(const float* v, int stride) {
    float a[32];
    for (int i = 0; i < 32; ++i) a[i] = v[i * stride];
    for (int d = 16; d >= 1; d >>= 1)
        for (int i = 0; i < d; ++i) a[i] = a[i] + a[i + d];
    return a[0];
}

EXPORT void orc_orientation(const float* gauss, int H, int W, const float* kpts, long N, float* out) {
    long HW = (long)H * W;
    #pragma omp parallel for schedule(dynamic, 16)
    for (long k = 0; k < N; ++k) {
        long long acc[36];
        memset(acc, 0, sizeof(acc));
        float ri = kpts[k * 4 + 0], ci = kpts[k * 4 + 1], sigma = kpts[k * 4 + 2];
        int si = (int)kpts[k * 4 + 3];
        int radius = (int)(4.5f * sigma + 0.5f);
        if (radius < 1) radius = 1;
        float sigma_w = 1.5f * sigma;
        float inv_2sw2 = 1.0f / (2.0f * sigma_w * sigma_w + 1e-12f);
        int r_min = (int)ri - radius; if (r_min < 1) r_min = 1;
        int r_max = (int)ri + radius; if (r_max > H - 2) r_max = H - 2;
        int c_min = (int)ci - radius; if (c_min < 1) c_min = 1;
        int c_max = (int)ci + radius; if (c_max > W - 2) c_max = W - 2;
        int n_cols = c_max - c_min + 1; if (n_cols < 1) n_cols = 1;
        int nr = r_max - r_min + 1; if (nr < 0) nr = 0;
        int total = nr * n_cols;
        const float* g = gauss + si * HW;
        for (int pidx = 0; pidx < total; ++pidx) {
            int r = r_min + pidx / n_cols;
            int c = c_min + pidx % n_cols;
            float dx = g[(long)r * W + c + 1] - g[(long)r * W + c - 1];
            float dy = g[(long)(r + 1) * W + c] - g[(long)(r - 1) * W + c];
            float mag = sqrtf(dx * dx + dy * dy);
            float ori = fmodf(orc_atan2f(dy, dx) * 57.29577951f + 360.0f, 360.0f);
            float fr = (float)r - ri, fc = (float)c - ci;
            float wt = orc_expf(-(fr * fr + fc * fc) * inv_2sw2);
            float bin_f = ori * 0.1f;
            int bin_i = ((int)bin_f) % 36;
            int bin_r = (bin_i + 1) % 36;
            float frac = bin_f - floorf(bin_f);
            float mw = mag * wt;
            acc[bin_i] += orc_fix(mw * (1.0f - frac));
            acc[bin_r] += orc_fix(mw * frac);
        }
        float hist[36], smooth[36];
        for (int b = 0; b < 36; ++b) hist[b] = orc_unfix(acc[b]);
        for (int it = 0; it < 2; ++it) {
            for (int b = 0; b < 36; ++b)
                smooth[b] = 0.25f * hist[(b + 35) % 36] + 0.5f * hist[b] + 0.25f * hist[(b + 1) % 36];
            for (int b = 0; b < 36; ++b) hist[b] = smooth[b];
        }
        float peak = 0.0f;
        for (int b = 0; b < 36; ++b) if (hist[b] > peak) peak = hist[b];
        float thr = 0.8f * peak;
        int o = 0;
        for (int b = 0; b < 36; ++b) {
            if (hist[b] >= thr) {
                float l = hist[(b + 35) % 36], rv = hist[(b + 1) % 36];
                if (hist[b] >= l && hist[b] >= rv) {
                    float denom = l - 2.0f * hist[b] + rv;
                    float fine = (float)b + (fabsf(denom) > 1e-12f ? 0.5f * (l - rv) / denom : 0.0f);
                    float angle = fmodf(fine / 36.0f * 360.0f + 360.0f, 360.0f);
                    if (o < 4) out[k * 4 + (o++)] = angle;
                }
            }
        }
        for (; o < 4; ++o) out[k * 4 + o] = -1.0f;
    }
}

/* ------------------------------------------------------------------ */
/* A11: SIFT descriptor, single-scale and DSP pooling                  */
/* (pysift/core.py:693-835, 845-997, 1772-1900).  gauss (L,H,W); kpts  */
/* (N,5) = [ri, ci, ang_rad, ph, si]; dsp_scales NULL/n_dsp=0 for the   */
/* single-scale descriptor.  Output: L2 -> clip 0.2 -> L2 vector (the   */
/* kernel output before RootSIFT).                                      */
/* Canonical: exact fixed-point histogram (orc_fix24) instead of shared-*/
/* memory float atomics; norms by the reference's warp tree then warp   */
/* partials 0..3 in order; 1/sqrtf instead of rsqrtf; orc_* math.        */
/* ------------------------------------------------------------------ */
static void desc_accumulate(const float* g, int H, int W, float ri, float ci, float cos_a, float sin_a,
                            float ang_rad, int ph, long long acc[128]) {
    float scale_sp = 4.0f / (2.0f * (float)ph);
    float sigma_d = (float)ph * 0.5657f;
    float inv_2s2 = 1.0f / (2.0f * sigma_d * sigma_d + 1e-12f);
    int side = 2 * ph + 1;
    int total = side * side;
    int r0 = (int)ri, c0 = (int)ci;
    for (int flat = 0; flat < total; ++flat) {
        int r_off = flat / side - ph;
        int c_off = flat % side - ph;
        int rr = r0 + r_off, cc = c0 + c_off;
        if (rr < 1 || rr >= H - 1 || cc < 1 || cc >= W - 1) continue;
        float fc = (float)c_off, fr = (float)r_off;
        float xr = cos_a * fc - sin_a * fr;
        float yr = sin_a * fc + cos_a * fr;
        float xb = xr * scale_sp + 1.5f;
        float yb = yr * scale_sp + 1.5f;
        if (xb < -0.5f || xb >= 3.5f || yb < -0.5f || yb >= 3.5f) continue;
        float dx = g[(long)rr * W + cc + 1] - g[(long)rr * W + cc - 1];
        float dy = g[(long)(rr + 1) * W + cc] - g[(long)(rr - 1) * W + cc];
        float mag = sqrtf(dx * dx + dy * dy);
        float ori_deg = fmodf((orc_atan2f(dy, dx) - ang_rad) * 57.29577951f + 360.0f, 360.0f);
        float gw = orc_expf(-(xr * xr + yr * yr) * inv_2s2);
        float wmag = mag * gw;
        float ob = ori_deg * 0.02222222f;
        int oi0 = (int)floorf(ob);
        float df = ob - (float)oi0;
        int xi0 = (int)floorf(xb), yi0 = (int)floorf(yb);
        float dx_b = xb - (float)xi0, dy_b = yb - (float)yi0;
        int xi0c = xi0 < 0 ? 0 : (xi0 > 3 ? 3 : xi0);
        int yi0c = yi0 < 0 ? 0 : (yi0 > 3 ? 3 : yi0);
        int xi1c = xi0 + 1 < 0 ? 0 : (xi0 + 1 > 3 ? 3 : xi0 + 1);
        int yi1c = yi0 + 1 < 0 ? 0 : (yi0 + 1 > 3 ? 3 : yi0 + 1);
        int oi0w = ((oi0 % 8) + 8) % 8;
        int oi1w = ((oi0 + 1) % 8 + 8) % 8;
        float w_y0 = 1.0f - dy_b, w_y1 = dy_b;
        float w_x0 = 1.0f - dx_b, w_x1 = dx_b;
        float w_o0 = 1.0f - df, w_o1 = df;
        acc[yi0c * 32 + xi0c * 8 + oi0w] += orc_fix24(w_y0 * w_x0 * w_o0 * wmag);
        acc[yi0c * 32 + xi0c * 8 + oi1w] += orc_fix24(w_y0 * w_x0 * w_o1 * wmag);
        acc[yi0c * 32 + xi1c * 8 + oi0w] += orc_fix24(w_y0 * w_x1 * w_o0 * wmag);
        acc[yi0c * 32 + xi1c * 8 + oi1w] += orc_fix24(w_y0 * w_x1 * w_o1 * wmag);
        acc[yi1c * 32 + xi0c * 8 + oi0w] += orc_fix24(w_y1 * w_x0 * w_o0 * wmag);
        acc[yi1c * 32 + xi0c * 8 + oi1w] += orc_fix24(w_y1 * w_x0 * w_o1 * wmag);
        acc[yi1c * 32 + xi1c * 8 + oi0w] += orc_fix24(w_y1 * w_x1 * w_o0 * wmag);
        acc[yi1c * 32 + xi1c * 8 + oi1w] += orc_fix24(w_y1 * w_x1 * w_o1 * wmag);
    }
}

static float norm_sq_tree(const float* v /*128*/) {
    float sq[128];
    for (int i = 0; i < 128; ++i) sq[i] = v[i] * v[i];
    float w0 = tree32(sq + 0, 1), w1 = tree32(sq + 32, 1), w2 = tree32(sq + 64, 1), w3 = tree32(sq + 96, 1);
    return w0 + w1 + w2 + w3;
}

EXPORT void orc_descriptor(const float* gauss, int n_slices, int H, int W, const float* kpts, long N,
                           const float* dsp_scales, int n_dsp, float* out) {
    long HW = (long)H * W;
    #pragma omp parallel for schedule(dynamic, 8)
    for (long k = 0; k < N; ++k) {
        long long acc[128];
        memset(acc, 0, sizeof(acc));
        float ri = kpts[k * 5 + 0], ci = kpts[k * 5 + 1], ang = kpts[k * 5 + 2];
        float phf = kpts[k * 5 + 3];
        int si = (int)kpts[k * 5 + 4];
        float* o = out + k * 128;
        if (n_dsp > 0) {
            if (si < 0 || si >= n_slices || phf < 1.0f || phf > 200.0f) { memset(o, 0, 512); continue; }
        } else {
            int ph = (int)phf;
            if (si < 0 || si >= n_slices || ph < 1 || ph > 200) { memset(o, 0, 512); continue; }
        }
        float cos_a, sin_a;
        orc_sincosf(ang, &sin_a, &cos_a);
        const float* g = gauss + si * HW;
        if (n_dsp > 0) {
            for (int d = 0; d < n_dsp; ++d) {
                int ph = (int)(phf * dsp_scales[d] + 0.5f);
                if (ph < 4) ph = 4;
                desc_accumulate(g, H, W, ri, ci, cos_a, sin_a, ang, ph, acc);
            }
        } else {
            desc_accumulate(g, H, W, ri, ci, cos_a, sin_a, ang, (int)phf, acc);
        }
        float v[128];
        for (int b = 0; b < 128; ++b) v[b] = orc_unfix24(acc[b]);
        if (n_dsp > 0) {
            float inv_n = 1.0f / (float)n_dsp;
            for (int b = 0; b < 128; ++b) v[b] = v[b] * inv_n;
        }
        float inv = 1.0f / sqrtf(norm_sq_tree(v) + 1e-14f);
        for (int b = 0; b < 128; ++b) {
            float t = v[b] * inv;
            v[b] = t > 0.2f ? 0.2f : t;
        }
        inv = 1.0f / sqrtf(norm_sq_tree(v) + 1e-14f);
        for (int b = 0; b < 128; ++b) o[b] = v[b] * inv;
    }
}

/* RootSIFT (pysift/core.py:1870-1873): x / (||x||_1 + 1e-7), clip >= 0,
 * sqrt.  Canonical L1 order: reference warp tree per 32 bins, warps 0..3. */
EXPORT void orc_rootsift(float* d, long N) {
    for (long k = 0; k < N; ++k) {
        float* v = d + k * 128;
        float a[128];
        for (int i = 0; i < 128; ++i) a[i] = fabsf(v[i]);
        float l1 = tree32(a, 1) + tree32(a + 32, 1) + tree32(a + 64, 1) + tree32(a + 96, 1);
        float den = l1 + 1e-7f;
        for (int i = 0; i < 128; ++i) {
            float t = v[i] / den;
            if (t < 0.0f) t = 0.0f;
            v[i] = sqrtf(t);
        }
    }
}

/* ------------------------------------------------------------------ */
/* Array wrappers of the elementary functions, for their accuracy tests. */
/* ------------------------------------------------------------------ */
EXPORT void orc_test_expf(const float* x, float* out, long n) {
    for (long i = 0; i < n; ++i) out[i] = orc_expf(x[i]);
}
EXPORT void orc_test_atan2f(const float* y, const float* x, float* out, long n) {
    for (long i = 0; i < n; ++i) out[i] = orc_atan2f(y[i], x[i]);
}
EXPORT void orc_test_sincosf(const float* a, float* s, float* c, long n) {
    for (long i = 0; i < n; ++i) orc_sincosf(a[i], &s[i], &c[i]);
}
EXPORT void orc_test_log2d(const double* p, double* out, long n) {
    for (long i = 0; i < n; ++i) out[i] = orc_log2d(p[i]);
}
