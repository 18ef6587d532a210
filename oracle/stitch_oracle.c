/*
 * stitch_oracle.c -- CPU restatement of PySIFT's stitch geometry path.
 *
 * TEST INFRASTRUCTURE ONLY (see sift_oracle.c).  Restates
 *   GPUPyStitch._normalize_points / _compute_homography  pysift/core.py:2946-2981
 *   _ransac_batch_eval / _ransac (MAGSAC++, LO refits)  pysift/core.py:2272-2313, 3011-3097
 *   _pca_compress / _match_features preparation          pysift/core.py:2703-2743, 2877-2888
 *   _warp_image + image-2 placement                      pysift/core.py:3210-3239, 3794-3800
 * with the canonical choices documented in pysift_b200/csrc/ransac.cu and
 * image.cu: fixed-order sums (256 contiguous chunks + pairwise tree; 32
 * lane-strided partials + warp tree), Gaussian elimination for the 4-point
 * null vector, Jacobi eigenvectors of A^T A for the refits, analytic T2^-1
 * and adjugate H^-1, its own float64 exp (oracle_exp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))
#define RT 256

static double oracle_exp(double x) {
    if (x < -745.0) return 0.0;
    const double LOG2E = 1.4426950408889634;
    const double LN2_HI = 0x1.62e42ffp-1;
    const double LN2_LO = -0x1.718432a1b0e26p-35;
    double n = rint(x * LOG2E);
    double r = fma(-n, LN2_HI, x);
    r = fma(-n, LN2_LO, r);
    double p = 1.0 / 6227020800.0;
    p = fma(p, r, 1.0 / 479001600.0);
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int ni = (int)n;
    union { uint64_t u; double d; } s1, s2;
    if (ni >= -1022) {
        s1.u = (uint64_t)(ni + 1023) << 52;
        return p * s1.d;
    }
    s1.u = (uint64_t)(ni + 600 + 1023) << 52;
    s2.u = (uint64_t)(1023 - 600) << 52;
    return (p * s1.d) * s2.d;
}

EXPORT double orc_test_exp_d(double x) { return oracle_exp(x); }

static double tree256(double* p) {
    for (int s = RT / 2; s > 0; s >>= 1)
        for (int t = 0; t < s; ++t) p[t] = p[t] + p[t + s];
    return p[0];
}

typedef struct { double s, cx, cy; } Norm;

static Norm hartley(const double* pts, const int* idx, int n) {
    double px[RT], py[RT], pd[RT];
    int chunk = (n + RT - 1) / RT;
    for (int t = 0; t < RT; ++t) {
        int b = t * chunk, e = b + chunk < n ? b + chunk : n;
        double sx = 0.0, sy = 0.0;
        for (int i = b; i < e; ++i) {
            int k = idx ? idx[i] : i;
            sx = sx + pts[2 * k];
            sy = sy + pts[2 * k + 1];
        }
        px[t] = sx;
        py[t] = sy;
    }
    Norm r;
    r.cx = tree256(px) / (double)n;
    r.cy = tree256(py) / (double)n;
    for (int t = 0; t < RT; ++t) {
        int b = t * chunk, e = b + chunk < n ? b + chunk : n;
        double sd = 0.0;
        for (int i = b; i < e; ++i) {
            int k = idx ? idx[i] : i;
            double dx = pts[2 * k] - r.cx, dy = pts[2 * k + 1] - r.cy;
            sd = sd + sqrt(dx * dx + dy * dy);
        }
        pd[t] = sd;
    }
    double md = tree256(pd) / (double)n;
    r.s = sqrt(2.0) / (md + 1e-10);
    return r;
}

static void mat3_mul(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = (A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j]) + A[3 * i + 2] * B[6 + j];
}

static void norm_mats(Norm n1, Norm n2, double* T1, double* T2inv) {
    double a[9] = {n1.s, 0.0, -n1.s * n1.cx, 0.0, n1.s, -n1.s * n1.cy, 0.0, 0.0, 1.0};
    double b[9] = {1.0 / n2.s, 0.0, n2.cx, 0.0, 1.0 / n2.s, n2.cy, 0.0, 0.0, 1.0};
    memcpy(T1, a, sizeof(a));
    memcpy(T2inv, b, sizeof(b));
}

static double nrm(double s, double c, double v) { return s * v + (-s * c); }

static void denormalise(const double* Hn, const double* T1, const double* T2inv, double* H) {
    double t[9];
    mat3_mul(T2inv, Hn, t);
    mat3_mul(t, T1, H);
    double s = H[8];
    double ss = fabs(s) > 1e-10 ? s : 1.0;
    for (int i = 0; i < 9; ++i) H[i] = H[i] / ss;
}

static void inv3_guarded(const double* a, double* inv, double guard) {
    double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                 a[2] * (a[3] * a[7] - a[4] * a[6]);
    double d = (guard > 0.0 && !(fabs(det) > guard)) ? 1.0 : det;
    inv[0] = (a[4] * a[8] - a[5] * a[7]) / d;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) / d;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) / d;
    inv[3] = (a[5] * a[6] - a[3] * a[8]) / d;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) / d;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) / d;
    inv[6] = (a[3] * a[7] - a[4] * a[6]) / d;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) / d;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) / d;
}

static double sym_err(const double* H, const double* Hi, double x1, double y1, double x2, double y2, int clamp) {
    double fx = (H[0] * x1 + H[1] * y1) + H[2];
    double fy = (H[3] * x1 + H[4] * y1) + H[5];
    double fw = (H[6] * x1 + H[7] * y1) + H[8];
    if (clamp) fw = fw < 1e-10 ? 1e-10 : fw;
    double ex = fx / fw - x2, ey = fy / fw - y2;
    double bx = (Hi[0] * x2 + Hi[1] * y2) + Hi[2];
    double by = (Hi[3] * x2 + Hi[4] * y2) + Hi[5];
    double bw = (Hi[6] * x2 + Hi[7] * y2) + Hi[8];
    if (clamp) bw = bw < 1e-10 ? 1e-10 : bw;
    double gx = bx / bw - x1, gy = by / bw - y1;
    return (ex * ex + ey * ey) + (gx * gx + gy * gy);
}

static int null_vector_8x9(const double* x1, const double* y1, const double* x2, const double* y2, double* h) {
    double A[8][9];
    for (int k = 0; k < 4; ++k) {
        double* e = A[2 * k];
        double* o = A[2 * k + 1];
        e[0] = -x1[k]; e[1] = -y1[k]; e[2] = -1.0; e[3] = 0.0; e[4] = 0.0; e[5] = 0.0;
        e[6] = x2[k] * x1[k]; e[7] = x2[k] * y1[k]; e[8] = x2[k];
        o[0] = 0.0; o[1] = 0.0; o[2] = 0.0; o[3] = -x1[k]; o[4] = -y1[k]; o[5] = -1.0;
        o[6] = y2[k] * x1[k]; o[7] = y2[k] * y1[k]; o[8] = y2[k];
    }
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        double best = fabs(A[c][c]);
        for (int r = c + 1; r < 8; ++r) {
            double v = fabs(A[r][c]);
            if (v > best) { best = v; piv = r; }
        }
        if (!(best > 1e-12)) return 0;
        if (piv != c)
            for (int j = 0; j < 9; ++j) { double t = A[c][j]; A[c][j] = A[piv][j]; A[piv][j] = t; }
        for (int r = c + 1; r < 8; ++r) {
            double f = A[r][c] / A[c][c];
            for (int j = c; j < 9; ++j) A[r][j] = A[r][j] - f * A[c][j];
        }
    }
    h[8] = 1.0;
    for (int c = 7; c >= 0; --c) {
        double s = A[c][8];
        for (int j = c + 1; j < 8; ++j) s = s + A[c][j] * h[j];
        h[c] = -s / A[c][c];
    }
    return 1;
}

static void dlt_refit(const double* p1, const double* p2, const int* idx, int m, double* H) {
    Norm n1 = hartley(p1, idx, m), n2 = hartley(p2, idx, m);
    static double part[RT][45];
    int chunk = (m + RT - 1) / RT;
    for (int t = 0; t < RT; ++t) {
        double* acc = part[t];
        for (int k = 0; k < 45; ++k) acc[k] = 0.0;
        int b = t * chunk, e = b + chunk < m ? b + chunk : m;
        for (int i = b; i < e; ++i) {
            int k = idx[i];
            double x1 = nrm(n1.s, n1.cx, p1[2 * k]), y1 = nrm(n1.s, n1.cy, p1[2 * k + 1]);
            double x2 = nrm(n2.s, n2.cx, p2[2 * k]), y2 = nrm(n2.s, n2.cy, p2[2 * k + 1]);
            double re[9] = {-x1, -y1, -1.0, 0.0, 0.0, 0.0, x2 * x1, x2 * y1, x2};
            double ro[9] = {0.0, 0.0, 0.0, -x1, -y1, -1.0, y2 * x1, y2 * y1, y2};
            int q = 0;
            for (int r = 0; r < 9; ++r)
                for (int c = r; c < 9; ++c, ++q) acc[q] = (acc[q] + re[r] * re[c]) + ro[r] * ro[c];
        }
    }
    double Mv[45];
    for (int q = 0; q < 45; ++q) {
        double col[RT];
        for (int t = 0; t < RT; ++t) col[t] = part[t][q];
        Mv[q] = tree256(col);
    }
    double M[9][9], V[9][9];
    int q = 0;
    for (int r = 0; r < 9; ++r)
        for (int c = r; c < 9; ++c, ++q) M[r][c] = M[c][r] = Mv[q];
    for (int r = 0; r < 9; ++r)
        for (int c = 0; c < 9; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
    /* parallel (round-robin) Jacobi: round r rotates the disjoint pairs
     * {(r+i) mod 9, (r-i) mod 9}, i = 1..4; angles from the start-of-round
     * matrix, then all column rotations, then all row rotations; only pairs
     * with |a_pq| > tol = 2^-52 trace rotate; stop when no upper
     * off-diagonal element exceeds tol (15 sweeps at most). */
    double tr = 0.0;
    for (int k = 0; k < 9; ++k) tr = tr + M[k][k];
    const double tol = tr * 0x1p-52;
    for (int sweep = 0; sweep < 15; ++sweep) {
        int nz = 0;
        for (int r = 0; r < 9; ++r)
            for (int c = r + 1; c < 9; ++c)
                if (fabs(M[r][c]) > tol) nz = 1;
        if (!nz) break;
        for (int rnd = 0; rnd < 9; ++rnd) {
            int P[4], Q[4], act[4];
            double C[4], S[4];
            for (int j = 0; j < 4; ++j) {
                int a = (rnd + j + 1) % 9, bb = (rnd + 9 - j - 1) % 9;
                int p = a < bb ? a : bb, qq = a < bb ? bb : a;
                P[j] = p;
                Q[j] = qq;
                act[j] = 0;
                double apq = M[p][qq];
                if (!(fabs(apq) > tol)) continue;
                double app = M[p][p], aqq = M[qq][qq];
                double theta = (aqq - app) / (2.0 * apq);
                double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(tt * tt + 1.0);
                C[j] = c;
                S[j] = tt * c;
                act[j] = 1;
            }
            for (int j = 0; j < 4; ++j) {
                if (!act[j]) continue;
                int p = P[j], qq = Q[j];
                for (int k = 0; k < 9; ++k) {
                    double mkp = M[k][p], mkq = M[k][qq];
                    M[k][p] = C[j] * mkp - S[j] * mkq;
                    M[k][qq] = S[j] * mkp + C[j] * mkq;
                }
            }
            for (int j = 0; j < 4; ++j) {
                if (!act[j]) continue;
                int p = P[j], qq = Q[j];
                for (int k = 0; k < 9; ++k) {
                    double mpk = M[p][k], mqk = M[qq][k];
                    M[p][k] = C[j] * mpk - S[j] * mqk;
                    M[qq][k] = S[j] * mpk + C[j] * mqk;
                    double vkp = V[k][p], vkq = V[k][qq];
                    V[k][p] = C[j] * vkp - S[j] * vkq;
                    V[k][qq] = S[j] * vkp + C[j] * vkq;
                }
            }
        }
    }
    int best = 0;
    for (int k = 1; k < 9; ++k)
        if (M[k][k] < M[best][best]) best = k;
    double hn[9], T1[9], T2inv[9], t9[9];
    for (int k = 0; k < 9; ++k) hn[k] = V[k][best];
    norm_mats(n1, n2, T1, T2inv);
    mat3_mul(T2inv, hn, t9);
    mat3_mul(t9, T1, H);
    double s = H[8];
    for (int k = 0; k < 9; ++k) H[k] = H[k] / s;
}

EXPORT void orc_dlt(const double* p1, const double* p2, int n, double* H) {
    int* idx = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) idx[i] = i;
    dlt_refit(p1, p2, idx, n, H);
    free(idx);
}

/* scores[h] for every hypothesis; H_out, mask_out, info = [n_inliers, best_i, stage] */
EXPORT void orc_ransac(const double* p1, const double* p2, int n, const uint32_t* rnd, int n_hyp,
                       double thr, double sigma_max, int magsac, int min_inliers, double* H_out,
                       uint8_t* mask_out, int* info, double* scores) {
    double tq = thr * thr, two_sig2 = 2.0 * (sigma_max * sigma_max);
    Norm n1 = hartley(p1, NULL, n), n2 = hartley(p2, NULL, n);
    double T1[9], T2inv[9];
    norm_mats(n1, n2, T1, T2inv);
    double* p1n = (double*)malloc(sizeof(double) * 2 * n);
    double* p2n = (double*)malloc(sizeof(double) * 2 * n);
    for (int i = 0; i < n; ++i) {
        p1n[2 * i] = nrm(n1.s, n1.cx, p1[2 * i]);
        p1n[2 * i + 1] = nrm(n1.s, n1.cy, p1[2 * i + 1]);
        p2n[2 * i] = nrm(n2.s, n2.cx, p2[2 * i]);
        p2n[2 * i + 1] = nrm(n2.s, n2.cy, p2[2 * i + 1]);
    }
    double* hypH = (double*)malloc(sizeof(double) * 9 * n_hyp);
    #pragma omp parallel for schedule(dynamic, 16)
    for (int h = 0; h < n_hyp; ++h) {
        double x1[4], y1[4], x2[4], y2[4];
        for (int k = 0; k < 4; ++k) {
            int i = (int)(rnd[4 * h + k] % (uint32_t)n);
            x1[k] = p1n[2 * i]; y1[k] = p1n[2 * i + 1];
            x2[k] = p2n[2 * i]; y2[k] = p2n[2 * i + 1];
        }
        double hn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, H[9], Hi[9];
        int ok = null_vector_8x9(x1, y1, x2, y2, hn);
        if (!ok) for (int k = 0; k < 9; ++k) hn[k] = 0.0;
        denormalise(hn, T1, T2inv, H);
        inv3_guarded(H, Hi, 1e-12);
        double lanes[32];
        for (int l = 0; l < 32; ++l) {
            double part = 0.0;
            if (ok)
                for (int i = l; i < n; i += 32) {
                    double e = sym_err(H, Hi, p1[2 * i], p1[2 * i + 1], p2[2 * i], p2[2 * i + 1], 1);
                    part = magsac ? part + oracle_exp(-e / two_sig2) : part + (e < tq ? 1.0 : 0.0);
                }
            lanes[l] = part;
        }
        for (int d = 16; d >= 1; d >>= 1)
            for (int l = 0; l < d; ++l) lanes[l] = lanes[l] + lanes[l + d];
        scores[h] = ok ? lanes[0] : -INFINITY;
        memcpy(hypH + 9 * h, H, sizeof(H));
    }
    /* first maximum; NaN scores never win; all -inf -> hypothesis 0 */
    double bs = -INFINITY;
    int best = -1;
    for (int h = 0; h < n_hyp; ++h)
        if (scores[h] > bs) { bs = scores[h]; best = h; }
    if (best < 0) best = 0;
    double H[9], Hi[9], H1[9], H1i[9];
    memcpy(H, hypH + 9 * best, sizeof(H));
    inv3_guarded(H, Hi, 1e-12);
    int* idx = (int*)malloc(sizeof(int) * n);
    int nb = 0;
    for (int i = 0; i < n; ++i) {
        mask_out[i] = sym_err(H, Hi, p1[2 * i], p1[2 * i + 1], p2[2 * i], p2[2 * i + 1], 1) < tq;
        if (mask_out[i]) idx[nb++] = i;
    }
    int stage = 0, n_final = nb;
    if (nb >= min_inliers) {
        dlt_refit(p1, p2, idx, nb, H1);
        inv3_guarded(H1, H1i, 0.0);
        int n2 = 0;
        for (int i = 0; i < n; ++i)
            if (sym_err(H1, H1i, p1[2 * i], p1[2 * i + 1], p2[2 * i], p2[2 * i + 1], 0) < tq) idx[n2++] = i;
        if (n2 >= min_inliers) {
            dlt_refit(p1, p2, idx, n2, H);
            memset(mask_out, 0, (size_t)(n > 0 ? n : 0));
            for (int k = 0; k < n2; ++k) mask_out[idx[k]] = 1;
            stage = 2;
            n_final = n2;
        } else {
            memcpy(H, H1, sizeof(H));
            stage = 1;
        }
    }
    memcpy(H_out, H, sizeof(H));
    info[0] = n_final;
    info[1] = best;
    info[2] = stage;
    free(p1n); free(p2n); free(hypH); free(idx);
}

/* ---- matcher preparation ---- */
static float tree32f(const float* v) {
    float a[32];
    for (int i = 0; i < 32; ++i) a[i] = v[i];
    for (int d = 16; d >= 1; d >>= 1)
        for (int i = 0; i < d; ++i) a[i] = a[i] + a[i + d];
    return a[0];
}

static float group_sum_sq(const float* v, int D) {
    float ss = 0.0f;
    for (int g = 0; g < D / 32; ++g) {
        float sq[32];
        for (int i = 0; i < 32; ++i) sq[i] = v[g * 32 + i] * v[g * 32 + i];
        float w = tree32f(sq);
        ss = g == 0 ? w : ss + w;
    }
    return ss;
}

EXPORT void orc_l2_normalize(const float* in, long n, int D, float* out) {
    for (long r = 0; r < n; ++r) {
        const float* v = in + r * D;
        float den = sqrtf(group_sum_sq(v, D)) + 1e-7f;
        for (int k = 0; k < D; ++k) out[r * D + k] = v[k] / den;
    }
}

/* float64 sums over fixed 128-row chunks, sequential inside a chunk, then the
 * chunk partials in order (pysift_b200/csrc/ransac.cu k_pca_*). */
EXPORT void orc_pca_stats(const float* x, long n, int D, float* mean, double* cov) {
    const long C = 128, nchunks = (n + C - 1) / C;
    for (int k = 0; k < D; ++k) {
        double s = 0.0;
        for (long c = 0; c < nchunks; ++c) {
            double p = 0.0;
            long i1 = (c + 1) * C < n ? (c + 1) * C : n;
            for (long i = c * C; i < i1; ++i) p = p + (double)x[i * D + k];
            s = s + p;
        }
        mean[k] = (float)(s / (double)n);
    }
    #pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < D; ++k)
        for (int l = k; l < D; ++l) {
            double s = 0.0;
            for (long c = 0; c < nchunks; ++c) {
                double p = 0.0;
                long i1 = (c + 1) * C < n ? (c + 1) * C : n;
                for (long i = c * C; i < i1; ++i) {
                    double a = (double)(x[i * D + k] - mean[k]), b = (double)(x[i * D + l] - mean[l]);
                    p = p + a * b;
                }
                s = s + p;
            }
            cov[k * D + l] = cov[l * D + k] = s / (double)n;
        }
}

/* projection + normalisation; output float32 (the caller rounds to fp16) */
/* ------------------------------------------------------------------ */
/* PCA basis (pysift/core.py:2729-2736 takes cp.linalg.eigh of the      */
/* covariance and keeps the eigenvectors of the P largest eigenvalues). */
/* Canonical: round-robin parallel cyclic Jacobi on the D x D float64    */
/* covariance (D even).  Round r = 0..D-2 rotates the D/2 disjoint      */
/* pairs {D-1, r} and {(r+i) mod (D-1), (r-i) mod (D-1)}, i = 1..D/2-1  */
/* (p < q); every angle comes from the matrix at the start of the round */
/* and only pairs with |a_pq| > tol rotate, tol = 2^-60 trace (the       */
/* trace summed in index order): all column rotations, then all row     */
/* rotations and the eigenvector columns.  Sweeps stop once no upper    */
/* off-diagonal element exceeds tol (60 at most).  The basis is the      */
/* eigenvectors of the last P indices in (eigenvalue asc, index asc)    */
/* order, in that order (as eigh's v[:, -P:]), rounded to float32.      */
/* The device kernel k_pca_basis performs the same operations.          */
/* ------------------------------------------------------------------ */
static void pca_pair(int D, int rnd, int i, int* p, int* q) {
    int a, b;
    if (i == 0) {
        a = D - 1;
        b = rnd;
    } else {
        a = (rnd + i) % (D - 1);
        b = (rnd - i + (D - 1)) % (D - 1);
    }
    *p = a < b ? a : b;
    *q = a < b ? b : a;
}

EXPORT int orc_pca_basis(const double* cov, int D, int P, float* proj, int* sweeps_out) {
    if (D < 2 || D > 128 || (D & 1) || P < 1 || P > D) return -1;
    static double A[128][128], V[128][128];
    double cs[64][2];
    int act[64], pq[64][2];
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) {
            A[r][c] = cov[(long)r * D + c];
            V[r][c] = r == c ? 1.0 : 0.0;
        }
    double tr = 0.0;
    for (int k = 0; k < D; ++k) tr = tr + A[k][k];
    const double tol = tr * 0x1p-60;
    int sweep = 0;
    for (; sweep < 60; ++sweep) {
        int any = 0;
        for (int r = 0; r < D && !any; ++r)
            for (int c = r + 1; c < D; ++c)
                if (fabs(A[r][c]) > tol) {
                    any = 1;
                    break;
                }
        if (!any) break;
        for (int rnd = 0; rnd < D - 1; ++rnd) {
            for (int j = 0; j < D / 2; ++j) {
                int p, q;
                pca_pair(D, rnd, j, &p, &q);
                pq[j][0] = p;
                pq[j][1] = q;
                const double apq = A[p][q];
                act[j] = 0;
                if (fabs(apq) > tol) {
                    const double app = A[p][p], aqq = A[q][q];
                    const double theta = (aqq - app) / (2.0 * apq);
                    const double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    const double c = 1.0 / sqrt(tt * tt + 1.0);
                    cs[j][0] = c;
                    cs[j][1] = tt * c;
                    act[j] = 1;
                }
            }
            for (int j = 0; j < D / 2; ++j) {
                if (!act[j]) continue;
                const int p = pq[j][0], q = pq[j][1];
                const double c = cs[j][0], s = cs[j][1];
                for (int k = 0; k < D; ++k) {
                    const double mkp = A[k][p], mkq = A[k][q];
                    A[k][p] = c * mkp - s * mkq;
                    A[k][q] = s * mkp + c * mkq;
                }
            }
            for (int j = 0; j < D / 2; ++j) {
                if (!act[j]) continue;
                const int p = pq[j][0], q = pq[j][1];
                const double c = cs[j][0], s = cs[j][1];
                for (int k = 0; k < D; ++k) {
                    const double mpk = A[p][k], mqk = A[q][k];
                    A[p][k] = c * mpk - s * mqk;
                    A[q][k] = s * mpk + c * mqk;
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
        }
    }
    /* rank of each index in (eigenvalue asc, index asc) order */
    int order[128];
    for (int i = 0; i < D; ++i) {
        int rk = 0;
        for (int j = 0; j < D; ++j)
            if (A[j][j] < A[i][i] || (A[j][j] == A[i][i] && j < i)) ++rk;
        order[rk] = i;
    }
    for (int k = 0; k < D; ++k)
        for (int c = 0; c < P; ++c) proj[(long)k * P + c] = (float)V[k][order[D - P + c]];
    if (sweeps_out) *sweeps_out = sweep;
    return 0;
}

EXPORT void orc_pca_project(const float* x, long n, int D, const float* mean, const float* proj, int P, float* out) {
    #pragma omp parallel for schedule(static)
    for (long r = 0; r < n; ++r) {
        float p[128];
        for (int c = 0; c < P; ++c) {
            float acc = 0.0f;
            for (int k = 0; k < D; ++k) acc = fmaf(x[r * D + k] - mean[k], proj[(long)k * P + c], acc);
            p[c] = acc;
        }
        float den = sqrtf(group_sum_sq(p, P)) + 1e-7f;
        for (int c = 0; c < P; ++c) out[r * P + c] = p[c] / den;
    }
}

/* ---- warp + feather (pysift_b200/csrc/image.cu k_warp_feather) ---- */
EXPORT void orc_warp_feather(const uint8_t* img1, int hs, int ws, const uint8_t* img2, int h2, int w2, int cw,
                             int ch, const float* hinv, float ox, float oy, int iox, int ioy, int feather,
                             uint8_t* out, uint8_t* warped, uint8_t* mask1, uint8_t* mask2) {
    #pragma omp parallel for schedule(static)
    for (int v = 0; v < ch; ++v)
        for (int u = 0; u < cw; ++u) {
            float X = (float)u - ox, Y = (float)v - oy;
            float s0 = hinv[0] * X + hinv[1] * Y + hinv[2];
            float s1 = hinv[3] * X + hinv[4] * Y + hinv[5];
            float s2 = hinv[6] * X + hinv[7] * Y + hinv[8];
            float den = s2 < 1e-10f ? 1e-10f : s2;
            float sx = s0 / den, sy = s1 / den;
            float sxn = (2.0f * sx / (float)(ws - 1)) - 1.0f;
            float syn = (2.0f * sy / (float)(hs - 1)) - 1.0f;
            int valid1 = (sxn >= -1.0f) && (sxn <= 1.0f) && (syn >= -1.0f) && (syn <= 1.0f);
            float ix = ((sxn + 1.0f) / 2.0f) * (float)(ws - 1);
            float iy = ((syn + 1.0f) / 2.0f) * (float)(hs - 1);
            float fx = floorf(ix), fy = floorf(iy);
            float c1[3] = {0.0f, 0.0f, 0.0f};
            int finite = isfinite(ix) && isfinite(iy) && fabsf(ix) < 1e9f && fabsf(iy) < 1e9f;
            if (finite) {
                int ixn = (int)fx, iyn = (int)fy;
                float ixse = fx + 1.0f, iyse = fy + 1.0f;
                float wnw = (ixse - ix) * (iyse - iy), wne = (ix - fx) * (iyse - iy);
                float wsw = (ixse - ix) * (iy - fy), wse = (ix - fx) * (iy - fy);
                int in_nw = ixn >= 0 && ixn < ws && iyn >= 0 && iyn < hs;
                int in_ne = ixn + 1 >= 0 && ixn + 1 < ws && iyn >= 0 && iyn < hs;
                int in_sw = ixn >= 0 && ixn < ws && iyn + 1 >= 0 && iyn + 1 < hs;
                int in_se = ixn + 1 >= 0 && ixn + 1 < ws && iyn + 1 >= 0 && iyn + 1 < hs;
                for (int c = 0; c < 3; ++c) {
                    float acc = 0.0f;
                    if (in_nw) acc = fmaf((float)img1[((long)iyn * ws + ixn) * 3 + c], wnw, acc);
                    if (in_ne) acc = fmaf((float)img1[((long)iyn * ws + ixn + 1) * 3 + c], wne, acc);
                    if (in_sw) acc = fmaf((float)img1[((long)(iyn + 1) * ws + ixn) * 3 + c], wsw, acc);
                    if (in_se) acc = fmaf((float)img1[((long)(iyn + 1) * ws + ixn + 1) * 3 + c], wse, acc);
                    c1[c] = acc;
                }
            }
            uint8_t w1b[3];
            for (int c = 0; c < 3; ++c) {
                float t = c1[c] < 0.0f ? 0.0f : (c1[c] > 255.0f ? 255.0f : c1[c]);
                w1b[c] = (uint8_t)(int)t;
            }
            int x2 = u - iox, y2 = v - ioy;
            int valid2 = x2 >= 0 && x2 < w2 && y2 >= 0 && y2 < h2;
            long o = ((long)v * cw + u) * 3;
            if (warped) for (int c = 0; c < 3; ++c) warped[o + c] = w1b[c];
            if (mask1) mask1[(long)v * cw + u] = (uint8_t)valid1;
            if (mask2) mask2[(long)v * cw + u] = (uint8_t)valid2;
            uint8_t res[3] = {0, 0, 0};
            if (valid1 && valid2 && feather) {
                float d1 = 1.0f + fminf(fminf(ix, (float)(ws - 1) - ix), fminf(iy, (float)(hs - 1) - iy));
                int m = x2 < w2 - 1 - x2 ? x2 : w2 - 1 - x2;
                int my = y2 < h2 - 1 - y2 ? y2 : h2 - 1 - y2;
                float d2 = 1.0f + (float)(m < my ? m : my);
                const uint8_t* p2 = img2 + ((long)y2 * w2 + x2) * 3;
                for (int c = 0; c < 3; ++c) {
                    float val = ((float)w1b[c] * d1 + (float)p2[c] * d2) / (d1 + d2);
                    float t = val + 0.5f;
                    t = t < 0.0f ? 0.0f : (t > 255.0f ? 255.0f : t);
                    res[c] = (uint8_t)(int)t;
                }
            } else if (valid2) {
                const uint8_t* p2 = img2 + ((long)y2 * w2 + x2) * 3;
                res[0] = p2[0]; res[1] = p2[1]; res[2] = p2[2];
            } else if (valid1) {
                res[0] = w1b[0]; res[1] = w1b[1]; res[2] = w1b[2];
            }
            for (int c = 0; c < 3; ++c) out[o + c] = res[c];
        }
}
