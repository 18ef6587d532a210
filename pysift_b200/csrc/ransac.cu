// ransac.cu -- batched RANSAC / MAGSAC++ scoring with LO refits, all on the GPU,
// and the descriptor preparation of the stitch matcher.
//
// Reference: GPUPyStitch._ransac / _ransac_batch_eval / _compute_homography /
// _normalize_points (pysift/core.py:2272-2313, 2946-2981, 3011-3097) and
// _match_features / _pca_compress (pysift/core.py:2703-2743, 2877-2888).
//
// Canonical arithmetic (the CPU oracle implements the same definition):
//   * sums over points use a fixed order: contiguous chunks per thread,
//     sequential inside a chunk, then a pairwise tree over the partials;
//   * a hypothesis' null vector is found by Gaussian elimination with partial
//     pivoting on its 8x9 system (the reference takes the last right singular
//     vector of a batched SVD); degenerate samples get score -inf;
//   * the least-squares refit takes the eigenvector of A^T A for the smallest
//     eigenvalue by cyclic Jacobi (until no off-diagonal element exceeds
//     2^-52 trace, 15 sweeps at most) instead of the SVD of A;
//   * T2^-1 is formed analytically, H^-1 by the adjugate; 3x3 products sum
//     k = 0, 1, 2 in order; exp is computed by ransac_exp (below);
//   * RANSAC samples are the reference's: torch.randint on a CPU generator
//     seeded 42 draws raw 32-bit MT19937 outputs r and returns r % N, so the
//     caller passes the raw stream and the kernel reduces it modulo N.
#include <cstdint>
#include <cstring>

#include "common.cuh"

namespace pysift {

constexpr int RT = 256;  // threads of the single-CTA kernels

// exp(x), x <= 0, float64: Cody-Waite reduction with ln2 split in a 32-bit
// head and a tail, Taylor series of exp(r) to degree 13, exact 2^n scaling.
__device__ __forceinline__ double ransac_exp(double x) {
    if (x < -745.0) return 0.0;
    const double LOG2E = 1.4426950408889634;
    const double LN2_HI = 0x1.62e42ffp-1;
    const double LN2_LO = -0x1.718432a1b0e26p-35;
    const double n = rint(x * LOG2E);
    double r = fma(-n, LN2_HI, x);
    r = fma(-n, LN2_LO, r);
    double p = 1.0 / 6227020800.0;  // 1/13!
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
    const int ni = (int)n;
    if (ni >= -1022) return p * __longlong_as_double((long long)(ni + 1023) << 52);
    return (p * __longlong_as_double((long long)(ni + 600 + 1023) << 52)) *
           __longlong_as_double((long long)(1023 - 600) << 52);
}

// NV fixed-order pairwise trees at once, the same pairs as block_tree_sum
// (t += t + s for s = 128, 64, ..., 1): the three top levels in shared
// memory, the rest with warp shuffles.  out (shared) receives the NV sums.
template <int NV>
__device__ __forceinline__ void block_tree_sums(const double (&v)[NV], double (*sh)[RT], double* out) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int u = 0; u < NV; ++u) sh[u][tid] = v[u];
    __syncthreads();
    if (tid < 128) {
#pragma unroll
        for (int u = 0; u < NV; ++u) sh[u][tid] = sh[u][tid] + sh[u][tid + 128];
    }
    __syncthreads();
    if (tid < 64) {
#pragma unroll
        for (int u = 0; u < NV; ++u) sh[u][tid] = sh[u][tid] + sh[u][tid + 64];
    }
    __syncthreads();
    if (tid < 32) {
#pragma unroll
        for (int u = 0; u < NV; ++u) {
            double x = sh[u][tid] + sh[u][tid + 32];
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) x = x + __shfl_down_sync(FULL_MASK, x, s);
            if (tid == 0) out[u] = x;
        }
    }
    __syncthreads();
}

struct Norm {
    double s, cx, cy;
};

// Hartley normalisation (pysift/core.py:2946-2957) of both point sets over
// the points listed in idx (or 0..n-1): c = mean, md = mean |p - c|,
// s = sqrt(2) / (md + 1e-10); sums over contiguous per-thread chunks, then
// the fixed-order trees of block_tree_sums.
__device__ void hartley2(const double* p1, const double* p2, const int* idx, int n, double (*sh)[RT], double* red,
                         Norm& n1, Norm& n2) {
    const int chunk = (n + RT - 1) / RT;
    const int b = threadIdx.x * chunk, e = min(n, b + chunk);
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = b; i < e; ++i) {
        const int k = idx ? idx[i] : i;
        s4[0] = s4[0] + p1[2 * k];
        s4[1] = s4[1] + p1[2 * k + 1];
        s4[2] = s4[2] + p2[2 * k];
        s4[3] = s4[3] + p2[2 * k + 1];
    }
    block_tree_sums<4>(s4, sh, red);
    n1.cx = red[0] / (double)n;
    n1.cy = red[1] / (double)n;
    n2.cx = red[2] / (double)n;
    n2.cy = red[3] / (double)n;
    __syncthreads();
    double s2[2] = {0.0, 0.0};
    for (int i = b; i < e; ++i) {
        const int k = idx ? idx[i] : i;
        const double dx1 = p1[2 * k] - n1.cx, dy1 = p1[2 * k + 1] - n1.cy;
        const double dx2 = p2[2 * k] - n2.cx, dy2 = p2[2 * k + 1] - n2.cy;
        s2[0] = s2[0] + sqrt(dx1 * dx1 + dy1 * dy1);
        s2[1] = s2[1] + sqrt(dx2 * dx2 + dy2 * dy2);
    }
    block_tree_sums<2>(s2, sh, red);
    n1.s = sqrt(2.0) / (red[0] / (double)n + 1e-10);
    n2.s = sqrt(2.0) / (red[1] / (double)n + 1e-10);
    __syncthreads();
}

__device__ __forceinline__ void mat3_mul(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = (A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j]) + A[3 * i + 2] * B[6 + j];
}

__device__ __forceinline__ void norm_mats(const Norm& n1, const Norm& n2, double* T1, double* T2inv) {
    T1[0] = n1.s; T1[1] = 0.0; T1[2] = -n1.s * n1.cx;
    T1[3] = 0.0; T1[4] = n1.s; T1[5] = -n1.s * n1.cy;
    T1[6] = 0.0; T1[7] = 0.0; T1[8] = 1.0;
    T2inv[0] = 1.0 / n2.s; T2inv[1] = 0.0; T2inv[2] = n2.cx;
    T2inv[3] = 0.0; T2inv[4] = 1.0 / n2.s; T2inv[5] = n2.cy;
    T2inv[6] = 0.0; T2inv[7] = 0.0; T2inv[8] = 1.0;
}

// Normalised coordinate: (s*x + 0*y) + (-s*c)
__device__ __forceinline__ double nrm(double s, double c, double v) { return s * v + (-s * c); }

// H = T2inv * Hn * T1, divided by H[2][2] when |H[2][2]| > 1e-10 (pysift/core.py:2290-2293)
__device__ __forceinline__ void denormalise(const double* Hn, const double* T1, const double* T2inv, double* H) {
    double t[9];
    mat3_mul(T2inv, Hn, t);
    mat3_mul(t, T1, H);
    const double s = H[8];
    const double ss = fabs(s) > 1e-10 ? s : 1.0;
    for (int i = 0; i < 9; ++i) H[i] = H[i] / ss;
}

// Adjugate inverse with the reference's determinant guard (pysift/core.py:2298-2307).
__device__ __forceinline__ void inv3_guarded(const double* a, double* inv, double guard) {
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    const double d = (guard > 0.0 && !(fabs(det) > guard)) ? 1.0 : det;
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

// Symmetric transfer error of one correspondence.  clamp: the batched
// evaluation clamps the projective denominator at 1e-10
// (pysift/core.py:2295, 2309); the LO reclassification divides plainly
// (pysift/core.py:3079-3083).
__device__ __forceinline__ double sym_err(const double* H, const double* Hi, double x1, double y1, double x2, double y2,
                                          bool clamp) {
    double fx = (H[0] * x1 + H[1] * y1) + H[2];
    double fy = (H[3] * x1 + H[4] * y1) + H[5];
    double fw = (H[6] * x1 + H[7] * y1) + H[8];
    if (clamp) fw = fw < 1e-10 ? 1e-10 : fw;
    const double ex = fx / fw - x2, ey = fy / fw - y2;
    double bx = (Hi[0] * x2 + Hi[1] * y2) + Hi[2];
    double by = (Hi[3] * x2 + Hi[4] * y2) + Hi[5];
    double bw = (Hi[6] * x2 + Hi[7] * y2) + Hi[8];
    if (clamp) bw = bw < 1e-10 ? 1e-10 : bw;
    const double gx = bx / bw - x1, gy = by / bw - y1;
    return (ex * ex + ey * ey) + (gx * gx + gy * gy);
}

// Null vector (h[8] = 1) of the 8x9 DLT system of 4 normalised
// correspondences by Gaussian elimination with partial pivoting; false if a
// pivot is <= 1e-12 (rank < 8).  Lanes 0..7 of a warp hold one row each
// (every lane of the warp must call it; lane r < 8 passes correspondence
// r >> 1).  The pivot of column c is the first maximum of |A[r][c]| over rows
// r >= c; rows move by shuffles; row r -= (A[r][c] / A[c][c]) * row c for
// columns c..8; back substitution sums j ascending.
__device__ bool null_vector_warp(double x1, double y1, double x2, double y2, double* h) {
    const int lane = threadIdx.x & 31;
    double R[9];
    if (lane >= 8) {
#pragma unroll
        for (int j = 0; j < 9; ++j) R[j] = 0.0;
    } else if ((lane & 1) == 0) {
        R[0] = -x1; R[1] = -y1; R[2] = -1.0; R[3] = 0.0; R[4] = 0.0; R[5] = 0.0;
        R[6] = x2 * x1; R[7] = x2 * y1; R[8] = x2;
    } else {
        R[0] = 0.0; R[1] = 0.0; R[2] = 0.0; R[3] = -x1; R[4] = -y1; R[5] = -1.0;
        R[6] = y2 * x1; R[7] = y2 * y1; R[8] = y2;
    }
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        double bv = (lane >= c && lane < 8) ? fabs(R[c]) : -1.0;
        int bi = lane;
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) {
            const double ov = __shfl_xor_sync(FULL_MASK, bv, off);
            const int oi = __shfl_xor_sync(FULL_MASK, bi, off);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        const double best = __shfl_sync(FULL_MASK, bv, 0);
        const int piv = __shfl_sync(FULL_MASK, bi, 0);
        if (!(best > 1e-12)) {
            ok = false;
            break;
        }
        if (piv != c) {
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                const double rc = __shfl_sync(FULL_MASK, R[j], c), rp = __shfl_sync(FULL_MASK, R[j], piv);
                if (lane == c) R[j] = rp;
                else if (lane == piv) R[j] = rc;
            }
        }
        double P[9];
#pragma unroll
        for (int j = c; j < 9; ++j) P[j] = __shfl_sync(FULL_MASK, R[j], c);
        if (lane > c && lane < 8) {
            const double f = R[c] / P[c];
#pragma unroll
            for (int j = c; j < 9; ++j) R[j] = R[j] - f * P[j];
        }
    }
    if (!ok) return false;
    h[8] = 1.0;
#pragma unroll
    for (int c = 7; c >= 0; --c) {
        double hc = 0.0;
        if (lane == c) {
            double s = R[8];
#pragma unroll
            for (int j = c + 1; j < 8; ++j) s = s + R[j] * h[j];
            hc = -s / R[c];
        }
        h[c] = __shfl_sync(FULL_MASK, hc, c);
    }
    return true;
}

struct RansacArgs {
    const double* p1;  // n x 2
    const double* p2;
    int n, n_hyp;
    const uint32_t* rnd;  // 4 * n_hyp raw MT19937 outputs
    double tq, two_sig2;
    int magsac, min_inliers;
    double* prep;     // [T1(9), T2inv(9), n1(3), n2(3)]
    double* p1n;      // n x 2 normalised
    double* p2n;
    double* hyp_H;    // n_hyp x 9
    double* score;    // n_hyp
    int* idx;         // n scratch indices
    uint8_t* mask;    // n output
    double* H_out;    // 9
    int* info;        // [n_inliers, best_i, stage]
    const int* n_dev; // if set: the point count on the device (n is then the capacity)
};

// The point count of a launch: n, or the device count clamped to 0..n.
// Fewer than 4 points leave no homography to fit: the kernels then write an
// empty result (info = 0, 0, 0) instead of sampling.
__device__ __forceinline__ int ransac_count(const RansacArgs& a) {
    if (!a.n_dev) return a.n;
    const int c = *a.n_dev;
    return c < 0 ? 0 : (c > a.n ? a.n : c);
}

__global__ void __launch_bounds__(RT) k_ransac_prep(const RansacArgs args) {
    __shared__ double sh[4][RT];
    __shared__ double red[4];
    RansacArgs a = args;
    a.n = ransac_count(args);
    if (a.n < 4) return;
    Norm n1, n2;
    hartley2(a.p1, a.p2, nullptr, a.n, sh, red, n1, n2);
    for (int i = threadIdx.x; i < a.n; i += RT) {
        a.p1n[2 * i] = nrm(n1.s, n1.cx, a.p1[2 * i]);
        a.p1n[2 * i + 1] = nrm(n1.s, n1.cy, a.p1[2 * i + 1]);
        a.p2n[2 * i] = nrm(n2.s, n2.cx, a.p2[2 * i]);
        a.p2n[2 * i + 1] = nrm(n2.s, n2.cy, a.p2[2 * i + 1]);
    }
    if (threadIdx.x == 0) {
        norm_mats(n1, n2, a.prep, a.prep + 9);
        a.prep[18] = n1.s; a.prep[19] = n1.cx; a.prep[20] = n1.cy;
        a.prep[21] = n2.s; a.prep[22] = n2.cx; a.prep[23] = n2.cy;
    }
}

// One warp per hypothesis: solve, denormalise, score all points
// (lane-strided partial sums, then the warp tree 16, 8, 4, 2, 1).
__global__ void __launch_bounds__(256) k_ransac_hyp(const RansacArgs args) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    RansacArgs a = args;
    a.n = ransac_count(args);
    if (warp >= a.n_hyp) return;
    if (a.n < 4) {
        if (lane == 0) a.score[warp] = -INFINITY;
        return;
    }
    double x1 = 0.0, y1 = 0.0, x2 = 0.0, y2 = 0.0;
    if (lane < 8) {
        const int i = (int)(a.rnd[4 * warp + (lane >> 1)] % (uint32_t)a.n);
        x1 = a.p1n[2 * i];
        y1 = a.p1n[2 * i + 1];
        x2 = a.p2n[2 * i];
        y2 = a.p2n[2 * i + 1];
    }
    double hn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, H[9], Hi[9];
    const bool ok = null_vector_warp(x1, y1, x2, y2, hn);
    if (!ok)
        for (int k = 0; k < 9; ++k) hn[k] = 0.0;
    denormalise(hn, a.prep, a.prep + 9, H);
    inv3_guarded(H, Hi, 1e-12);
    double part = 0.0;
    if (ok) {
        for (int i = lane; i < a.n; i += 32) {
            const double e = sym_err(H, Hi, a.p1[2 * i], a.p1[2 * i + 1], a.p2[2 * i], a.p2[2 * i + 1], true);
            if (a.magsac)
                part = part + ransac_exp(-e / a.two_sig2);
            else
                part = part + (e < a.tq ? 1.0 : 0.0);
        }
    }
    for (int o = 16; o > 0; o >>= 1) part = part + __shfl_down_sync(FULL_MASK, part, o);
    if (lane == 0) {
        a.score[warp] = ok ? part : -INFINITY;
        for (int k = 0; k < 9; ++k) a.hyp_H[9 * warp + k] = H[k];
    }
}

// Smallest-eigenvalue eigenvector of the symmetric 9x9 M (row-major, shared
// memory) by parallel Jacobi, run by warp 0 (V: shared 9x9 eigenvectors).
// Round-robin ordering of the 36 index pairs: round r = 0..8 rotates the 4
// disjoint pairs {(r+i) mod 9, (r-i) mod 9}, i = 1..4 (p < q); index r rests.
// The 4 angles of a round come from the matrix at the start of the round,
// then all column rotations are applied, then all row rotations (exact, as
// the pairs are disjoint).  Only pairs with |a_pq| > tol = 2^-52 trace
// (the trace summed in index order) rotate; sweeps stop once no upper
// off-diagonal element exceeds tol, at 15 at most.  Returns the index of the
// smallest diagonal element (lowest on ties).
__device__ int jacobi9_smallest(double (*M)[9], double (*V)[9]) {
    __shared__ double s_cs[4][2];
    __shared__ int s_pq[4][2];
    __shared__ int s_act[4];
    __shared__ int s_best;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        for (int it = lane; it < 81; it += 32) V[it / 9][it % 9] = (it / 9 == it % 9) ? 1.0 : 0.0;
        double tr = 0.0;
        for (int k = 0; k < 9; ++k) tr = tr + M[k][k];
        const double tol = tr * 0x1p-52;
        __syncwarp();
        for (int sweep = 0; sweep < 15; ++sweep) {
            // no upper off-diagonal element above tol -> converged
            bool nz = false;
            for (int it = lane; it < 81; it += 32) {
                const int r = it / 9, c = it % 9;
                if (c > r && fabs(M[r][c]) > tol) nz = true;
            }
            if (!__any_sync(FULL_MASK, nz)) break;
            for (int rnd = 0; rnd < 9; ++rnd) {
                if (lane < 4) {
                    const int a = (rnd + lane + 1) % 9, bb = (rnd + 9 - lane - 1) % 9;
                    const int p = a < bb ? a : bb, q = a < bb ? bb : a;
                    s_pq[lane][0] = p;
                    s_pq[lane][1] = q;
                    const double apq = M[p][q];
                    int act = 0;
                    if (fabs(apq) > tol) {
                        const double app = M[p][p], aqq = M[q][q];
                        const double theta = (aqq - app) / (2.0 * apq);
                        const double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                        const double c = 1.0 / sqrt(tt * tt + 1.0);
                        s_cs[lane][0] = c;
                        s_cs[lane][1] = tt * c;
                        act = 1;
                    }
                    s_act[lane] = act;
                }
                __syncwarp();
                // column rotations: item = (pair j, row k)
                for (int it = lane; it < 36; it += 32) {
                    const int j = it / 9, k = it % 9;
                    if (s_act[j]) {
                        const int p = s_pq[j][0], q = s_pq[j][1];
                        const double c = s_cs[j][0], s = s_cs[j][1];
                        const double mkp = M[k][p], mkq = M[k][q];
                        M[k][p] = c * mkp - s * mkq;
                        M[k][q] = s * mkp + c * mkq;
                    }
                }
                __syncwarp();
                // row rotations and the eigenvector columns
                for (int it = lane; it < 36; it += 32) {
                    const int j = it / 9, k = it % 9;
                    if (s_act[j]) {
                        const int p = s_pq[j][0], q = s_pq[j][1];
                        const double c = s_cs[j][0], s = s_cs[j][1];
                        const double mpk = M[p][k], mqk = M[q][k];
                        M[p][k] = c * mpk - s * mqk;
                        M[q][k] = s * mpk + c * mqk;
                        const double vkp = V[k][p], vkq = V[k][q];
                        V[k][p] = c * vkp - s * vkq;
                        V[k][q] = s * vkp + c * vkq;
                    }
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            int best = 0;
            for (int k = 1; k < 9; ++k)
                if (M[k][k] < M[best][best]) best = k;
            s_best = best;
        }
    }
    __syncthreads();
    return s_best;
}

// Least-squares homography of the points idx[0..m): Hartley normalisation of
// the subset, A^T A accumulated in a fixed order (contiguous chunks per
// thread, then a pairwise tree over the RT partials), its smallest-eigenvalue
// eigenvector by jacobi9_smallest, denormalised (pysift/core.py:2959-2981).
__device__ void dlt_refit(const double* p1, const double* p2, const int* idx, int m, double* H, double* sh,
                          double* s_M) {
    constexpr int NB = 9;  // tree sums run 9 at a time
    __shared__ double s_part[NB][RT];
    __shared__ double s_Mj[9][9], s_Vj[9][9];
    __shared__ double s_red[NB];
    Norm n1, n2;
    hartley2(p1, p2, idx, m, s_part, s_red, n1, n2);
    double acc[45];
    for (int k = 0; k < 45; ++k) acc[k] = 0.0;
    const int chunk = (m + RT - 1) / RT;
    const int b = threadIdx.x * chunk, e = min(m, b + chunk);
    for (int i = b; i < e; ++i) {
        const int k = idx[i];
        const double x1 = nrm(n1.s, n1.cx, p1[2 * k]), y1 = nrm(n1.s, n1.cy, p1[2 * k + 1]);
        const double x2 = nrm(n2.s, n2.cx, p2[2 * k]), y2 = nrm(n2.s, n2.cy, p2[2 * k + 1]);
        const double re[9] = {-x1, -y1, -1.0, 0.0, 0.0, 0.0, x2 * x1, x2 * y1, x2};
        const double ro[9] = {0.0, 0.0, 0.0, -x1, -y1, -1.0, y2 * x1, y2 * y1, y2};
        int t = 0;
#pragma unroll
        for (int r = 0; r < 9; ++r)
#pragma unroll
            for (int c = r; c < 9; ++c, ++t) acc[t] = (acc[t] + re[r] * re[c]) + ro[r] * ro[c];
    }
#pragma unroll
    for (int t0 = 0; t0 < 45; t0 += NB) {
        double vv[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) vv[u] = acc[t0 + u];
        block_tree_sums<NB>(vv, s_part, s_M + t0);
    }
    for (int it = threadIdx.x; it < 45; it += RT) {
        // upper-triangle index it -> (r, c)
        int r = 0, rem = it;
        while (rem >= 9 - r) {
            rem -= 9 - r;
            ++r;
        }
        const int c = r + rem;
        s_Mj[r][c] = s_M[it];
        s_Mj[c][r] = s_M[it];
    }
    __syncthreads();
    const int best = jacobi9_smallest(s_Mj, s_Vj);
    if (threadIdx.x == 0) {
        double hn[9], T1[9], T2inv[9];
        for (int k = 0; k < 9; ++k) hn[k] = s_Vj[k][best];
        norm_mats(n1, n2, T1, T2inv);
        double t9[9];
        mat3_mul(T2inv, hn, t9);
        mat3_mul(t9, T1, H);
        const double s = H[8];
        for (int k = 0; k < 9; ++k) H[k] = H[k] / s;
    }
    __syncthreads();
}

// Compacts flags[0..n) into idx (in order); returns the count (all threads).
__device__ int compact_mask(const uint8_t* flags, int n, int* idx, int* shi) {
    int base = 0;
    for (int c0 = 0; c0 < n; c0 += RT) {
        const int i = c0 + threadIdx.x;
        const int f = (i < n && flags[i]) ? 1 : 0;
        int tot;
        const int pos = base + block_excl_scan(f, &tot, shi);
        if (f) idx[pos] = i;
        base += tot;
    }
    return base;
}

// Best hypothesis (first maximum), its inlier set, LO refits (pysift/core.py:3060-3092).
__global__ void __launch_bounds__(RT) k_ransac_select(const RansacArgs args) {
    RansacArgs a = args;
    a.n = ransac_count(args);
    if (a.n < 4) {
        if (threadIdx.x < 9) a.H_out[threadIdx.x] = 0.0;
        if (threadIdx.x < 3) a.info[threadIdx.x] = 0;
        return;
    }
    __shared__ double sh[RT];
    __shared__ int shi[33];
    __shared__ double s_M[45];
    __shared__ double s_H[9], s_Hi[9], s_H1[9];
    __shared__ int s_best;
    __shared__ double s_bscore[RT / 32];
    __shared__ int s_bidx[RT / 32];
    // argmax, lowest index on ties
    double bs = -INFINITY;
    int bi = 0x7fffffff;
    for (int h = threadIdx.x; h < a.n_hyp; h += RT) {
        const double v = a.score[h];
        if (v > bs || (v == bs && h < bi)) {
            bs = v;
            bi = h;
        }
    }
    // (score desc, index asc) is a total order on the non-NaN candidates the
    // threads kept, so a shuffle tree gives the serial scan's choice
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(FULL_MASK, bs, o);
        const int oi = __shfl_xor_sync(FULL_MASK, bi, o);
        if (ov > bs || (ov == bs && oi < bi)) {
            bs = ov;
            bi = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        s_bscore[threadIdx.x >> 5] = bs;
        s_bidx[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double B = s_bscore[0];
        int I = s_bidx[0];
        for (int t = 1; t < RT / 32; ++t)
            if (s_bscore[t] > B || (s_bscore[t] == B && s_bidx[t] < I)) {
                B = s_bscore[t];
                I = s_bidx[t];
            }
        s_best = (I == 0x7fffffff) ? 0 : I;
        for (int k = 0; k < 9; ++k) s_H[k] = a.hyp_H[9 * s_best + k];
        inv3_guarded(s_H, s_Hi, 1e-12);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < a.n; i += RT)
        a.mask[i] = sym_err(s_H, s_Hi, a.p1[2 * i], a.p1[2 * i + 1], a.p2[2 * i], a.p2[2 * i + 1], true) < a.tq;
    __syncthreads();
    const int nb = compact_mask(a.mask, a.n, a.idx, shi);
    int stage = 0, n_final = nb;
    if (nb >= a.min_inliers) {
        dlt_refit(a.p1, a.p2, a.idx, nb, s_H1, sh, s_M);
        if (threadIdx.x == 0) inv3_guarded(s_H1, s_Hi, 0.0);
        __syncthreads();
        // reclassify with H1 into idx via a second flag pass (mask keeps the hypothesis set for now)
        int base = 0;
        for (int c0 = 0; c0 < a.n; c0 += RT) {
            const int i = c0 + threadIdx.x;
            int f = 0;
            if (i < a.n) f = sym_err(s_H1, s_Hi, a.p1[2 * i], a.p1[2 * i + 1], a.p2[2 * i], a.p2[2 * i + 1], false) < a.tq;
            int tot;
            const int pos = base + block_excl_scan(f, &tot, shi);
            if (f) a.idx[pos] = i;
            base += tot;
        }
        const int n2 = base;
        if (n2 >= a.min_inliers) {
            dlt_refit(a.p1, a.p2, a.idx, n2, s_H, sh, s_M);
            // mask = reclassified set
            for (int i = threadIdx.x; i < a.n; i += RT) a.mask[i] = 0;
            __syncthreads();
            for (int k = threadIdx.x; k < n2; k += RT) a.mask[a.idx[k]] = 1;
            stage = 2;
            n_final = n2;
        } else {
            if (threadIdx.x < 9) s_H[threadIdx.x] = s_H1[threadIdx.x];
            stage = 1;
        }
        __syncthreads();
    }
    if (threadIdx.x < 9) a.H_out[threadIdx.x] = s_H[threadIdx.x];
    if (threadIdx.x == 0) {
        a.info[0] = n_final;
        a.info[1] = s_best;
        a.info[2] = stage;
    }
}

// Plain DLT on all points (the reference's preliminary estimate, core.py:3753).
__global__ void __launch_bounds__(RT) k_dlt_all(const double* p1, const double* p2, int n, int* idx, double* H_out) {
    __shared__ double sh[RT];
    __shared__ double s_M[45];
    __shared__ double s_H[9];
    for (int i = threadIdx.x; i < n; i += RT) idx[i] = i;
    __syncthreads();
    dlt_refit(p1, p2, idx, n, s_H, sh, s_M);
    if (threadIdx.x < 9) H_out[threadIdx.x] = s_H[threadIdx.x];
}

// ---------------------------------------------------------------------------
// Descriptor preparation for the stitch matcher (pysift/core.py:2877-2888,
// 2703-2743): L2-normalise (+1e-7), optional PCA projection, L2-normalise,
// round to fp16.  Norms sum squares in groups of 32 dimensions (warp tree
// 16, 8, 4, 2, 1) and the groups in order; the projection is a fmaf chain
// over k ascending of (d_k - mean_k) * proj[k][c].
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_tree(float v) {
    v += __shfl_down_sync(FULL_MASK, v, 16);
    v += __shfl_down_sync(FULL_MASK, v, 8);
    v += __shfl_down_sync(FULL_MASK, v, 4);
    v += __shfl_down_sync(FULL_MASK, v, 2);
    v += __shfl_down_sync(FULL_MASK, v, 1);
    return __shfl_sync(FULL_MASK, v, 0);
}

// one warp per row; D <= 128 (D % 32 == 0)
__global__ void k_l2_normalize(const float* __restrict__ in, int n, int D, float* __restrict__ out) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* r = in + (size_t)row * D;
    float v[4];
    float ss = 0.0f;
    for (int g = 0; g < D / 32; ++g) {
        v[g] = r[g * 32 + lane];
        const float w = warp_tree(v[g] * v[g]);
        ss = (g == 0) ? w : ss + w;
    }
    const float den = sqrtf(ss) + 1e-7f;
    for (int g = 0; g < D / 32; ++g) out[(size_t)row * D + g * 32 + lane] = v[g] / den;
}

// Projection (D -> P), normalisation and fp16 rounding of 64-row blocks.
// Each output is the fmaf chain over k ascending of (x_k - mean_k) * proj[k][c];
// a thread computes a 4 x 4 register block of outputs from shared-memory
// copies of the centred rows and of the projection.  Row norms sum squares
// in groups of 32 outputs (warp tree 16, 8, 4, 2, 1) and the groups in order.
constexpr int PJ_ROWS = 64;
constexpr int PJ_T = 256;

// OUT_F32: the normalised float32 rows (for the int8 matcher) instead of fp16
template <int D, int P, bool OUT_F32 = false>
__global__ void __launch_bounds__(PJ_T) k_pca_project_f16(const float* __restrict__ in, int n,
                                                         const float* __restrict__ mean, const float* __restrict__ proj,
                                                         void* __restrict__ out_v) {
    extern __shared__ float pj_smem[];
    float* s_proj = pj_smem;                  // D x P
    float* s_x = s_proj + D * P;              // PJ_ROWS x (D + 1), centred
    float* s_y = s_x + PJ_ROWS * (D + 1);     // PJ_ROWS x (P + 1), projected
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * PJ_ROWS;
    for (int q = tid; q < D * P; q += PJ_T) s_proj[q] = proj[q];
    for (int q = tid; q < PJ_ROWS * D; q += PJ_T) {
        const int r = q / D, k = q - r * D;
        s_x[r * (D + 1) + k] = (r0 + r < n) ? in[(size_t)(r0 + r) * D + k] - mean[k] : 0.0f;
    }
    __syncthreads();
    constexpr int CT = P / 4;                // threads along the outputs
    constexpr int RT_ = PJ_T / CT;           // threads along the rows
    constexpr int RPT = PJ_ROWS / RT_;       // rows per thread
    const int tc = tid % CT, tr = tid / CT;
    float acc[RPT][4];
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
#pragma unroll 4
    for (int k = 0; k < D; ++k) {
        float pv[4], xv[RPT];
#pragma unroll
        for (int j = 0; j < 4; ++j) pv[j] = s_proj[k * P + tc + CT * j];
#pragma unroll
        for (int i = 0; i < RPT; ++i) xv[i] = s_x[(tr + RT_ * i) * (D + 1) + k];
#pragma unroll
        for (int i = 0; i < RPT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(xv[i], pv[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) s_y[(tr + RT_ * i) * (P + 1) + tc + CT * j] = acc[i][j];
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5;
    for (int r = warp; r < PJ_ROWS; r += PJ_T / 32) {
        if (r0 + r >= n) break;
        float pvv[P / 32];
        float ss = 0.0f;
#pragma unroll
        for (int g = 0; g < P / 32; ++g) {
            pvv[g] = s_y[r * (P + 1) + g * 32 + lane];
            const float w = warp_tree(pvv[g] * pvv[g]);
            ss = (g == 0) ? w : ss + w;
        }
        const float den = sqrtf(ss) + 1e-7f;
#pragma unroll
        for (int g = 0; g < P / 32; ++g) {
            const float y = pvv[g] / den;
            if (OUT_F32)
                static_cast<float*>(out_v)[(size_t)(r0 + r) * P + g * 32 + lane] = y;
            else
                static_cast<uint16_t*>(out_v)[(size_t)(r0 + r) * P + g * 32 + lane] = __half_as_ushort(__float2half_rn(y));
        }
    }
}

__global__ void k_to_f16(const float* __restrict__ in, size_t n, uint16_t* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __half_as_ushort(__float2half_rn(in[i]));
}

// PCA statistics of the stacked normalised sets, in float64 over fixed
// 128-row chunks: each chunk is summed sequentially, then the chunk partials
// in chunk order.  mean = (sum of rows) / n, rounded to float32; covariance =
// (sum of products of the float32 centred values) / n.
constexpr int PCA_CHUNK = 128;

__global__ void k_pca_mean_part(const float* __restrict__ x, int n, int D, double* __restrict__ part) {
    const int k = threadIdx.x, c = blockIdx.x;
    if (k >= D) return;
    const int i0 = c * PCA_CHUNK, i1 = min(n, i0 + PCA_CHUNK);
    double s = 0.0;
    for (int i = i0; i < i1; ++i) s = s + (double)x[(size_t)i * D + k];
    part[(size_t)c * D + k] = s;
}

__global__ void k_pca_mean_final(const double* __restrict__ part, int nchunks, int n, int D, float* __restrict__ mean) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D) return;
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s = s + part[(size_t)c * D + k];
    mean[k] = (float)(s / (double)n);
}

// block = (chunk, 32 x 32 tile of the covariance); thread = 4 entries
__global__ void __launch_bounds__(256) k_pca_cov_part(const float* __restrict__ x, int n, int D,
                                                     const float* __restrict__ mean, double* __restrict__ part) {
    __shared__ float s_a[PCA_CHUNK][33], s_b[PCA_CHUNK][33];
    const int c = blockIdx.x, tk = blockIdx.y, tl = blockIdx.z;
    if (tl < tk) return;
    const int i0 = c * PCA_CHUNK, m = min(n - i0, PCA_CHUNK);
    for (int q = threadIdx.x; q < PCA_CHUNK * 32; q += 256) {
        const int i = q >> 5, j = q & 31;
        const int k = tk * 32 + j, l = tl * 32 + j;
        s_a[i][j] = (i < m && k < D) ? x[(size_t)(i0 + i) * D + k] - mean[k] : 0.0f;
        s_b[i][j] = (i < m && l < D) ? x[(size_t)(i0 + i) * D + l] - mean[l] : 0.0f;
    }
    __syncthreads();
    const int jl = threadIdx.x & 31, jk0 = threadIdx.x >> 5;  // entries (jk0 + 8 u, jl)
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < m; ++i) {
        const double bv = (double)s_b[i][jl];
#pragma unroll
        for (int u = 0; u < 4; ++u) s[u] = s[u] + (double)s_a[i][jk0 + 8 * u] * bv;
    }
    const size_t DD = (size_t)D * D;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int k = tk * 32 + jk0 + 8 * u, l = tl * 32 + jl;
        if (k < D && l < D) part[(size_t)c * DD + (size_t)k * D + l] = s[u];
    }
}

__global__ void k_pca_cov_final(const double* __restrict__ part, int nchunks, int n, int D, double* __restrict__ cov) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= D * D) return;
    const int k = q / D, l = q - k * D;
    if (l < k) return;
    const size_t DD = (size_t)D * D;
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s = s + part[(size_t)c * DD + q];
    const double v = s / (double)n;
    cov[(size_t)k * D + l] = v;
    cov[(size_t)l * D + k] = v;
}

struct RansacLayout {
    size_t off_prep, off_p1n, off_p2n, off_hyp, off_score, off_idx, total;
};

// PCA basis (pysift/core.py:2729-2736: cp.linalg.eigh of the covariance,
// the eigenvectors of the P largest eigenvalues).  Round-robin parallel
// cyclic Jacobi on the D x D float64 covariance in one CTA (D even, <= 128):
// round r = 0..D-2 rotates the D/2 disjoint pairs {D-1, r} and
// {(r+i) mod (D-1), (r-i) mod (D-1)}, i = 1..D/2-1 (p < q); every angle comes
// from the matrix at the start of the round and only pairs with
// |a_pq| > tol = 2^-60 trace rotate; all column rotations, then all row
// rotations and the eigenvector columns.  Sweeps stop once no upper
// off-diagonal element exceeds tol (60 at most).  The basis is the
// eigenvectors of the last P indices in (eigenvalue asc, index asc) order,
// in that order (as eigh's v[:, -P:]), rounded to float32.  A lives in
// shared memory, V (stored transposed, so that its column rotations are
// coalesced row rotations) in the caller's workspace.
__device__ __forceinline__ void pca_pair(int D, int rnd, int i, int* p, int* q) {
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

constexpr int PCA_BT = 1024;
constexpr int PCA_IT = 4;  // items per thread loaded together (a pass has 128 x 64 / 1024 = 8)

// DC: the dimension as a compile-time constant (64, 128), or 0 for any even
// D <= 128 given at run time (the same operations either way).
template <int DC>
__global__ void __launch_bounds__(PCA_BT) k_pca_basis(const double* __restrict__ cov, int D_rt, int P,
                                                       double* __restrict__ V, float* __restrict__ proj,
                                                       int* __restrict__ sweeps_out) {
    const int D = DC ? DC : D_rt;
    extern __shared__ __align__(16) double A[];  // D x D
    __shared__ double s_cs[64][2];
    __shared__ int s_pq[64][2];
    __shared__ int s_act[64];
    __shared__ int s_order[128];
    __shared__ double s_tol;
    const int tid = threadIdx.x, nt = blockDim.x, npair = D / 2;
    for (int it = tid; it < D * D; it += nt) {
        A[it] = cov[it];
        V[it] = (it / D == it % D) ? 1.0 : 0.0;
    }
    __syncthreads();
    if (tid == 0) {
        double tr = 0.0;
        for (int k = 0; k < D; ++k) tr = tr + A[k * D + k];
        s_tol = tr * 0x1p-60;
    }
    __syncthreads();
    const double tol = s_tol;
    int sweep = 0;
    for (; sweep < 60; ++sweep) {
        int any = 0;
        for (int it = tid; it < D * D; it += nt) {
            const int r = it / D, c = it - r * D;
            if (c > r && fabs(A[it]) > tol) any = 1;
        }
        if (!__syncthreads_or(any)) break;
        for (int rnd = 0; rnd < D - 1; ++rnd) {
            if (tid < npair) {
                int p, q;
                pca_pair(D, rnd, tid, &p, &q);
                s_pq[tid][0] = p;
                s_pq[tid][1] = q;
                const double apq = A[p * D + q];
                int act = 0;
                if (fabs(apq) > tol) {
                    const double app = A[p * D + p], aqq = A[q * D + q];
                    const double theta = (aqq - app) / (2.0 * apq);
                    const double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    const double c = 1.0 / sqrt(tt * tt + 1.0);
                    s_cs[tid][0] = c;
                    s_cs[tid][1] = tt * c;
                    act = 1;
                }
                s_act[tid] = act;
            }
            __syncthreads();
            // each pass: a thread's items it = tid + (g + m) nt, PCA_IT at a
            // time, load all of a group first, then rotate and store, so a
            // pass costs two memory round trips
            // column rotations: item = (row k, pair j), pairs adjacent
            for (int g = 0; g * nt < D * npair; g += PCA_IT) {
                double x0[PCA_IT], x1[PCA_IT];
#pragma unroll
                for (int m = 0; m < PCA_IT; ++m) {
                    const int it = tid + (g + m) * nt, k = it / npair, j = it - k * npair;
                    if (it < D * npair && s_act[j]) {
                        x0[m] = A[k * D + s_pq[j][0]];
                        x1[m] = A[k * D + s_pq[j][1]];
                    }
                }
#pragma unroll
                for (int m = 0; m < PCA_IT; ++m) {
                    const int it = tid + (g + m) * nt, k = it / npair, j = it - k * npair;
                    if (it < D * npair && s_act[j]) {
                        const double c = s_cs[j][0], s = s_cs[j][1];
                        const double mkp = x0[m], mkq = x1[m];
                        A[k * D + s_pq[j][0]] = c * mkp - s * mkq;
                        A[k * D + s_pq[j][1]] = s * mkp + c * mkq;
                    }
                }
            }
            __syncthreads();
            // row rotations and eigenvector columns: item = (pair j, column k),
            // columns adjacent (V^T[p][k] is V[k][p])
            for (int g = 0; g * nt < D * npair; g += PCA_IT) {
                double x0[PCA_IT], x1[PCA_IT], y0[PCA_IT], y1[PCA_IT];
#pragma unroll
                for (int m = 0; m < PCA_IT; ++m) {
                    const int it = tid + (g + m) * nt;
                    if (it < npair * D) {
                        const int j = it / D, k = it - j * D;
                        if (s_act[j]) {
                            x0[m] = A[s_pq[j][0] * D + k];
                            x1[m] = A[s_pq[j][1] * D + k];
                        }
                        if (s_act[j]) {  // V is kept transposed: rows p, q of V^T, columns adjacent
                            y0[m] = V[s_pq[j][0] * D + k];
                            y1[m] = V[s_pq[j][1] * D + k];
                        }
                    }
                }
#pragma unroll
                for (int m = 0; m < PCA_IT; ++m) {
                    const int it = tid + (g + m) * nt;
                    if (it < npair * D) {
                        const int j = it / D, k = it - j * D;
                        if (s_act[j]) {
                            const double c = s_cs[j][0], s = s_cs[j][1];
                            const double mpk = x0[m], mqk = x1[m];
                            A[s_pq[j][0] * D + k] = c * mpk - s * mqk;
                            A[s_pq[j][1] * D + k] = s * mpk + c * mqk;
                        }
                        if (s_act[j]) {
                            const double c = s_cs[j][0], s = s_cs[j][1];
                            const double vkp = y0[m], vkq = y1[m];
                            V[s_pq[j][0] * D + k] = c * vkp - s * vkq;
                            V[s_pq[j][1] * D + k] = s * vkp + c * vkq;
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    if (tid < D) {
        const double v = A[tid * D + tid];
        int rk = 0;
        for (int j = 0; j < D; ++j) {
            const double w = A[j * D + j];
            if (w < v || (w == v && j < tid)) ++rk;
        }
        s_order[rk] = tid;
    }
    __syncthreads();
    for (int it = tid; it < D * P; it += nt) {
        const int k = it / P, c = it - k * P;
        proj[it] = (float)V[s_order[D - P + c] * D + k];
    }
    if (tid == 0 && sweeps_out) *sweeps_out = sweep;
}

static RansacLayout ransac_layout(int n, int n_hyp) {
    RansacLayout l;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t r = off;
        off = align_up(off + bytes, 256);
        return r;
    };
    l.off_prep = take(32 * sizeof(double));
    l.off_p1n = take((size_t)n * 2 * sizeof(double));
    l.off_p2n = take((size_t)n * 2 * sizeof(double));
    l.off_hyp = take((size_t)n_hyp * 9 * sizeof(double));
    l.off_score = take((size_t)n_hyp * sizeof(double));
    l.off_idx = take((size_t)n * sizeof(int));
    l.total = off;
    return l;
}

template <int D, int P, bool OUT_F32>
static int launch_project(const float* x, int n, const float* mean, const float* proj, void* out, cudaStream_t st) {
    const size_t smem = ((size_t)D * P + (size_t)PJ_ROWS * (D + 1) + (size_t)PJ_ROWS * (P + 1)) * sizeof(float);
    PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_pca_project_f16<D, P, OUT_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    k_pca_project_f16<D, P, OUT_F32><<<ceil_div(n, PJ_ROWS), PJ_T, smem, st>>>(x, n, mean, proj, out);
    PYSIFT_LAUNCH_CHECK("k_pca_project_f16");
    return PYSIFT_OK;
}

template <bool OUT_F32>
static int project_any(const float* x, int n, int D, const float* mean, const float* proj, int P, void* out,
                       cudaStream_t st) {
    if (D == 128 && P == 64) return launch_project<128, 64, OUT_F32>(x, n, mean, proj, out, st);
    if (D == 128 && P == 32) return launch_project<128, 32, OUT_F32>(x, n, mean, proj, out, st);
    if (D == 128 && P == 128) return launch_project<128, 128, OUT_F32>(x, n, mean, proj, out, st);
    if (D == 64 && P == 64) return launch_project<64, 64, OUT_F32>(x, n, mean, proj, out, st);
    return launch_project<64, 32, OUT_F32>(x, n, mean, proj, out, st);
}

// Symmetric int8 quantisation per row (pysift/core.py:2902-2905), one warp a
// row: scale = 127 / (max |x| + 1e-7) evaluated as torch evaluates a scalar
// divided by a tensor, reciprocal(max |x| + 1e-7) * 127, all in float32;
// q = trunc(clamp(x * scale, -127, 127)).
__global__ void k_quantize_i8_rows(const float* __restrict__ in, int n, int D, int8_t* __restrict__ q,
                                   float* __restrict__ scale) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* r = in + (size_t)row * D;
    float v[4];
    float amax = 0.0f;
    for (int g = 0; g < D / 32; ++g) {
        v[g] = r[g * 32 + lane];
        amax = fmaxf(amax, fabsf(v[g]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(FULL_MASK, amax, o));
    const float s = __fmul_rn(__frcp_rn(__fadd_rn(amax, 1e-7f)), 127.0f);
    for (int g = 0; g < D / 32; ++g) {
        float y = __fmul_rn(v[g], s);
        y = fminf(fmaxf(y, -127.0f), 127.0f);
        q[(size_t)row * D + g * 32 + lane] = (int8_t)(int)y;
    }
    if (lane == 0) scale[row] = s;
}

}  // namespace pysift

using namespace pysift;

extern "C" {

void pysift_mt19937_u32(uint32_t seed, uint32_t* out, int64_t n) {
    uint32_t mt[624];
    mt[0] = seed;
    for (int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
    int idx = 624;
    for (int64_t k = 0; k < n; ++k) {
        if (idx >= 624) {
            for (int i = 0; i < 624; ++i) {
                const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
                mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
            }
            idx = 0;
        }
        uint32_t y = mt[idx++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        out[k] = y;
    }
}

int pysift_ransac_workspace_size(int32_t n, int32_t n_hyp, size_t* bytes) {
    PYSIFT_CHECK_ARG(bytes && n >= 0 && n_hyp >= 1, "bad arguments");
    *bytes = ransac_layout(n, n_hyp).total;
    return PYSIFT_OK;
}

static int run_ransac(const double* pts1, const double* pts2, int32_t n, const int32_t* n_dev,
                      const uint32_t* rand_u32, int32_t n_hyp, double inlier_thresh, double sigma_max,
                      int32_t magsac, int32_t min_inliers, void* workspace, size_t workspace_bytes, double* H_out,
                      uint8_t* mask_out, int32_t* info, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(pts1 && pts2 && rand_u32 && workspace && H_out && mask_out && info, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n_hyp >= 1 && inlier_thresh > 0.0 && sigma_max > 0.0, "bad RANSAC parameters");
    RansacLayout l = ransac_layout(n, n_hyp);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    RansacArgs a;
    a.p1 = pts1;
    a.p2 = pts2;
    a.n = n;
    a.n_dev = n_dev;
    a.n_hyp = n_hyp;
    a.rnd = rand_u32;
    a.tq = inlier_thresh * inlier_thresh;
    a.two_sig2 = 2.0 * (sigma_max * sigma_max);
    a.magsac = magsac;
    a.min_inliers = min_inliers;
    char* ws = static_cast<char*>(workspace);
    a.prep = reinterpret_cast<double*>(ws + l.off_prep);
    a.p1n = reinterpret_cast<double*>(ws + l.off_p1n);
    a.p2n = reinterpret_cast<double*>(ws + l.off_p2n);
    a.hyp_H = reinterpret_cast<double*>(ws + l.off_hyp);
    a.score = reinterpret_cast<double*>(ws + l.off_score);
    a.idx = reinterpret_cast<int*>(ws + l.off_idx);
    a.mask = mask_out;
    a.H_out = H_out;
    a.info = info;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_ransac_prep<<<1, RT, 0, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_ransac_prep");
    k_ransac_hyp<<<ceil_div(n_hyp * 32, 256), 256, 0, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_ransac_hyp");
    k_ransac_select<<<1, RT, 0, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_ransac_select");
    return PYSIFT_OK;
}

int pysift_ransac(const double* pts1, const double* pts2, int32_t n, const uint32_t* rand_u32, int32_t n_hyp,
                  double inlier_thresh, double sigma_max, int32_t magsac, int32_t min_inliers, void* workspace,
                  size_t workspace_bytes, double* H_out, uint8_t* mask_out, int32_t* info, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(n >= 4, "Need >= 4 correspondences, got %d", n);
    return run_ransac(pts1, pts2, n, nullptr, rand_u32, n_hyp, inlier_thresh, sigma_max, magsac, min_inliers,
                      workspace, workspace_bytes, H_out, mask_out, info, stream);
}

int pysift_ransac_count(const double* pts1, const double* pts2, const int32_t* n_dev, int32_t n_cap,
                        const uint32_t* rand_u32, int32_t n_hyp, double inlier_thresh, double sigma_max,
                        int32_t magsac, int32_t min_inliers, void* workspace, size_t workspace_bytes, double* H_out,
                        uint8_t* mask_out, int32_t* info, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(n_dev != nullptr, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n_cap >= 1, "bad capacity %d", n_cap);
    return run_ransac(pts1, pts2, n_cap, n_dev, rand_u32, n_hyp, inlier_thresh, sigma_max, magsac, min_inliers,
                      workspace, workspace_bytes, H_out, mask_out, info, stream);
}

int pysift_dlt_homography(const double* pts1, const double* pts2, int32_t n, int32_t* idx_scratch, double* H_out,
                          pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(pts1 && pts2 && idx_scratch && H_out, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n >= 4, "Need >= 4 correspondences, got %d", n);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_dlt_all<<<1, RT, 0, st>>>(pts1, pts2, n, idx_scratch, H_out);
    PYSIFT_LAUNCH_CHECK("k_dlt_all");
    return PYSIFT_OK;
}

int pysift_l2_normalize_rows(const float* in, int32_t n, int32_t D, float* out, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(in && out && n >= 0 && D > 0 && D <= 128 && D % 32 == 0, "bad arguments");
    if (n == 0) return PYSIFT_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_l2_normalize<<<ceil_div(n * 32, 256), 256, 0, st>>>(in, n, D, out);
    PYSIFT_LAUNCH_CHECK("k_l2_normalize");
    return PYSIFT_OK;
}

int pysift_pca_workspace_size(int32_t n, int32_t D, size_t* bytes) {
    PYSIFT_CHECK_ARG(bytes && n >= 1 && D > 0 && D <= 1024, "bad arguments");
    const size_t nchunks = (size_t)ceil_div(n, PCA_CHUNK);
    *bytes = nchunks * (size_t)D * sizeof(double) + nchunks * (size_t)D * D * sizeof(double);
    return PYSIFT_OK;
}

int pysift_pca_stats(const float* x, int32_t n, int32_t D, void* workspace, size_t workspace_bytes, float* mean,
                     double* cov, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(x && mean && cov && workspace && n >= 1 && D > 0 && D <= 1024, "bad arguments");
    size_t need = 0;
    pysift_pca_workspace_size(n, D, &need);
    if (workspace_bytes < need) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, need);
        return PYSIFT_ERR_WORKSPACE;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int nchunks = ceil_div(n, PCA_CHUNK);
    double* mpart = static_cast<double*>(workspace);
    double* cpart = mpart + (size_t)nchunks * D;
    k_pca_mean_part<<<nchunks, ceil_div(D, 32) * 32, 0, st>>>(x, n, D, mpart);
    PYSIFT_LAUNCH_CHECK("k_pca_mean_part");
    k_pca_mean_final<<<ceil_div(D, 128), 128, 0, st>>>(mpart, nchunks, n, D, mean);
    PYSIFT_LAUNCH_CHECK("k_pca_mean_final");
    k_pca_cov_part<<<dim3(nchunks, ceil_div(D, 32), ceil_div(D, 32)), 256, 0, st>>>(x, n, D, mean, cpart);
    PYSIFT_LAUNCH_CHECK("k_pca_cov_part");
    k_pca_cov_final<<<ceil_div(D * D, 256), 256, 0, st>>>(cpart, nchunks, n, D, cov);
    PYSIFT_LAUNCH_CHECK("k_pca_cov_final");
    return PYSIFT_OK;
}

int pysift_pca_basis_workspace_size(int32_t D, size_t* bytes) {
    PYSIFT_CHECK_ARG(bytes != nullptr, "bytes is NULL");
    PYSIFT_CHECK_ARG(D >= 2 && D <= 128 && (D & 1) == 0, "D must be even and <= 128");
    *bytes = align_up((size_t)D * D * sizeof(double), 256) + 256;
    return PYSIFT_OK;
}

int pysift_pca_basis(const double* cov, int32_t D, int32_t P, void* workspace, size_t workspace_bytes, float* proj,
                     int32_t* sweeps, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(cov && workspace && proj, "NULL pointer argument");
    PYSIFT_CHECK_ARG(D >= 2 && D <= 128 && (D & 1) == 0, "D must be even and <= 128");
    PYSIFT_CHECK_ARG(P >= 1 && P <= D, "P must be in 1..D");
    size_t need = 0;
    pysift_pca_basis_workspace_size(D, &need);
    if (workspace_bytes < need) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, need);
        return PYSIFT_ERR_WORKSPACE;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const size_t smem = (size_t)D * D * sizeof(double);
    int* sw = reinterpret_cast<int*>(static_cast<char*>(workspace) + align_up((size_t)D * D * sizeof(double), 256));
    double* V = static_cast<double*>(workspace);
    if (D == 128) {
        PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_pca_basis<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_pca_basis<128><<<1, PCA_BT, smem, st>>>(cov, D, P, V, proj, sw);
    } else if (D == 64) {
        PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_pca_basis<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_pca_basis<64><<<1, PCA_BT, smem, st>>>(cov, D, P, V, proj, sw);
    } else {
        PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_pca_basis<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_pca_basis<0><<<1, PCA_BT, smem, st>>>(cov, D, P, V, proj, sw);
    }
    PYSIFT_LAUNCH_CHECK("k_pca_basis");
    if (sweeps) PYSIFT_CUDA_TRY(cudaMemcpyAsync(sweeps, sw, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    return PYSIFT_OK;
}

int pysift_pca_project_f16(const float* x, int32_t n, int32_t D, const float* mean, const float* proj, int32_t P,
                           uint16_t* out, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(x && mean && proj && out && n >= 0, "bad arguments");
    PYSIFT_CHECK_ARG((D == 128 || D == 64) && (P == 32 || P == 64 || P == 128) && P <= D,
                     "unsupported sizes (D in {64, 128}, P in {32, 64, 128}, P <= D)");
    if (n == 0) return PYSIFT_OK;
    return project_any<false>(x, n, D, mean, proj, P, out, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_pca_project_f32(const float* x, int32_t n, int32_t D, const float* mean, const float* proj, int32_t P,
                           float* out, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(x && mean && proj && out && n >= 0, "bad arguments");
    PYSIFT_CHECK_ARG((D == 128 || D == 64) && (P == 32 || P == 64 || P == 128) && P <= D,
                     "unsupported sizes (D in {64, 128}, P in {32, 64, 128}, P <= D)");
    if (n == 0) return PYSIFT_OK;
    return project_any<true>(x, n, D, mean, proj, P, out, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_quantize_i8_rows(const float* x, int32_t n, int32_t D, int8_t* q, float* scale, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(x && q && scale && n >= 0, "bad arguments");
    PYSIFT_CHECK_ARG(D == 32 || D == 64 || D == 96 || D == 128, "D must be a multiple of 32, at most 128");
    if (n == 0) return PYSIFT_OK;
    k_quantize_i8_rows<<<ceil_div(n, 8), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, n, D, q, scale);
    PYSIFT_LAUNCH_CHECK("k_quantize_i8_rows");
    return PYSIFT_OK;
}

int pysift_to_f16(const float* in, int64_t n, uint16_t* out, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(in && out && n >= 0, "bad arguments");
    if (n == 0) return PYSIFT_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_to_f16<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, (size_t)n, out);
    PYSIFT_LAUNCH_CHECK("k_to_f16");
    return PYSIFT_OK;
}

}  // extern "C"
