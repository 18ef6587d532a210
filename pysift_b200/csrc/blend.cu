// blend.cu -- the reference's two-image composition on the GPU: gain
// compensation, seam cost, dynamic-programming seam, seam mask and the
// 6-level Laplacian (multi-band) blend (pysift/core.py:3286-3553, 3686-3714,
// 3794-3814), with no host synchronisation.
//
// Arithmetic follows the numpy / scipy.ndimage restatement (the algorithms
// cupyx implements): float32 images and elementwise ops without contraction;
// gaussian_filter(sigma = 1) and sobel as scipy's correlate1d does them
// (float64 sums, symmetric filters as w0 * x[i] + sum_k w_k (x[i-k] + x[i+k])
// from the outermost tap in, half-sample symmetric reflection, axis 0 then
// axis 1, float32 between the passes); zoom(order = 1) with the coordinate
// k * (in - 1) / (out - 1) and products ((v * w_row) * w_col) summed over the
// 2 x 2 corners in row-major order, in float64; the DP in float64 with
// numpy's first-minimum tie order.  Canonical choices: the gain means are
// exact (int64 sums / count); the seam-mask blur (cv2.GaussianBlur, sigma 3)
// is separable with the 25 float32 taps the caller passes (exp(-x^2 / 18)
// normalised), reflect-101, rows then columns, float64 sums.
#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace pysift {

constexpr double BL_INF = 1e18;

__device__ __forceinline__ int refl_half(int i, int n) {
    while (i < 0 || i >= n) {
        if (i < 0) i = -i - 1;
        if (i >= n) i = 2 * n - 1 - i;
    }
    return i;
}

__device__ __forceinline__ int refl_101(int i, int n) {
    if (n == 1) return 0;
    while (i < 0 || i >= n) {
        if (i < 0) i = -i;
        if (i >= n) i = 2 * n - 2 - i;
    }
    return i;
}

struct BlendCtl {
    unsigned long long sum1[3], sum2[3], n_ov, sq;
    float gain[3];
    int have_ov, vertical, first_side;  // first_side: image 1 left of (vertical) / above the seam
    int line0, line1;                   // first and last DP line holding overlap
    int n_lines, seam_end;              // overlap lines; seam position on the last one
    int chunk;                          // backtrack chunk length
    int hist;                           // colour matching: 0 gain, 1 histograms (pysift/core.py:3694-3699)
    unsigned int hist1[3][256], hist2[3][256];  // overlap histograms of images 1 and 2
    double lut[3][256];                 // histogram-matching LUT per channel
};

// image 1 after the colour matching of pysift/core.py:3692-3699 where both
// images overlap (unchanged without overlap): the clipped gain, or the
// histogram-matching LUT applied as np.interp(clip(v, 0, 255), 0..255, lut)
// does (pysift/core.py:3621-3623): the LUT entry at integers, else
// (lut[j + 1] - lut[j]) * (v - j) + lut[j] in float64
__device__ __forceinline__ float color_matched(const BlendCtl* ctl, float v, int c) {
    if (!ctl->have_ov) return v;
    if (ctl->hist) {
        const float vc = v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v);
        const int j = (int)floorf(vc);
        const double* lut = ctl->lut[c];
        double r;
        if (j >= 255) r = lut[255];
        else if (vc == (float)j) r = lut[j];
        else r = ((lut[j + 1] - lut[j]) / 1.0) * ((double)vc - (double)j) + lut[j];
        return (float)r;
    }
    const float x = v * ctl->gain[c];
    return x < 0.0f ? 0.0f : (x > 255.0f ? 255.0f : x);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_or(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Image 1 of a blend: a uint8 canvas (the warped image) or a float32 one (the
// unclipped result of an earlier blend, as the second pass of a three-image
// stitch takes it, pysift/core.py:3931-3947).
struct Img1 {
    const uint8_t* u8;
    const float* f32;
    __device__ __forceinline__ float at(long long p, int c) const {
        return f32 ? f32[p * 3 + c] : (float)u8[p * 3 + c];
    }
};

// image-1 values for the gain means: rounded to multiples of 2^-24 (exact for
// uint8) and summed as 64-bit integers, an order-free sum
__device__ __forceinline__ long long fixed24(float v) { return __double2ll_rn((double)v * 16777216.0); }

// Per pixel: overlap sums (order-free) and line flags per row and column
// (bit 0 overlap, bit 1 image 1 only, bit 2 image 2 only).  One row per block.
__global__ void __launch_bounds__(256) k_blend_stats(const Img1 w1, const uint8_t* __restrict__ m1,
                                                     const uint8_t* __restrict__ c2, const uint8_t* __restrict__ m2,
                                                     int cw, BlendCtl* ctl, int* __restrict__ rowf,
                                                     int* __restrict__ colf, int* __restrict__ rlo,
                                                     int* __restrict__ rhi, int* __restrict__ clo,
                                                     int* __restrict__ chi, int hist) {
    __shared__ unsigned int sh1[3][256], sh2[3][256];
    if (hist)
        for (int k = threadIdx.x; k < 3 * 256; k += blockDim.x) {
            (&sh1[0][0])[k] = 0u;
            (&sh2[0][0])[k] = 0u;
        }
    __shared__ unsigned int s[7];
    __shared__ unsigned long long s1[3];
    __shared__ int s_or, s_lo, s_hi;
    if (threadIdx.x < 7) s[threadIdx.x] = 0u;
    if (threadIdx.x < 3) s1[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) {
        s_or = 0;
        s_lo = 0x7fffffff;
        s_hi = -1;
    }
    __syncthreads();
    const int v = blockIdx.y;
    int f_row = 0, lo = 0x7fffffff, hi = -1;
    unsigned int acc[7] = {0, 0, 0, 0, 0, 0, 0};  // [3..5]: image 2, [6]: count
    long long acc1[3] = {0, 0, 0};               // image 1, fixed point 2^-24
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < cw; u += gridDim.x * blockDim.x) {
        const long long p = (long long)v * cw + u;
        const bool a = m1[p] != 0, b = m2[p] != 0;
        const int f = (a && b ? 1 : 0) | (a && !b ? 2 : 0) | (!a && b ? 4 : 0);
        if (f) atomicOr(&colf[u], f);
        f_row |= f;
        if (a && b) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float v1 = w1.at(p, c);
                acc1[c] += fixed24(v1);
                acc[3 + c] += c2[p * 3 + c];
                if (hist) {
                    // np.histogram with edges 0..256: bin floor(v), 255 inclusive
                    const float vc = v1 < 0.0f ? 0.0f : (v1 > 255.0f ? 255.0f : v1);
                    atomicAdd(&sh1[c][min((int)floorf(vc), 255)], 1u);
                    atomicAdd(&sh2[c][c2[p * 3 + c]], 1u);
                }
            }
            acc[6] += 1u;
            lo = min(lo, u);
            hi = max(hi, u);
            atomicMin(&clo[u], v);
            atomicMax(&chi[u], v);
        }
    }
    f_row = warp_or(f_row);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && hi >= 0) {
        atomicMin(&s_lo, lo);
        atomicMax(&s_hi, hi);
    }
#pragma unroll
    for (int k = 3; k < 7; ++k) acc[k] = warp_sum(acc[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) acc1[k] = warp_sum(acc1[k]);
    if ((threadIdx.x & 31) == 0) {
        if (f_row) atomicOr(&s_or, f_row);
        if (acc[6]) {
#pragma unroll
            for (int k = 3; k < 7; ++k) atomicAdd(&s[k], acc[k]);
#pragma unroll
            for (int k = 0; k < 3; ++k) atomicAdd(&s1[k], (unsigned long long)acc1[k]);
        }
    }
    __syncthreads();
    if (hist && s[6])
        for (int k = threadIdx.x; k < 3 * 256; k += blockDim.x) {
            const unsigned a = (&sh1[0][0])[k], b = (&sh2[0][0])[k];
            if (a) atomicAdd(&(&ctl->hist1[0][0])[k], a);
            if (b) atomicAdd(&(&ctl->hist2[0][0])[k], b);
        }
    if (threadIdx.x == 0) {
        rlo[v] = s_lo;
        rhi[v] = s_hi;
        if (s_or) atomicOr(&rowf[v], s_or);
        if (s[6]) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                atomicAdd(&ctl->sum1[c], s1[c]);
                atomicAdd(&ctl->sum2[c], (unsigned long long)s[3 + c]);
            }
            atomicAdd(&ctl->n_ov, (unsigned long long)s[6]);
        }
    }
}

// block-wide sums of 6 integers (1024 threads)
__device__ void block_sum6(long long v[6], long long* sh /* [32][6] */) {
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = warp_sum(v[k]);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) sh[w * 6 + k] = v[k];
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            long long t = l < nw ? sh[l * 6 + k] : 0;
            v[k] = warp_sum(t);
        }
    }
}

// gain (pysift/core.py:3692-3699) and the seam orientation (pysift/core.py:3424-3438)
__global__ void __launch_bounds__(1024) k_blend_decide(BlendCtl* ctl, const int* __restrict__ rowf,
                                                       const int* __restrict__ colf, int cw, int ch, int hist) {
    __shared__ long long sh[32 * 6];
    __shared__ long long s_rows[6];
    __shared__ int s_lo, s_hi;
    // rows: {n overlap rows, n rows with image 1 only, sum of their indices, same for image 2, -}
    long long v[6] = {0, 0, 0, 0, 0, 0};
    for (int r = threadIdx.x; r < ch; r += blockDim.x) {
        const int f = rowf[r];
        if (f & 1) v[0] += 1;
        if (f & 2) { v[1] += 1; v[2] += r; }
        if (f & 4) { v[3] += 1; v[4] += r; }
    }
    block_sum6(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) s_rows[k] = v[k];
    }
    __syncthreads();
    long long c[6] = {0, 0, 0, 0, 0, 0};
    for (int u = threadIdx.x; u < cw; u += blockDim.x) {
        const int f = colf[u];
        if (f & 1) c[0] += 1;
        if (f & 2) { c[1] += 1; c[2] += u; }
        if (f & 4) { c[3] += 1; c[4] += u; }
    }
    block_sum6(c, sh);
    if (threadIdx.x == 0) {
        const unsigned long long n = ctl->n_ov;
        ctl->have_ov = n > 0;
        ctl->hist = hist;
        for (int k = 0; k < 3; ++k) {
            float g = 1.0f;
            if (n > 0) {
                const float mean1 = (float)(((double)(long long)ctl->sum1[k] / 16777216.0) / (double)n);
                const float mean2 = (float)((double)ctl->sum2[k] / (double)n);
                g = (mean2 + 1e-3f) / (mean1 + 1e-3f);
                g = g < 0.5f ? 0.5f : (g > 2.0f ? 2.0f : g);
            }
            ctl->gain[k] = g;
        }
        const bool vert = s_rows[0] >= c[0];
        ctl->vertical = vert;
        if (vert)
            ctl->first_side = c[1] == 0 || c[3] == 0 || (double)c[2] / (double)c[1] <= (double)c[4] / (double)c[3];
        else
            ctl->first_side = s_rows[1] == 0 || s_rows[3] == 0 ||
                              (double)s_rows[2] / (double)s_rows[1] <= (double)s_rows[4] / (double)s_rows[3];
        s_lo = 0x7fffffff;
        s_hi = -1;
    }
    __syncthreads();
    const bool vert = ctl->vertical != 0;
    const int L = vert ? ch : cw;
    const int* lf = vert ? rowf : colf;
    for (int i = threadIdx.x; i < L; i += blockDim.x)
        if (lf[i] & 1) {
            atomicMin(&s_lo, i);
            atomicMax(&s_hi, i);
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->line0 = s_lo;
        ctl->line1 = s_hi;
    }
}

// image 1 after gain, the pyramid inputs I1 / I2 (pysift/core.py:3703-3708)
// at one pixel, from the uint8 canvases; the level-0 passes recompute them
// instead of storing two float images
struct Level0 {
    Img1 w1;
    const uint8_t* m1;
    const uint8_t* c2;
    const uint8_t* m2;
    const BlendCtl* ctl;
    __device__ __forceinline__ void px(long long p, float i1[3], float i2[3]) const {
        const bool a = m1[p] != 0, b = m2[p] != 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float x = color_matched(ctl, w1.at(p, c), c);
            const float y = (float)c2[p * 3 + c];
            i1[c] = a ? x : (b ? y : 0.0f);
            i2[c] = b ? y : (a ? x : 0.0f);
        }
    }
};

// The histogram-matching LUT of one channel (pysift/core.py:3611-3620), one
// block of 256 threads a channel: CDFs of the overlap histograms in float64,
// each divided by (total + 1e-8); lut[k] = np.interp(cdf1[k], cdf2, 0..255):
// 0 below cdf2[0], 255 above cdf2[255], else with j the last index where
// cdf2[j] <= x: j if j == 255 or cdf2[j] == x, else
// (1 / (cdf2[j + 1] - cdf2[j])) * (x - cdf2[j]) + j.
__global__ void __launch_bounds__(256) k_blend_hist_lut(BlendCtl* ctl) {
    __shared__ int sh[33];
    __shared__ double cdf2[256];
    if (!ctl->hist || !ctl->have_ov) return;
    const int c = blockIdx.x, k = threadIdx.x;
    int tot1, tot2;
    const int a = (int)ctl->hist1[c][k], b = (int)ctl->hist2[c][k];
    const int cum1 = block_excl_scan(a, &tot1, sh) + a;
    const int cum2 = block_excl_scan(b, &tot2, sh) + b;
    const double x = (double)cum1 / ((double)tot1 + 1e-8);
    cdf2[k] = (double)cum2 / ((double)tot2 + 1e-8);
    __syncthreads();
    double r;
    if (x > cdf2[255]) {
        r = 255.0;
    } else if (x < cdf2[0]) {
        r = 0.0;
    } else {
        int lo = 0, hi = 256;  // first index with cdf2 > x
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (x >= cdf2[mid]) lo = mid + 1;
            else hi = mid;
        }
        const int j = lo - 1;
        if (j == 255 || cdf2[j] == x) r = (double)j;
        else r = (1.0 / (cdf2[j + 1] - cdf2[j])) * (x - cdf2[j]) + (double)j;
    }
    ctl->lut[c][k] = r;
}

// colour cost, average gray (pysift/core.py:3411-3415) and the seam-RMSE sum
// (pysift/core.py:3555-3562) of the gained image 1
__global__ void k_blend_prepare(const Img1 w1, const uint8_t* __restrict__ m1,
                                const uint8_t* __restrict__ c2, const uint8_t* __restrict__ m2, int cw,
                                BlendCtl* ctl, float* __restrict__ color, float* __restrict__ avg) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    unsigned int sq = 0;
    if (u < cw) {
        const long long p = (long long)v * cw + u;
        const bool ov = m1[p] != 0 && m2[p] != 0;
        float g1[3], g2[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float x = color_matched(ctl, w1.at(p, c), c);
            g1[c] = x;
            g2[c] = (float)c2[p * 3 + c];
            if (ov) {
                const int d = (int)x - (int)c2[p * 3 + c];
                sq += (unsigned int)(d * d);
            }
        }
        const float d0 = g1[0] - g2[0], d1 = g1[1] - g2[1], d2 = g1[2] - g2[2];
        color[p] = sqrtf((d0 * d0 + d1 * d1) + d2 * d2);
        const float s0 = (g1[0] + g2[0]) * 0.5f, s1 = (g1[1] + g2[1]) * 0.5f, s2 = (g1[2] + g2[2]) * 0.5f;
        avg[p] = ((s0 + s1) + s2) / 3.0f;
    }
    // one atomic per block on the single seam-RMSE counter (per-warp atomics
    // on one address serialise in L2); a block's sum stays below 2^32
    __shared__ unsigned int s_sq[32];
    sq = warp_sum(sq);
    if ((threadIdx.x & 31) == 0) s_sq[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_sq[w];
        if (t) atomicAdd(&ctl->sq, (unsigned long long)t);
    }
}

// scipy sobel of the average gray along both axes and the seam cost
// (pysift/core.py:3416-3420).  Each sobel is correlate1d([-1, 0, 1]) along its
// axis (antisymmetric: x[i+1] - x[i-1]) rounded to float32, then [1, 2, 1]
// along the other (2 x[i] + (x[i-1] + x[i+1])), both in float64 with
// half-sample reflection.  The DP reads `dpc`: the cost where both images
// cover the canvas, else -1, line by line (transposed for a horizontal seam).
__global__ void k_sobel_cost(const float* __restrict__ avg, const float* __restrict__ color,
                             const uint8_t* __restrict__ m1, const uint8_t* __restrict__ m2, const BlendCtl* ctl,
                             float* __restrict__ dpc, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const long long p = (long long)y * W + x;
    const int xl = refl_half(x - 1, W), xr = refl_half(x + 1, W);
    const int yu = refl_half(y - 1, H), yd = refl_half(y + 1, H);
    auto dxr = [&](int r) {  // the axis-1 derivative on row r, as float32
        return (double)(float)((double)avg[(long long)r * W + xr] - (double)avg[(long long)r * W + xl]);
    };
    auto dyc = [&](int c) {  // the axis-0 derivative on column c, as float32
        return (double)(float)((double)avg[(long long)yd * W + c] - (double)avg[(long long)yu * W + c]);
    };
    const float gx = (float)(2.0 * dxr(y) + (dxr(yu) + dxr(yd)));
    const float gy = (float)(2.0 * dyc(x) + (dyc(xl) + dyc(xr)));
    const float c = color[p] + 0.05f * sqrtf(gx * gx + gy * gy);
    const float out = (m1[p] && m2[p]) ? c : -1.0f;
    if (ctl->vertical) dpc[p] = out;
    else dpc[(long long)x * H + y] = out;
}

__device__ __forceinline__ void bl_cp_async4(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void bl_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bl_cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Dynamic-programming seam, forward pass (pysift/core.py:3286-3383), in one
// CTA: overlap lines in order (rows for a vertical seam, columns for a
// horizontal one), positions in parallel.  Line q only computes its window:
// its own overlap range widened to one past the previous overlap line's range.
// Outside it all three predecessors are INF, so the DP value is INF and the
// argmin is 0 (dir is cleared beforehand).  The DP lines hold INF outside the
// window (positions of the line before last that fall outside are reset) and
// carry one INF sentinel at each end.  With K > 0 the cost lines stream
// through a K-deep cp.async ring, each thread copying the positions it reads.
// Outputs: dir[line][pos] = argmin (0 left, 1 centre, 2 right), the compacted
// overlap lines, and in ctl their count and the seam position on the last one
// (numpy's first minimum over the whole line).
template <int K>
__global__ void __launch_bounds__(1024) k_blend_dp(const float* __restrict__ dpc, const int* __restrict__ rowf,
                                                   const int* __restrict__ colf, const int* __restrict__ rlo,
                                                   const int* __restrict__ rhi, const int* __restrict__ clo,
                                                   const int* __restrict__ chi, int cw, int ch, BlendCtl* ctl,
                                                   double* __restrict__ gA, double* __restrict__ gB,
                                                   int4* __restrict__ gwin, int in_global,
                                                   uint8_t* __restrict__ dir, int* __restrict__ ovl) {
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ int s_sh[33];
    __shared__ double s_best[32];
    __shared__ int s_idx[32];
    if (!ctl->have_ov) return;
    const bool vert = ctl->vertical != 0;
    const int L = vert ? ch : cw, M = vert ? cw : ch;
    const int* lf = vert ? rowf : colf;
    const int* lo_of = vert ? rlo : clo;
    const int* hi_of = vert ? rhi : chi;
    const int nfw = (L + 31) >> 5;
    const int tid = threadIdx.x, nt = blockDim.x;
    // shared layout: line bitmask | windows {lo, hi, line} | the two DP lines (M + 2 each) | ring
    unsigned* fl = reinterpret_cast<unsigned*>(dsm);
    size_t off = ((size_t)nfw * 4 + 15) & ~(size_t)15;
    int4* win = in_global ? gwin : reinterpret_cast<int4*>(dsm + off);
    if (!in_global) off += (size_t)L * 16;
    double* lineA = in_global ? gA : reinterpret_cast<double*>(dsm + off);
    double* lineB = in_global ? gB : lineA + (M + 2);
    if (!in_global) off += (size_t)(M + 2) * 16;
    float* ring = reinterpret_cast<float*>(dsm + off);
    // overlap-line bitmask and the compacted list of overlap lines
    const int per = (nfw + nt - 1) / nt;
    const int w0 = min(nfw, tid * per), w1 = min(nfw, (tid + 1) * per);
    int cnt = 0;
    for (int w = w0; w < w1; ++w) {
        unsigned b = 0u;
        for (int k = 0; k < 32; ++k) {
            const int i = (w << 5) + k;
            if (i < L && (lf[i] & 1)) b |= 1u << k;
        }
        fl[w] = b;
        cnt += __popc(b);
    }
    int nL;
    int base = block_excl_scan(cnt, &nL, s_sh);
    for (int w = w0; w < w1; ++w) {
        unsigned b = fl[w];
        while (b) {
            const int k = __ffs(b) - 1;
            b &= b - 1u;
            const int line = (w << 5) + k;
            const int lo = lo_of[line], hi = hi_of[line];
            int4 wn = make_int4(lo, hi, line, 0);
            if (base > 0) {
                // the previous overlap line: the highest set bit below `line`
                int pw = line >> 5;
                unsigned pb = fl[pw] & ((1u << (line & 31)) - 1u);
                while (!pb) pb = fl[--pw];  // base > 0: an earlier overlap line exists
                const int pline = (pw << 5) + 31 - __clz(pb);
                wn.x = max(0, min(lo_of[pline] - 1, lo));
                wn.y = min(M - 1, max(hi_of[pline] + 1, hi));
            }
            win[base] = wn;
            ovl[base++] = line;
        }
    }
    for (int j = tid; j < M + 2; j += nt) {
        lineA[j] = BL_INF;
        lineB[j] = BL_INF;
    }
    __syncthreads();
    double* prev = lineA + 1;  // prev[-1] and prev[M] stay INF
    double* cur = lineB + 1;
    {
        const int4 w = win[0];
        const float* crow = dpc + (long long)w.z * M;
        for (int j = w.x + tid; j <= w.y; j += nt) {
            const float c = crow[j];
            prev[j] = c >= 0.0f ? (double)c : BL_INF;
        }
    }
    constexpr int KR = K > 0 ? K : 1;
    if (K > 0) {
        for (int s = 0; s < K - 1; ++s) {
            const int q = 1 + s;
            if (q < nL) {
                const int4 w = win[q];
                const float* src = dpc + (long long)w.z * M;
                float* slot = ring + (size_t)s * M;
                for (int j = w.x + tid; j <= w.y; j += nt) bl_cp_async4(slot + j, src + j);
            }
            bl_cp_commit();
        }
    }
    __syncthreads();
    for (int q = 1; q < nL; ++q) {
        const int4 w = win[q];
        const float* crow;
        if (K > 0) {
            const int qn = q + K - 1;
            if (qn < nL) {
                const int4 wn = win[qn];
                const float* src = dpc + (long long)wn.z * M;
                float* slot = ring + (size_t)((q + K - 2) % KR) * M;
                for (int j = wn.x + tid; j <= wn.y; j += nt) bl_cp_async4(slot + j, src + j);
            }
            bl_cp_commit();
            bl_cp_wait<KR - 1>();
            crow = ring + (size_t)((q - 1) % KR) * M;
        } else {
            crow = dpc + (long long)w.z * M;
        }
        // positions of the line before last outside this window go back to INF
        if (q >= 2) {
            const int4 o = win[q - 2];
            for (int j = o.x + tid; j < min(o.y + 1, w.x); j += nt) cur[j] = BL_INF;
            for (int j = max(o.x, w.y + 1) + tid; j <= o.y; j += nt) cur[j] = BL_INF;
        }
        uint8_t* drow = dir + (long long)w.z * M;
        for (int j = w.x + tid; j <= w.y; j += nt) {
            const float c = crow[j];
            const double pl = prev[j - 1], pm = prev[j], pr = prev[j + 1];
            int a = 0;
            double best = pl;
            if (pm < best) { best = pm; a = 1; }
            if (pr < best) { best = pr; a = 2; }
            cur[j] = c >= 0.0f ? (double)c + best : BL_INF;
            if (a) drow[j] = (uint8_t)a;
        }
        __syncthreads();
        double* t = prev;
        prev = cur;
        cur = t;
    }
    if (K > 0) bl_cp_wait<0>();
    // first minimum of the last overlap line (non-overlap positions count as INF)
    const int last = win[nL - 1].z;
    double bv = BL_INF * 4.0;
    int bj = 0x7fffffff;
    for (int j = tid; j < M; j += nt) {
        const double vv = dpc[(long long)last * M + j] >= 0.0f ? prev[j] : BL_INF;
        if (vv < bv) { bv = vv; bj = j; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oj = __shfl_xor_sync(0xffffffffu, bj, o);
        if (ov < bv || (ov == bv && oj < bj)) { bv = ov; bj = oj; }
    }
    if ((tid & 31) == 0) {
        s_best[tid >> 5] = bv;
        s_idx[tid >> 5] = bj;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < (nt >> 5); ++w)
            if (s_best[w] < bv || (s_best[w] == bv && s_idx[w] < bj)) { bv = s_best[w]; bj = s_idx[w]; }
        ctl->seam_end = bj;
        ctl->n_lines = nL;
        int R = 16;
        while (2 * R * R < nL) R *= 2;
        ctl->chunk = R;
    }
}

// one backtrack step from overlap line q (position p) to overlap line q - 1
__device__ __forceinline__ int bt_step(const uint8_t* __restrict__ dir, const int* __restrict__ ovl, int M, int q,
                                       int p) {
    const int k = p + (int)dir[(long long)ovl[q] * M + p] - 1;
    return k < 0 ? 0 : (k > M - 1 ? M - 1 : k);
}

// Backtrack, stage 1: the overlap lines are cut into chunks of R; for chunk
// c below the last and every position j on overlap line (c + 1) R, the
// position the seam reaches on overlap line c R.
__global__ void k_seam_jump(const uint8_t* __restrict__ dir, const int* __restrict__ ovl, const BlendCtl* ctl,
                            int cw, int ch, int* __restrict__ jump) {
    if (!ctl->have_ov) return;
    const int R = ctl->chunk;
    const int M = ctl->vertical ? cw : ch;
    const int C = (ctl->n_lines + R - 1) / R;
    const int c = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C - 1 || j >= M) return;
    int p = j;
    for (int q = (c + 1) * R; q > c * R; --q) p = bt_step(dir, ovl, M, q, p);
    jump[(long long)c * M + j] = p;
}

// Backtrack, stage 2 (one CTA): the chunk entry positions in sequence, then
// the lines of every chunk in parallel; lines without overlap keep the end
// position (pysift/core.py:3326-3334).
__global__ void __launch_bounds__(1024) k_seam_walk(const uint8_t* __restrict__ dir, const int* __restrict__ ovl,
                                                    const BlendCtl* ctl, int cw, int ch,
                                                    const int* __restrict__ jump, int* __restrict__ entry,
                                                    int* __restrict__ seam) {
    if (!ctl->have_ov) return;
    const int R = ctl->chunk;
    const bool vert = ctl->vertical != 0;
    const int L = vert ? ch : cw, M = vert ? cw : ch;
    const int nL = ctl->n_lines, sc = ctl->seam_end;
    const int C = (nL + R - 1) / R;
    for (int i = threadIdx.x; i < L; i += blockDim.x) seam[i] = sc;
    if (threadIdx.x == 0) {
        int p = sc;
        for (int q = nL - 1; q > (C - 1) * R; --q) p = bt_step(dir, ovl, M, q, p);
        entry[C - 1] = p;  // the position on overlap line (C - 1) R
        for (int c = C - 2; c >= 0; --c) {
            p = jump[(long long)c * M + p];
            entry[c] = p;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const int qtop = c == C - 1 ? nL - 1 : (c + 1) * R;
        int p = c == C - 1 ? sc : entry[c + 1];
        seam[ovl[qtop]] = p;
        for (int q = qtop; q > c * R; --q) {
            p = bt_step(dir, ovl, M, q, p);
            seam[ovl[q - 1]] = p;
        }
    }
}

// filter taps passed by value (kernel parameters: no host copies, so the
// composition can be captured in a CUDA graph)
struct SeamTaps {
    float k[25];
};
struct GaussTaps {
    double w[9];
};

// the seam mask before its blur (pysift/core.py:3406-3467): 1 = image 1
__device__ __forceinline__ float seam_value(const uint8_t* __restrict__ m1, const uint8_t* __restrict__ m2,
                                            const int* __restrict__ seam, const BlendCtl* ctl, int u, int v, int cw) {
    const long long p = (long long)v * cw + u;
    const bool a = m1[p] != 0, b = m2[p] != 0;
    if (!a) return 0.0f;
    if (!b) return 1.0f;
    const bool first = ctl->vertical ? (u <= seam[v]) : (v <= seam[u]);
    return (ctl->first_side ? first : !first) ? 1.0f : 0.0f;
}

// seam-mask blur (sigma 3, 25 taps, reflect-101, float64 sums in tap order):
// the row pass over the mask values ...  A block stages the mask values of
// SR_T x SR_R outputs (+12 each side) in shared memory, one padding word per
// 8 values so that lanes reading 8-value strips hit distinct banks; a thread
// widens its SR_R + 24 inputs to float64 once and forms SR_R outputs, each
// the same 25-tap sum in tap order.
constexpr int SR_T = 64, SR_R = 8, SR_N = SR_T * SR_R + 24;
__device__ __forceinline__ int sr_phys(int i) { return i + (i >> 3); }

__global__ void __launch_bounds__(SR_T) k_seam_rows(const uint8_t* __restrict__ m1, const uint8_t* __restrict__ m2,
                                                    const int* __restrict__ seam, const BlendCtl* ctl,
                                                    const SeamTaps k25, float* __restrict__ out, int W) {
    __shared__ float sv[SR_N + SR_N / 8 + 1];
    const int y = blockIdx.y, x0 = blockIdx.x * SR_T * SR_R;
    for (int i = threadIdx.x; i < SR_N; i += SR_T)
        sv[sr_phys(i)] = seam_value(m1, m2, seam, ctl, refl_101(x0 + i - 12, W), y, W);
    __syncthreads();
    const int b = threadIdx.x * SR_R;
    if (x0 + b >= W) return;
    double v[SR_R + 24];
#pragma unroll
    for (int m = 0; m < SR_R + 24; ++m) v[m] = (double)sv[sr_phys(b + m)];
#pragma unroll
    for (int j = 0; j < SR_R; ++j) {
        const int x = x0 + b + j;
        if (x >= W) break;
        double s = 0.0;
#pragma unroll
        for (int t = 0; t < 25; ++t) s = s + (double)k25.k[t] * v[j + t];
        out[(long long)y * W + x] = (float)s;
    }
}

// ... then the column pass; the blurred value replaces the mask where both
// images cover the canvas (pysift/core.py:3469-3471)
__global__ void k_seam_cols(const float* __restrict__ rows, const uint8_t* __restrict__ m1,
                            const uint8_t* __restrict__ m2, const int* __restrict__ seam, const BlendCtl* ctl,
                            const SeamTaps k25, float* __restrict__ gm0, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const long long p = (long long)y * W + x;
    if (m1[p] && m2[p]) {
        double s = 0.0;
#pragma unroll 5
        for (int t = 0; t < 25; ++t) s = s + (double)k25.k[t] * (double)rows[(long long)refl_101(y + t - 12, H) * W + x];
        gm0[p] = (float)s;
    } else {
        gm0[p] = seam_value(m1, m2, seam, ctl, x, y, W);
    }
}

// The Gaussian pyramids of I1, I2 and the seam mask (pysift/core.py:3520-3526):
// gaussian_filter(sigma = 1) per channel followed by [::2, ::2]
// (pysift/core.py:3475-3483).  Two channel groups: the images (I1 and I2,
// six channels; level 0 recomputed from the uint8 canvases) and the mask,
// so the image pyramids can run while the seam is being found.  Row pass at
// even rows, then the column pass at even columns.
struct PyrLevel {
    const float* g1;  // (h, w, 3)
    const float* g2;
    const float* gm;  // (h, w)
};

template <int NC, bool L0>
__device__ __forceinline__ void pyr_load(const Level0& src, const PyrLevel& in, long long p, double v[NC]) {
    if (NC == 1) {
        v[0] = (double)in.gm[p];
    } else if (L0) {
        float i1[3], i2[3];
        src.px(p, i1, i2);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            v[c] = (double)i1[c];
            v[3 + c] = (double)i2[c];
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            v[c] = (double)in.g1[p * 3 + c];
            v[3 + c] = (double)in.g2[p * 3 + c];
        }
    }
}

// NC = 6: t1 / t2 get I1 / I2 (3 floats a pixel); NC = 1: t1 gets the mask
template <int NC, bool L0>
__global__ void k_pyr_rows(const Level0 src, const PyrLevel in, int W, int H, float* __restrict__ t1,
                           float* __restrict__ t2, const GaussTaps w9) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, yo = blockIdx.y;
    if (x >= W) return;
    const int y = 2 * yo;
    double s[NC], a[NC], b[NC];
    pyr_load<NC, L0>(src, in, (long long)y * W + x, a);
#pragma unroll
    for (int c = 0; c < NC; ++c) s[c] = w9.w[4] * a[c];
#pragma unroll
    for (int k = 4; k >= 1; --k) {
        pyr_load<NC, L0>(src, in, (long long)refl_half(y - k, H) * W + x, a);
        pyr_load<NC, L0>(src, in, (long long)refl_half(y + k, H) * W + x, b);
        const double w = w9.w[4 - k];
#pragma unroll
        for (int c = 0; c < NC; ++c) s[c] = s[c] + (a[c] + b[c]) * w;
    }
    const long long o = (long long)yo * W + x;
    if (NC == 1) {
        t1[o] = (float)s[0];
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            t1[o * 3 + c] = (float)s[c];
            t2[o * 3 + c] = (float)s[(3 + c) % NC];
        }
    }
}

template <int NC>
__global__ void k_pyr_cols(const float* __restrict__ t1, const float* __restrict__ t2, int W, int Wo,
                           const GaussTaps w9, float* __restrict__ g1, float* __restrict__ g2) {
    const int xo = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (xo >= Wo) return;
    const int col = 2 * xo;
    const long long row = (long long)y * W;
    auto load = [&](int cc, double v[NC]) {
        const long long p = row + cc;
        if (NC == 1) {
            v[0] = (double)t1[p];
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                v[c] = (double)t1[p * 3 + c];
                v[(3 + c) % NC] = (double)t2[p * 3 + c];
            }
        }
    };
    double s[NC], a[NC], b[NC];
    load(col, a);
#pragma unroll
    for (int c = 0; c < NC; ++c) s[c] = w9.w[4] * a[c];
#pragma unroll
    for (int k = 4; k >= 1; --k) {
        load(refl_half(col - k, W), a);
        load(refl_half(col + k, W), b);
        const double w = w9.w[4 - k];
#pragma unroll
        for (int c = 0; c < NC; ++c) s[c] = s[c] + (a[c] + b[c]) * w;
    }
    const long long o = (long long)y * Wo + xo;
    if (NC == 1) {
        g1[o] = (float)s[0];
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            g1[o * 3 + c] = (float)s[c];
            g2[o * 3 + c] = (float)s[(3 + c) % NC];
        }
    }
}

// zoom(order = 1) of an (h, w) level to (H, W) (pysift/core.py:3485-3493):
// coordinate k * (in - 1) / (out - 1), corners reflected (mirror) at the edge
struct ZoomF {
    double zy, zx;  // (in - 1) / (out - 1) per axis, 1 when out == 1
};

static ZoomF zoom_factors(int h, int w, int H, int W) {
    ZoomF z;
    z.zy = H > 1 ? (double)(h - 1) / (double)(H - 1) : 1.0;
    z.zx = W > 1 ? (double)(w - 1) / (double)(W - 1) : 1.0;
    return z;
}

struct Zoom1 {
    long long o[4];
    double wy[2], wx[2];
    __device__ Zoom1(int h, int w, ZoomF f, int y, int x) {
        const double cy = (double)y * f.zy, cx = (double)x * f.zx;
        const int y0 = (int)floor(cy), x0 = (int)floor(cx);
        const double ty = cy - (double)y0, tx = cx - (double)x0;
        wy[0] = 1.0 - ty;
        wy[1] = ty;
        wx[0] = 1.0 - tx;
        wx[1] = tx;
        const int ya = refl_101(y0, h), yb = refl_101(y0 + 1, h);
        const int xa = refl_101(x0, w), xb = refl_101(x0 + 1, w);
        o[0] = (long long)ya * w + xa;
        o[1] = (long long)ya * w + xb;
        o[2] = (long long)yb * w + xa;
        o[3] = (long long)yb * w + xb;
    }
    // sum over the corners in row-major order of ((v * wy) * wx)
    __device__ float at(const float* __restrict__ in, int C, int c) const {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double coeff = (double)in[o[k] * C + c];
            coeff = coeff * wy[k >> 1];
            coeff = coeff * wx[k & 1];
            t = t + coeff;
        }
        return (float)t;
    }
};

// one blended Laplacian level k >= 1: m * (G1 - up(G1')) + (1 - m) * (G2 - up(G2'))
// (pysift/core.py:3529-3541); the coarsest level blends the Gaussians
__global__ void k_blend_level(const float* __restrict__ g1, const float* __restrict__ g2,
                              const float* __restrict__ gm, const float* __restrict__ g1n,
                              const float* __restrict__ g2n, int H, int W, int hn, int wn, ZoomF zf,
                              float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const long long p = (long long)y * W + x;
    const float m = gm[p];
    const float mc = 1.0f - m;
    if (g1n) {
        const Zoom1 z(hn, wn, zf, y, x);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float l1 = g1[p * 3 + c] - z.at(g1n, 3, c);
            const float l2 = g2[p * 3 + c] - z.at(g2n, 3, c);
            out[p * 3 + c] = m * l1 + mc * l2;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) out[p * 3 + c] = m * g1[p * 3 + c] + mc * g2[p * 3 + c];
    }
}

// reconstruction step (pysift/core.py:3544-3547): out = up(res) + lb
__global__ void k_blend_reconstruct(const float* __restrict__ res, int hn, int wn, const float* __restrict__ lb,
                                    int H, int W, ZoomF zf, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const long long p = (long long)y * W + x;
    const Zoom1 z(hn, wn, zf, y, x);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[p * 3 + c] = z.at(res, 3, c) + lb[p * 3 + c];
}

// Level 0 in one pass: its Laplacian blend, the last reconstruction step
// (result = up(res) + lb0) and the paste (pysift/core.py:3806-3809): uint8
// truncation of the clipped value where either image covers the canvas.
// With one level there is no pyramid: result = m * I1 + (1 - m) * I2.
__global__ void k_blend_final(const Level0 src, const float* __restrict__ gm0, const float* __restrict__ g1n,
                              const float* __restrict__ g2n, const float* __restrict__ res, int hn, int wn, int H,
                              int W, ZoomF zf, uint8_t* __restrict__ pano, uint8_t* __restrict__ both,
                              float* __restrict__ blended, double* __restrict__ seam_rmse) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x == 0 && y == 0 && seam_rmse) {
        const BlendCtl* ctl = src.ctl;
        *seam_rmse = ctl->n_ov ? sqrt((double)ctl->sq / (3.0 * (double)ctl->n_ov))
                               : __longlong_as_double(0x7ff8000000000000ll);
    }
    if (x >= W) return;
    const long long p = (long long)y * W + x;
    const bool any = src.m1[p] || src.m2[p];
    if (both) both[p] = any;
    float i1[3], i2[3];
    src.px(p, i1, i2);
    const float m = gm0[p];
    const float mc = 1.0f - m;
    float v[3];
    if (res) {
        const Zoom1 z(hn, wn, zf, y, x);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float l1 = i1[c] - z.at(g1n, 3, c);
            const float l2 = i2[c] - z.at(g2n, 3, c);
            const float lb = m * l1 + mc * l2;
            v[c] = z.at(res, 3, c) + lb;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = m * i1[c] + mc * i2[c];
    }
    if (blended) {
#pragma unroll
        for (int c = 0; c < 3; ++c) blended[p * 3 + c] = v[c];
    }
    if (pano) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float t = v[c] < 0.0f ? 0.0f : (v[c] > 255.0f ? 255.0f : v[c]);
            pano[p * 3 + c] = any ? (uint8_t)(int)t : (uint8_t)0;
        }
    }
}

__global__ void k_fill_i32(int* __restrict__ p, int n, int v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// per-row and per-column extents of a coverage mask (the inner-rectangle
// crop's inputs, pysift/core.py:3655-3675); one row per block
__global__ void __launch_bounds__(256) k_mask_extents(const uint8_t* __restrict__ mask, int cw, int* __restrict__ row_lo,
                                                      int* __restrict__ row_hi, int* __restrict__ col_lo,
                                                      int* __restrict__ col_hi) {
    __shared__ int s_lo, s_hi;
    if (threadIdx.x == 0) {
        s_lo = 0x7fffffff;
        s_hi = -1;
    }
    __syncthreads();
    const int v = blockIdx.y;
    int lo = 0x7fffffff, hi = -1;
    for (int u = threadIdx.x; u < cw; u += blockDim.x) {
        if (mask[(long long)v * cw + u]) {
            lo = min(lo, u);
            hi = max(hi, u);
            atomicMin(&col_lo[u], v);
            atomicMax(&col_hi[u], v);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && hi >= 0) {
        atomicMin(&s_lo, lo);
        atomicMax(&s_hi, hi);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        row_lo[v] = s_lo;
        row_hi[v] = s_hi;
    }
}

// image 2 pasted on the canvas at (iox, ioy) (pysift/core.py:3794-3800)
__global__ void k_place_image(const uint8_t* __restrict__ img, int h, int w, int pitch, int cw, int iox, int ioy,
                              uint8_t* __restrict__ canvas, uint8_t* __restrict__ mask) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= cw) return;
    const int x = u - iox, y = v - ioy;
    const bool in = x >= 0 && x < w && y >= 0 && y < h;
    const long long p = (long long)v * cw + u;
#pragma unroll
    for (int c = 0; c < 3; ++c) canvas[p * 3 + c] = in ? img[(long long)y * pitch + 3 * x + c] : (uint8_t)0;
    if (mask) mask[p] = in;
}

constexpr int DP_SMEM_MAX = 200 * 1024;
constexpr int DP_THREADS = 256;

// backtrack chunks: the chunk length R (a power of two, at least 16, with
// 2 R^2 >= the number of overlap lines, which balances the sequential walk of
// about 2 R + lines / R steps) is chosen on the device, so there are at most
// ceil(sqrt(2 M)) + 1 chunks for lines of M positions
static int max_seam_chunks(int M) {
    int c = 1;
    while ((long long)c * c < 2LL * M) ++c;
    return c + 1;
}

// another stream on the current device for work that can overlap the seam
// search; one per host thread and device, created on first use
static cudaStream_t side_stream() {
    constexpr int MAXDEV = 64;
    thread_local cudaStream_t streams[MAXDEV] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAXDEV) {
        set_error("side_stream: no current device");
        return nullptr;
    }
    if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess) {
        set_error("side_stream: cudaStreamCreateWithFlags failed");
        streams[dev] = nullptr;
    }
    return streams[dev];
}

struct BlendLayout {
    size_t off_ctl, off_rowf, off_colf, off_rlo, off_rhi, off_clo, off_chi, off_win, off_color, off_avg, off_dpc,
        off_rowA, off_rowB, off_dir, off_seam, off_ovl, off_jump, off_entry, off_srow, off_t1,
        off_t2, off_tm;
    int nchunk;
    size_t off_g1[8], off_g2[8], off_gm[8], off_lb[8], off_res[2];
    int h[8], w[8];
    size_t total;
};

// level k >= 1 holds G1, G2 (3 floats a pixel), the mask and the blended
// Laplacian; level 0 keeps only the seam mask (I1 / I2 come from the canvases)
static BlendLayout blend_layout(int cw, int ch, int levels) {
    BlendLayout l;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t r = off;
        off = align_up(off + bytes, 256);
        return r;
    };
    const size_t N = (size_t)cw * ch;
    const int M = cw > ch ? cw : ch;
    l.off_ctl = take(sizeof(BlendCtl));
    l.off_rowf = take((size_t)ch * 4);
    l.off_colf = take((size_t)cw * 4);
    l.off_rlo = take((size_t)ch * 4);
    l.off_rhi = take((size_t)ch * 4);
    l.off_clo = take((size_t)cw * 4);
    l.off_chi = take((size_t)cw * 4);
    l.off_win = take((size_t)M * 16);
    l.off_color = take(N * 4);
    l.off_avg = take(N * 4);
    l.off_dpc = take(N * 4);
    l.off_rowA = take((size_t)(M + 2) * 8);
    l.off_rowB = take((size_t)(M + 2) * 8);
    l.off_dir = take(N);
    l.off_seam = take((size_t)M * 4);
    l.off_ovl = take((size_t)M * 4);
    l.nchunk = max_seam_chunks(M);
    l.off_jump = take((size_t)l.nchunk * M * 4);
    l.off_entry = take((size_t)(l.nchunk + 1) * 4);
    l.off_srow = take(N * 4);
    const size_t half = (size_t)((ch + 1) / 2) * cw;
    l.off_t1 = take(half * 12);
    l.off_t2 = take(half * 12);
    l.off_tm = take(half * 4);
    int h = ch, w = cw;
    for (int k = 0; k < levels; ++k) {
        l.h[k] = h;
        l.w[k] = w;
        const size_t n = (size_t)h * w;
        l.off_gm[k] = take(n * 4);
        if (k > 0) {
            l.off_g1[k] = take(n * 12);
            l.off_g2[k] = take(n * 12);
            l.off_lb[k] = take(n * 12);
        }
        h = (h + 1) / 2;
        w = (w + 1) / 2;
    }
    const size_t n1 = levels > 1 ? (size_t)l.h[1] * l.w[1] : 1;
    l.off_res[0] = take(n1 * 12);
    l.off_res[1] = take(n1 * 12);
    l.total = off;
    return l;
}

template <typename T>
static T* bwp(void* ws, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(ws) + off);
}

}  // namespace pysift

using namespace pysift;

extern "C" {

int pysift_place_image(const uint8_t* img, int32_t h, int32_t w, int32_t pitch, int32_t cw, int32_t ch, int32_t iox,
                       int32_t ioy, uint8_t* canvas, uint8_t* mask, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(img && canvas, "NULL pointer argument");
    PYSIFT_CHECK_ARG(h > 0 && w > 0 && pitch >= 3 * w && cw > 0 && ch > 0, "bad sizes");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_place_image<<<dim3(ceil_div(cw, 256), ch), 256, 0, st>>>(img, h, w, pitch, cw, iox, ioy, canvas, mask);
    PYSIFT_LAUNCH_CHECK("k_place_image");
    return PYSIFT_OK;
}

int pysift_blend_workspace_size(int32_t cw, int32_t ch, int32_t n_levels, size_t* bytes) {
    PYSIFT_CHECK_ARG(bytes && cw > 1 && ch > 1 && n_levels >= 1 && n_levels <= 8, "bad arguments");
    *bytes = blend_layout(cw, ch, n_levels).total;
    return PYSIFT_OK;
}

int pysift_mask_extents(const uint8_t* mask, int32_t cw, int32_t ch, int32_t* row_lo, int32_t* row_hi,
                        int32_t* col_lo, int32_t* col_hi, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(mask && row_lo && row_hi && col_lo && col_hi, "NULL pointer argument");
    PYSIFT_CHECK_ARG(cw > 0 && ch > 0, "bad sizes");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_fill_i32<<<ceil_div(cw, 256), 256, 0, st>>>(col_lo, cw, 0x7fffffff);
    PYSIFT_CUDA_TRY(cudaMemsetAsync(col_hi, 0xff, (size_t)cw * 4, st));
    k_mask_extents<<<dim3(1, ch), 256, 0, st>>>(mask, cw, row_lo, row_hi, col_lo, col_hi);
    PYSIFT_LAUNCH_CHECK("k_mask_extents");
    return PYSIFT_OK;
}

int pysift_autocrop_box(const int32_t* row_lo, const int32_t* row_hi, const int32_t* col_lo, const int32_t* col_hi,
                        int32_t cw, int32_t ch, int32_t* box) {
    PYSIFT_CHECK_ARG(row_lo && row_hi && col_lo && col_hi && box, "NULL pointer argument");
    PYSIFT_CHECK_ARG(cw > 0 && ch > 0, "bad sizes");
    int r0 = -1, r1 = -1, c0 = -1, c1 = -1;
    for (int r = 0; r < ch; ++r)
        if (row_hi[r] >= 0) {
            if (r0 < 0) r0 = r;
            r1 = r;
        }
    for (int c = 0; c < cw; ++c)
        if (col_hi[c] >= 0) {
            if (c0 < 0) c0 = c;
            c1 = c;
        }
    if (r0 < 0 || c0 < 0) {  // nothing covered: the whole canvas
        box[0] = 0, box[1] = 0, box[2] = cw, box[3] = ch, box[4] = 0;
        return PYSIFT_OK;
    }
    const int nr = r1 - r0 + 1, nc = c1 - c0 + 1;
    // the largest left / top edge and the smallest right / bottom edge over
    // the covered lines of the bounding box (uncovered lines do not bind)
    int left = INT32_MIN, right = INT32_MAX, top = INT32_MIN, bot = INT32_MAX;
    for (int r = r0; r <= r1; ++r) {
        const bool cov = row_hi[r] >= 0;
        left = std::max(left, cov ? row_lo[r] - c0 : 0);
        right = std::min(right, cov ? row_hi[r] - c0 : nc - 1);
    }
    for (int c = c0; c <= c1; ++c) {
        const bool cov = col_hi[c] >= 0;
        top = std::max(top, cov ? col_lo[c] - r0 : 0);
        bot = std::min(bot, cov ? col_hi[c] - r0 : nr - 1);
    }
    if (left >= right || top >= bot) {  // no inner rectangle: the bounding box
        box[0] = c0, box[1] = r0, box[2] = nc, box[3] = nr, box[4] = 1;
        return PYSIFT_OK;
    }
    box[0] = c0 + left, box[1] = r0 + top, box[2] = right - left + 1, box[3] = bot - top + 1, box[4] = 2;
    return PYSIFT_OK;
}

int pysift_copy2d(void* dst, size_t dst_pitch, const void* src, size_t src_pitch, size_t width_bytes, size_t height,
                  pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(dst && src, "NULL pointer argument");
    PYSIFT_CHECK_ARG(width_bytes <= dst_pitch && width_bytes <= src_pitch, "bad pitches");
    if (width_bytes == 0 || height == 0) return PYSIFT_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    PYSIFT_CUDA_TRY(cudaMemcpy2DAsync(dst, dst_pitch, src, src_pitch, width_bytes, height, cudaMemcpyDefault, st));
    return PYSIFT_OK;
}

int pysift_blend_multiband(const void* image1, int32_t image1_f32, const uint8_t* mask1, const uint8_t* canvas2,
                           const uint8_t* mask2, int32_t cw, int32_t ch, int32_t n_levels, int32_t color_match,
                           const float* seam_k25,
                           const double* gauss_w9, void* workspace, size_t workspace_bytes, uint8_t* pano,
                           uint8_t* both, float* blended, double* seam_rmse, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(image1 && mask1 && canvas2 && mask2 && seam_k25 && gauss_w9 && workspace && (pano || blended),
                     "NULL pointer argument");
    Img1 w1;
    w1.u8 = image1_f32 ? nullptr : static_cast<const uint8_t*>(image1);
    w1.f32 = image1_f32 ? static_cast<const float*>(image1) : nullptr;
    PYSIFT_CHECK_ARG(cw > 1 && ch > 1 && n_levels >= 1 && n_levels <= 8, "bad sizes");
    PYSIFT_CHECK_ARG(color_match == 0 || color_match == 1, "color_match must be 0 (gain) or 1 (histograms)");
    const BlendLayout l = blend_layout(cw, ch, n_levels);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    void* ws = workspace;
    BlendCtl* ctl = bwp<BlendCtl>(ws, l.off_ctl);
    int* rowf = bwp<int>(ws, l.off_rowf);
    int* colf = bwp<int>(ws, l.off_colf);
    int* rlo = bwp<int>(ws, l.off_rlo);
    int* rhi = bwp<int>(ws, l.off_rhi);
    int* clo = bwp<int>(ws, l.off_clo);
    int* chi = bwp<int>(ws, l.off_chi);
    PYSIFT_CUDA_TRY(cudaMemsetAsync(ctl, 0, sizeof(BlendCtl), st));
    PYSIFT_CUDA_TRY(cudaMemsetAsync(rowf, 0, (size_t)ch * 4, st));
    PYSIFT_CUDA_TRY(cudaMemsetAsync(colf, 0, (size_t)cw * 4, st));
    PYSIFT_CUDA_TRY(cudaMemsetAsync(clo, 0x7f, (size_t)cw * 4, st));
    PYSIFT_CUDA_TRY(cudaMemsetAsync(chi, 0xff, (size_t)cw * 4, st));
    GaussTaps w9;
    SeamTaps k25;
    for (int i = 0; i < 9; ++i) w9.w[i] = gauss_w9[i];
    for (int i = 0; i < 25; ++i) k25.k[i] = seam_k25[i];
    const dim3 g2d(ceil_div(cw, 256), ch);
    // gain, overlap flags and ranges, seam orientation
    const int hist = color_match == 1;
    k_blend_stats<<<dim3(1, ch), 256, 0, st>>>(w1, mask1, canvas2, mask2, cw, ctl, rowf, colf, rlo, rhi, clo, chi,
                                                hist);
    PYSIFT_LAUNCH_CHECK("k_blend_stats");
    k_blend_decide<<<1, 1024, 0, st>>>(ctl, rowf, colf, cw, ch, hist);
    PYSIFT_LAUNCH_CHECK("k_blend_decide");
    if (hist) {
        k_blend_hist_lut<<<3, 256, 0, st>>>(ctl);
        PYSIFT_LAUNCH_CHECK("k_blend_hist_lut");
    }
    // Gaussian pyramids of I1 and I2 on a side stream: they need only the gain
    Level0 src;
    src.w1 = w1;
    src.m1 = mask1;
    src.c2 = canvas2;
    src.m2 = mask2;
    src.ctl = ctl;
    cudaStream_t side = side_stream();
    if (!side) return PYSIFT_ERR_CUDA;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    PYSIFT_CUDA_TRY(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    PYSIFT_CUDA_TRY(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
    PYSIFT_CUDA_TRY(cudaEventRecord(fork_ev, st));
    PYSIFT_CUDA_TRY(cudaStreamWaitEvent(side, fork_ev, 0));
    {
        float* t1 = bwp<float>(ws, l.off_t1);
        float* t2 = bwp<float>(ws, l.off_t2);
        for (int k = 0; k + 1 < n_levels; ++k) {
            PyrLevel in;
            in.g1 = k ? bwp<float>(ws, l.off_g1[k]) : nullptr;
            in.g2 = k ? bwp<float>(ws, l.off_g2[k]) : nullptr;
            in.gm = nullptr;
            const int ho = l.h[k + 1], wo = l.w[k + 1];
            const dim3 gr(ceil_div(l.w[k], 128), ho), gc(ceil_div(wo, 128), ho);
            if (k == 0) k_pyr_rows<6, true><<<gr, 128, 0, side>>>(src, in, l.w[k], l.h[k], t1, t2, w9);
            else k_pyr_rows<6, false><<<gr, 128, 0, side>>>(src, in, l.w[k], l.h[k], t1, t2, w9);
            k_pyr_cols<6><<<gc, 128, 0, side>>>(t1, t2, l.w[k], wo, w9, bwp<float>(ws, l.off_g1[k + 1]),
                                                bwp<float>(ws, l.off_g2[k + 1]));
        }
        PYSIFT_LAUNCH_CHECK("k_pyr images");
    }
    PYSIFT_CUDA_TRY(cudaEventRecord(join_ev, side));
    // seam cost
    float* color = bwp<float>(ws, l.off_color);
    float* avg = bwp<float>(ws, l.off_avg);
    float* dpc = bwp<float>(ws, l.off_dpc);
    k_blend_prepare<<<g2d, 256, 0, st>>>(w1, mask1, canvas2, mask2, cw, ctl, color, avg);
    PYSIFT_LAUNCH_CHECK("k_blend_prepare");
    k_sobel_cost<<<g2d, 256, 0, st>>>(avg, color, mask1, mask2, ctl, dpc, cw, ch);
    PYSIFT_LAUNCH_CHECK("k_sobel_cost");
    // DP seam and backtrack
    int* seam = bwp<int>(ws, l.off_seam);
    {
        int* ovl = bwp<int>(ws, l.off_ovl);
        uint8_t* dir = bwp<uint8_t>(ws, l.off_dir);
        // the orientation is decided on the device: size shared memory for the longer side
        const int M = cw > ch ? cw : ch;
        const size_t flags = (((size_t)(M + 31) / 32) * 4 + 15) & ~(size_t)15;
        const size_t wins = (size_t)M * 16;
        const size_t lines = (size_t)(M + 2) * 16;
        double* gA = bwp<double>(ws, l.off_rowA);
        double* gB = bwp<double>(ws, l.off_rowB);
        int4* gwin = bwp<int4>(ws, l.off_win);
        PYSIFT_CUDA_TRY(cudaMemsetAsync(dir, 0, (size_t)cw * ch, st));
        const size_t base = flags + wins + lines;
        if (base + (size_t)M * 32 <= (size_t)DP_SMEM_MAX) {
            const size_t sm = base + (size_t)M * 32;
            PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_blend_dp<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_blend_dp<8><<<1, DP_THREADS, sm, st>>>(dpc, rowf, colf, rlo, rhi, clo, chi, cw, ch, ctl, gA, gB, gwin, 0, dir,
                                               ovl);
        } else if (base + (size_t)M * 16 <= (size_t)DP_SMEM_MAX) {
            const size_t sm = base + (size_t)M * 16;
            PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_blend_dp<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_blend_dp<4><<<1, DP_THREADS, sm, st>>>(dpc, rowf, colf, rlo, rhi, clo, chi, cw, ch, ctl, gA, gB, gwin, 0, dir,
                                               ovl);
        } else if (base <= (size_t)DP_SMEM_MAX) {
            PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_blend_dp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)base));
            k_blend_dp<0><<<1, DP_THREADS, base, st>>>(dpc, rowf, colf, rlo, rhi, clo, chi, cw, ch, ctl, gA, gB, gwin, 0, dir,
                                                 ovl);
        } else {
            PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_blend_dp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)flags));
            k_blend_dp<0><<<1, DP_THREADS, flags, st>>>(dpc, rowf, colf, rlo, rhi, clo, chi, cw, ch, ctl, gA, gB, gwin, 1,
                                                  dir, ovl);
        }
        PYSIFT_LAUNCH_CHECK("k_blend_dp");
        int* jump = bwp<int>(ws, l.off_jump);
        k_seam_jump<<<dim3(ceil_div(M, 256), l.nchunk), 256, 0, st>>>(dir, ovl, ctl, cw, ch, jump);
        PYSIFT_LAUNCH_CHECK("k_seam_jump");
        k_seam_walk<<<1, 1024, 0, st>>>(dir, ovl, ctl, cw, ch, jump, bwp<int>(ws, l.off_entry), seam);
        PYSIFT_LAUNCH_CHECK("k_seam_walk");
    }
    // seam mask and its blur
    float* gm0 = bwp<float>(ws, l.off_gm[0]);
    float* srow = bwp<float>(ws, l.off_srow);
    k_seam_rows<<<dim3(ceil_div(cw, SR_T * SR_R), ch), SR_T, 0, st>>>(mask1, mask2, seam, ctl, k25, srow, cw);
    PYSIFT_LAUNCH_CHECK("k_seam_rows");
    k_seam_cols<<<g2d, 256, 0, st>>>(srow, mask1, mask2, seam, ctl, k25, gm0, cw, ch);
    PYSIFT_LAUNCH_CHECK("k_seam_cols");
    // Gaussian pyramid of the seam mask, then join the image pyramids
    {
        float* tm = bwp<float>(ws, l.off_tm);
        for (int k = 0; k + 1 < n_levels; ++k) {
            PyrLevel in;
            in.g1 = nullptr;
            in.g2 = nullptr;
            in.gm = bwp<float>(ws, l.off_gm[k]);
            const int ho = l.h[k + 1], wo = l.w[k + 1];
            k_pyr_rows<1, false><<<dim3(ceil_div(l.w[k], 128), ho), 128, 0, st>>>(src, in, l.w[k], l.h[k], tm, nullptr,
                                                                                  w9);
            k_pyr_cols<1><<<dim3(ceil_div(wo, 128), ho), 128, 0, st>>>(tm, nullptr, l.w[k], wo, w9,
                                                                       bwp<float>(ws, l.off_gm[k + 1]), nullptr);
        }
        PYSIFT_LAUNCH_CHECK("k_pyr mask");
    }
    PYSIFT_CUDA_TRY(cudaStreamWaitEvent(st, join_ev, 0));
    cudaEventDestroy(fork_ev);
    cudaEventDestroy(join_ev);
    // blended Laplacian levels 1 .. n - 1 and the reconstruction down to level 1
    for (int k = 1; k < n_levels; ++k) {
        const bool top = k + 1 == n_levels;
        k_blend_level<<<dim3(ceil_div(l.w[k], 256), l.h[k]), 256, 0, st>>>(
            bwp<float>(ws, l.off_g1[k]), bwp<float>(ws, l.off_g2[k]), bwp<float>(ws, l.off_gm[k]),
            top ? nullptr : bwp<float>(ws, l.off_g1[k + 1]), top ? nullptr : bwp<float>(ws, l.off_g2[k + 1]), l.h[k],
            l.w[k], top ? 0 : l.h[k + 1], top ? 0 : l.w[k + 1],
            top ? ZoomF{1.0, 1.0} : zoom_factors(l.h[k + 1], l.w[k + 1], l.h[k], l.w[k]), bwp<float>(ws, l.off_lb[k]));
    }
    PYSIFT_LAUNCH_CHECK("k_blend_level");
    const float* res = n_levels > 1 ? bwp<float>(ws, l.off_lb[n_levels - 1]) : nullptr;
    int rh = l.h[n_levels - 1], rw = l.w[n_levels - 1];
    for (int k = n_levels - 2; k >= 1; --k) {
        float* out = bwp<float>(ws, l.off_res[k & 1]);
        k_blend_reconstruct<<<dim3(ceil_div(l.w[k], 256), l.h[k]), 256, 0, st>>>(
            res, rh, rw, bwp<float>(ws, l.off_lb[k]), l.h[k], l.w[k], zoom_factors(rh, rw, l.h[k], l.w[k]), out);
        res = out;
        rh = l.h[k];
        rw = l.w[k];
    }
    PYSIFT_LAUNCH_CHECK("k_blend_reconstruct");
    // level 0: Laplacian blend, last reconstruction step and paste
    k_blend_final<<<g2d, 256, 0, st>>>(src, gm0, n_levels > 1 ? bwp<float>(ws, l.off_g1[1]) : nullptr,
                                       n_levels > 1 ? bwp<float>(ws, l.off_g2[1]) : nullptr, res, rh, rw, ch, cw,
                                       zoom_factors(rh, rw, ch, cw), pano, both, blended, seam_rmse);
    PYSIFT_LAUNCH_CHECK("k_blend_final");
    return PYSIFT_OK;
}

}  // extern "C"
