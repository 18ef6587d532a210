// grad.cu -- differentiable forms of the descriptor and of the warp + feather
// blend, with hand-written backward kernels (used by pysift_b200/grad.py).
//
// Descriptor (pysift/core.py:693-835 with keypoint location, scale and
// orientation held fixed): a keypoint is (centre row r0, centre column c0,
// angle in degrees) on one Gaussian level, patch half-width ph.  Each patch
// sample (r0 + dr, c0 + dc), |dr|, |dc| <= ph, inside the rotated 4x4-bin
// window contributes w_y * w_x * w_o * mag * gw to 8 trilinear bins; the
// descriptor is L2-normalise (+1e-14) -> clip 0.2 -> L2-normalise of the
// float histogram.  Backward: through the normalisation and clip to the
// histogram, then per sample through mag = |(dx, dy)|, the orientation
// theta = atan2(dy, dx) (which moves the orientation interpolation weights)
// into the central differences dx = G[r][c+1] - G[r][c-1],
// dy = G[r+1][c] - G[r-1][c] (float atomics into the level's gradient).
//
// Blur adjoint: the transpose of the separable blur with half-sample
// symmetric reflection (pysift/core.py:477-483): a reflected tap folds back
// onto the pixel it was read from.
//
// Warp + feather (float form of image.cu k_warp_feather, no uint8 rounding):
// canvas pixel (u, v) samples image 1 at (sx, sy) = Hinv (u - ox, v - oy)
// (bilinear, zero outside), image 2 sits at integer offset (iox, ioy); where
// both cover, out = (w1 d1 + i2 d2) / (d1 + d2) with d = 1 + distance to the
// image's border.  Backward: image 2 directly, image 1 by the bilinear
// weights (atomics), Hinv through (sx, sy) -> bilinear slope and the feather
// weight d1 (block reduction, then float64 atomics).  Canvas geometry and the
// homography terms are computed in float64 (the images and pixel values stay
// float32): the per-pixel terms of the homography gradient cancel over the
// canvas.
#include <cstdint>

#include "common.cuh"

namespace pysift {

constexpr int GD_T = 256;
constexpr float GD_PI = 3.14159265358979323846f;

struct DescSample {
    bool act;
    int rr, cc;
    float xr, yr, xb, yb;
};

__device__ __forceinline__ DescSample desc_sample(int idx, int side, int ph, int r0, int c0, int H, int W, float cos_a,
                                                  float sin_a, float scale_sp) {
    DescSample s;
    const int r_off = idx / side - ph, c_off = idx % side - ph;
    s.rr = r0 + r_off;
    s.cc = c0 + c_off;
    s.act = !(s.rr < 1 || s.rr >= H - 1 || s.cc < 1 || s.cc >= W - 1);
    const float fc = (float)c_off, fr = (float)r_off;
    s.xr = cos_a * fc - sin_a * fr;
    s.yr = sin_a * fc + cos_a * fr;
    s.xb = s.xr * scale_sp + 1.5f;
    s.yb = s.yr * scale_sp + 1.5f;
    s.act = s.act && !(s.xb < -0.5f || s.xb >= 3.5f || s.yb < -0.5f || s.yb >= 3.5f);
    return s;
}

struct Corners {
    int bin[8];
    float wsp[4];  // spatial weights of (y0,x0), (y0,x1), (y1,x0), (y1,x1)
    float df;      // orientation fraction: w_o0 = 1 - df, w_o1 = df
};

__device__ __forceinline__ Corners desc_corners(float xb, float yb, float ori_deg) {
    Corners k;
    const float ob = ori_deg * (8.0f / 360.0f);
    const int oi0 = (int)floorf(ob);
    k.df = ob - (float)oi0;
    const int xi0 = (int)floorf(xb), yi0 = (int)floorf(yb);
    const float dxb = xb - (float)xi0, dyb = yb - (float)yi0;
    const int xa = max(0, min(xi0, 3)), xc = max(0, min(xi0 + 1, 3));
    const int ya = max(0, min(yi0, 3)), yc = max(0, min(yi0 + 1, 3));
    const int o0 = ((oi0 % 8) + 8) % 8, o1 = ((oi0 + 1) % 8 + 8) % 8;
    k.wsp[0] = (1.0f - dyb) * (1.0f - dxb);
    k.wsp[1] = (1.0f - dyb) * dxb;
    k.wsp[2] = dyb * (1.0f - dxb);
    k.wsp[3] = dyb * dxb;
    const int sp[4] = {ya * 32 + xa * 8, ya * 32 + xc * 8, yc * 32 + xa * 8, yc * 32 + xc * 8};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        k.bin[2 * q] = sp[q] + o0;
        k.bin[2 * q + 1] = sp[q] + o1;
    }
    return k;
}

__device__ __forceinline__ float block_sum_f(float v, float* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL_MASK, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    float t = 0.0f;
    if (threadIdx.x < 32) {
        t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(FULL_MASK, t, o);
        if (threadIdx.x == 0) sh[32] = t;
    }
    __syncthreads();
    t = sh[32];
    __syncthreads();
    return t;
}

// kp: (n, 3) float rows [r0, c0, angle_deg]; hist (n, 128) raw, desc (n, 128)
__global__ void __launch_bounds__(GD_T) k_desc_f32_fwd(const float* __restrict__ G, int H, int W, long long P,
                                                       const float* __restrict__ kp, int n, int ph,
                                                       float* __restrict__ hist, float* __restrict__ desc) {
    __shared__ float h[128];
    __shared__ float sh[33];
    const float scale_sp = 4.0f / (2.0f * (float)ph);
    const float sigma_d = (float)ph * 0.5657f;
    const float inv_2s2 = 1.0f / (2.0f * sigma_d * sigma_d + 1e-12f);
    const int side = 2 * ph + 1;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        for (int b = threadIdx.x; b < 128; b += GD_T) h[b] = 0.0f;
        __syncthreads();
        const int r0 = (int)kp[3 * k], c0 = (int)kp[3 * k + 1];
        const float ang = kp[3 * k + 2] * (GD_PI / 180.0f);
        float sin_a, cos_a;
        sincosf(ang, &sin_a, &cos_a);
        for (int idx = threadIdx.x; idx < side * side; idx += GD_T) {
            const DescSample s = desc_sample(idx, side, ph, r0, c0, H, W, cos_a, sin_a, scale_sp);
            if (!s.act) continue;
            const float* gp = G + (long long)s.rr * P + s.cc;
            const float dx = gp[1] - gp[-1], dy = gp[P] - gp[-P];
            const float mag = sqrtf(dx * dx + dy * dy);
            float ori = (atan2f(dy, dx) - ang) * (180.0f / GD_PI) + 360.0f;
            ori = ori >= 360.0f ? ori - 360.0f : ori;
            const float gw = expf(-(s.xr * s.xr + s.yr * s.yr) * inv_2s2);
            const Corners c = desc_corners(s.xb, s.yb, ori);
            const float wm = mag * gw;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                atomicAdd(&h[c.bin[2 * q]], c.wsp[q] * (1.0f - c.df) * wm);
                atomicAdd(&h[c.bin[2 * q + 1]], c.wsp[q] * c.df * wm);
            }
        }
        __syncthreads();
        const float v = threadIdx.x < 128 ? h[threadIdx.x] : 0.0f;
        const float n1 = sqrtf(block_sum_f(v * v, sh) + 1e-14f);
        float t = v / n1;
        t = t > 0.2f ? 0.2f : t;
        const float n2 = sqrtf(block_sum_f(threadIdx.x < 128 ? t * t : 0.0f, sh) + 1e-14f);
        if (threadIdx.x < 128) {
            hist[(long long)k * 128 + threadIdx.x] = v;
            desc[(long long)k * 128 + threadIdx.x] = t / n2;
        }
        __syncthreads();
    }
}

// gdesc: dL/ddesc (n, 128); gG: dL/dG accumulated with atomics (pitch P)
__global__ void __launch_bounds__(GD_T) k_desc_f32_bwd(const float* __restrict__ G, int H, int W, long long P,
                                                       const float* __restrict__ kp, int n, int ph,
                                                       const float* __restrict__ hist,
                                                       const float* __restrict__ gdesc, float* __restrict__ gG) {
    __shared__ float hb[128];  // dL/dhist
    __shared__ float sh[33];
    const float scale_sp = 4.0f / (2.0f * (float)ph);
    const float sigma_d = (float)ph * 0.5657f;
    const float inv_2s2 = 1.0f / (2.0f * sigma_d * sigma_d + 1e-12f);
    const int side = 2 * ph + 1;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        // backward of L2 -> clip 0.2 -> L2
        const bool own = threadIdx.x < 128;
        const float v = own ? hist[(long long)k * 128 + threadIdx.x] : 0.0f;
        const float gd = own ? gdesc[(long long)k * 128 + threadIdx.x] : 0.0f;
        const float n1 = sqrtf(block_sum_f(v * v, sh) + 1e-14f);
        const float t = v / n1;
        const float c = t > 0.2f ? 0.2f : t;
        const float n2 = sqrtf(block_sum_f(own ? c * c : 0.0f, sh) + 1e-14f);
        const float gc_dot = block_sum_f(gd * c, sh);
        const float gcv = gd / n2 - c * gc_dot / (n2 * n2 * n2);
        const float gt = (t > 0.2f) ? 0.0f : gcv;
        const float gt_dot = block_sum_f(gt * v, sh);
        const float gh = gt / n1 - v * gt_dot / (n1 * n1 * n1);
        if (own) hb[threadIdx.x] = gh;
        __syncthreads();
        const int r0 = (int)kp[3 * k], c0 = (int)kp[3 * k + 1];
        const float ang = kp[3 * k + 2] * (GD_PI / 180.0f);
        float sin_a, cos_a;
        sincosf(ang, &sin_a, &cos_a);
        for (int idx = threadIdx.x; idx < side * side; idx += GD_T) {
            const DescSample s = desc_sample(idx, side, ph, r0, c0, H, W, cos_a, sin_a, scale_sp);
            if (!s.act) continue;
            const float* gp = G + (long long)s.rr * P + s.cc;
            const float dx = gp[1] - gp[-1], dy = gp[P] - gp[-P];
            const float m2 = dx * dx + dy * dy;
            if (!(m2 > 0.0f)) continue;
            const float mag = sqrtf(m2);
            float ori = (atan2f(dy, dx) - ang) * (180.0f / GD_PI) + 360.0f;
            ori = ori >= 360.0f ? ori - 360.0f : ori;
            const float gw = expf(-(s.xr * s.xr + s.yr * s.yr) * inv_2s2);
            const Corners cr = desc_corners(s.xb, s.yb, ori);
            float gmag = 0.0f, gdf = 0.0f;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float g0 = hb[cr.bin[2 * q]], g1 = hb[cr.bin[2 * q + 1]];
                gmag += cr.wsp[q] * ((1.0f - cr.df) * g0 + cr.df * g1);
                gdf += cr.wsp[q] * (g1 - g0);
            }
            gmag *= gw;
            // d(df)/d(theta) = (180 / pi) / 45 per radian
            const float gth = gdf * gw * mag * (4.0f / GD_PI);
            const float gdx = gmag * dx / mag - gth * dy / m2;
            const float gdy = gmag * dy / mag + gth * dx / m2;
            float* g = gG + (long long)s.rr * P + s.cc;
            atomicAdd(g + 1, gdx);
            atomicAdd(g - 1, -gdx);
            atomicAdd(g + P, gdy);
            atomicAdd(g - P, -gdy);
        }
        __syncthreads();
    }
}

// One axis of the adjoint of y[i] = sum_k w[k] x[refl(i + k - R)] (half-sample
// symmetric reflection, R < n): x_bar[j] = sum_k w[k] sum over the reads of
// pixel j.  axis 0: along rows (x), axis 1: along columns (y).  out = in^T-applied.
__global__ void k_blur_adjoint_axis(const float* __restrict__ in, long long in_pitch, float* __restrict__ out,
                                    long long out_pitch, int H, int W, const float* __restrict__ w, int R, int axis,
                                    int accumulate) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    const int n = axis == 0 ? W : H, j = axis == 0 ? x : y;
    float acc = 0.0f;
    for (int k = 0; k <= 2 * R; ++k) {
        const float wk = w[k];
        const int cand[3] = {j - k + R, -1 - j - k + R, 2 * n - 1 - j - k + R};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int i = cand[q];
            if (i < 0 || i >= n) continue;
            if (q == 1 && -1 - j == j) continue;            // never (j >= 0)
            if (q == 2 && 2 * n - 1 - j == j) continue;     // never (j <= n - 1)
            const float v = axis == 0 ? in[(long long)y * in_pitch + i] : in[(long long)i * in_pitch + x];
            acc += wk * v;
        }
    }
    float* o = out + (long long)y * out_pitch + x;
    *o = accumulate ? *o + acc : acc;
}

struct WarpF32Args {
    const float* img1;
    int hs, ws, C;
    const float* img2;
    int h2, w2;
    int cw, ch;
    double hinv[9];
    double ox, oy;
    int iox, ioy;
    float* out;      // (ch, cw, C)
    const float* gout;
    float* gimg1;    // (hs, ws, C), atomics
    float* gimg2;    // (h2, w2, C)
    double* ghinv;   // 9, atomics
};

struct WarpGeom {
    bool v1, v2, clamped;
    double X, Y, den, sx, sy;
    float d1, d2;
    int x0, y0, x2, y2;
    float fx, fy;
};

__device__ __forceinline__ WarpGeom warp_geom(const WarpF32Args& a, int u, int v) {
    WarpGeom g;
    g.X = (double)u - a.ox;
    g.Y = (double)v - a.oy;
    const double s0 = a.hinv[0] * g.X + a.hinv[1] * g.Y + a.hinv[2];
    const double s1 = a.hinv[3] * g.X + a.hinv[4] * g.Y + a.hinv[5];
    const double s2 = a.hinv[6] * g.X + a.hinv[7] * g.Y + a.hinv[8];
    g.clamped = !(s2 >= 1e-10);
    g.den = g.clamped ? 1e-10 : s2;
    g.sx = s0 / g.den;
    g.sy = s1 / g.den;
    g.v1 = g.sx >= 0.0 && g.sx <= (double)(a.ws - 1) && g.sy >= 0.0 && g.sy <= (double)(a.hs - 1);
    g.x0 = (int)floor(g.sx);
    g.y0 = (int)floor(g.sy);
    g.fx = (float)(g.sx - (double)g.x0);
    g.fy = (float)(g.sy - (double)g.y0);
    g.d1 = (float)(1.0 + fmin(fmin(g.sx, (double)(a.ws - 1) - g.sx), fmin(g.sy, (double)(a.hs - 1) - g.sy)));
    g.x2 = u - a.iox;
    g.y2 = v - a.ioy;
    g.v2 = g.x2 >= 0 && g.x2 < a.w2 && g.y2 >= 0 && g.y2 < a.h2;
    g.d2 = 1.0f + (float)min(min(g.x2, a.w2 - 1 - g.x2), min(g.y2, a.h2 - 1 - g.y2));
    return g;
}

__device__ __forceinline__ float img1_at(const WarpF32Args& a, int x, int y, int c) {
    return (x >= 0 && x < a.ws && y >= 0 && y < a.hs) ? a.img1[((long long)y * a.ws + x) * a.C + c] : 0.0f;
}

__global__ void k_warp_f32_fwd(const WarpF32Args a) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= a.cw) return;
    const WarpGeom g = warp_geom(a, u, v);
    for (int c = 0; c < a.C; ++c) {
        float w1 = 0.0f;
        if (g.v1) {
            const float p00 = img1_at(a, g.x0, g.y0, c), p01 = img1_at(a, g.x0 + 1, g.y0, c);
            const float p10 = img1_at(a, g.x0, g.y0 + 1, c), p11 = img1_at(a, g.x0 + 1, g.y0 + 1, c);
            w1 = (1.0f - g.fy) * ((1.0f - g.fx) * p00 + g.fx * p01) + g.fy * ((1.0f - g.fx) * p10 + g.fx * p11);
        }
        const float i2 = g.v2 ? a.img2[((long long)g.y2 * a.w2 + g.x2) * a.C + c] : 0.0f;
        float o = 0.0f;
        if (g.v1 && g.v2) o = (w1 * g.d1 + i2 * g.d2) / (g.d1 + g.d2);
        else if (g.v2) o = i2;
        else if (g.v1) o = w1;
        a.out[((long long)v * a.cw + u) * a.C + c] = o;
    }
}

__global__ void __launch_bounds__(256) k_warp_f32_bwd(const WarpF32Args a) {
    __shared__ double sh[9][8];
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    double gh[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (u < a.cw) {
        const WarpGeom g = warp_geom(a, u, v);
        double gsx = 0.0, gsy = 0.0, gd1 = 0.0;
        for (int c = 0; c < a.C; ++c) {
            const float go = a.gout[((long long)v * a.cw + u) * a.C + c];
            float w1 = 0.0f, dwdx = 0.0f, dwdy = 0.0f, p00 = 0, p01 = 0, p10 = 0, p11 = 0;
            if (g.v1) {
                p00 = img1_at(a, g.x0, g.y0, c);
                p01 = img1_at(a, g.x0 + 1, g.y0, c);
                p10 = img1_at(a, g.x0, g.y0 + 1, c);
                p11 = img1_at(a, g.x0 + 1, g.y0 + 1, c);
                w1 = (1.0f - g.fy) * ((1.0f - g.fx) * p00 + g.fx * p01) + g.fy * ((1.0f - g.fx) * p10 + g.fx * p11);
                dwdx = (1.0f - g.fy) * (p01 - p00) + g.fy * (p11 - p10);
                dwdy = (1.0f - g.fx) * (p10 - p00) + g.fx * (p11 - p01);
            }
            float gw1 = 0.0f;
            if (g.v1 && g.v2) {
                const float i2 = a.img2[((long long)g.y2 * a.w2 + g.x2) * a.C + c];
                const float s = g.d1 + g.d2;
                const float o = (w1 * g.d1 + i2 * g.d2) / s;
                gw1 = go * g.d1 / s;
                a.gimg2[((long long)g.y2 * a.w2 + g.x2) * a.C + c] += go * g.d2 / s;
                gd1 += go * (w1 - o) / s;
            } else if (g.v2) {
                a.gimg2[((long long)g.y2 * a.w2 + g.x2) * a.C + c] += go;
            } else if (g.v1) {
                gw1 = go;
            }
            if (g.v1 && gw1 != 0.0f) {
                const float wts[4] = {(1.0f - g.fy) * (1.0f - g.fx), (1.0f - g.fy) * g.fx, g.fy * (1.0f - g.fx),
                                      g.fy * g.fx};
                const int xs[4] = {g.x0, g.x0 + 1, g.x0, g.x0 + 1}, ys[4] = {g.y0, g.y0, g.y0 + 1, g.y0 + 1};
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (xs[q] >= 0 && xs[q] < a.ws && ys[q] >= 0 && ys[q] < a.hs)
                        atomicAdd(&a.gimg1[((long long)ys[q] * a.ws + xs[q]) * a.C + c], gw1 * wts[q]);
                gsx += gw1 * dwdx;
                gsy += gw1 * dwdy;
            }
        }
        if (g.v1 && g.v2) {
            // d1 = 1 + min(sx, ws-1-sx, sy, hs-1-sy): slope of the active term
            const double t0 = g.sx, t1 = (double)(a.ws - 1) - g.sx, t2 = g.sy, t3 = (double)(a.hs - 1) - g.sy;
            const double m = fmin(fmin(t0, t1), fmin(t2, t3));
            if (m == t0) gsx += gd1;
            else if (m == t1) gsx -= gd1;
            else if (m == t2) gsy += gd1;
            else gsy -= gd1;
        }
        if (g.v1 && !g.clamped) {
            const double a0 = gsx / g.den, a1 = gsy / g.den, a2 = -(gsx * g.sx + gsy * g.sy) / g.den;
            gh[0] = a0 * g.X; gh[1] = a0 * g.Y; gh[2] = a0;
            gh[3] = a1 * g.X; gh[4] = a1 * g.Y; gh[5] = a1;
            gh[6] = a2 * g.X; gh[7] = a2 * g.Y; gh[8] = a2;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        double x = gh[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL_MASK, x, o);
        if (lane == 0) sh[q][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[threadIdx.x][w];
        atomicAdd(&a.ghinv[threadIdx.x], s);
    }
}

}  // namespace pysift

using namespace pysift;

extern "C" {

int pysift_desc_f32_forward(const float* level, int32_t H, int32_t W, int32_t pitch, const float* kp, int32_t n,
                            int32_t ph, float* hist, float* desc, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(level && kp && hist && desc && H > 2 && W > 2 && pitch >= W && n >= 0 && ph >= 1 && ph <= 200,
                     "bad arguments");
    if (n == 0) return PYSIFT_OK;
    k_desc_f32_fwd<<<std::min(n, 148 * 8), GD_T, 0, reinterpret_cast<cudaStream_t>(stream)>>>(level, H, W, pitch, kp,
                                                                                             n, ph, hist, desc);
    PYSIFT_LAUNCH_CHECK("k_desc_f32_fwd");
    return PYSIFT_OK;
}

int pysift_desc_f32_backward(const float* level, int32_t H, int32_t W, int32_t pitch, const float* kp, int32_t n,
                             int32_t ph, const float* hist, const float* gdesc, float* glevel,
                             pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(level && kp && hist && gdesc && glevel && H > 2 && W > 2 && pitch >= W && n >= 0 && ph >= 1 &&
                         ph <= 200,
                     "bad arguments");
    if (n == 0) return PYSIFT_OK;
    k_desc_f32_bwd<<<std::min(n, 148 * 8), GD_T, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        level, H, W, pitch, kp, n, ph, hist, gdesc, glevel);
    PYSIFT_LAUNCH_CHECK("k_desc_f32_bwd");
    return PYSIFT_OK;
}

int pysift_blur_adjoint(const float* gout, int32_t gout_pitch, float* gin, int32_t gin_pitch, float* tmp,
                        int32_t tmp_pitch, int32_t H, int32_t W, const float* weights_dev, int32_t radius,
                        int32_t accumulate, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(gout && gin && tmp && weights_dev && H > 0 && W > 0, "bad arguments");
    PYSIFT_CHECK_ARG(radius >= 0 && radius < H && radius < W && radius <= PYSIFT_MAX_RADIUS,
                     "radius %d must be below both image sides", radius);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    dim3 grid(ceil_div(W, 128), H);
    // forward = horizontal then vertical; adjoint = vertical^T then horizontal^T
    k_blur_adjoint_axis<<<grid, 128, 0, st>>>(gout, gout_pitch, tmp, tmp_pitch, H, W, weights_dev, radius, 1, 0);
    PYSIFT_LAUNCH_CHECK("k_blur_adjoint_axis");
    k_blur_adjoint_axis<<<grid, 128, 0, st>>>(tmp, tmp_pitch, gin, gin_pitch, H, W, weights_dev, radius, 0, accumulate);
    PYSIFT_LAUNCH_CHECK("k_blur_adjoint_axis");
    return PYSIFT_OK;
}

static int warp_args(WarpF32Args& a, const float* img1, int32_t hs, int32_t ws, int32_t C, const float* img2,
                     int32_t h2, int32_t w2, int32_t cw, int32_t ch, const double* hinv, double ox, double oy,
                     int32_t iox, int32_t ioy) {
    PYSIFT_CHECK_ARG(img1 && img2 && hinv && hs > 1 && ws > 1 && h2 > 0 && w2 > 0 && cw > 0 && ch > 0 && C >= 1 &&
                         C <= 4,
                     "bad arguments");
    a.img1 = img1;
    a.hs = hs;
    a.ws = ws;
    a.C = C;
    a.img2 = img2;
    a.h2 = h2;
    a.w2 = w2;
    a.cw = cw;
    a.ch = ch;
    for (int i = 0; i < 9; ++i) a.hinv[i] = hinv[i];
    a.ox = ox;
    a.oy = oy;
    a.iox = iox;
    a.ioy = ioy;
    return PYSIFT_OK;
}

int pysift_warp_f32_forward(const float* img1, int32_t hs, int32_t ws, int32_t C, const float* img2, int32_t h2,
                            int32_t w2, int32_t cw, int32_t ch, const double* hinv_host, double ox, double oy,
                            int32_t iox, int32_t ioy, float* out, pysift_stream_t stream) {
    WarpF32Args a = {};
    int rc = warp_args(a, img1, hs, ws, C, img2, h2, w2, cw, ch, hinv_host, ox, oy, iox, ioy);
    if (rc) return rc;
    PYSIFT_CHECK_ARG(out != nullptr, "out is NULL");
    a.out = out;
    k_warp_f32_fwd<<<dim3(ceil_div(cw, 256), ch), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
    PYSIFT_LAUNCH_CHECK("k_warp_f32_fwd");
    return PYSIFT_OK;
}

int pysift_warp_f32_backward(const float* img1, int32_t hs, int32_t ws, int32_t C, const float* img2, int32_t h2,
                             int32_t w2, int32_t cw, int32_t ch, const double* hinv_host, double ox, double oy,
                             int32_t iox, int32_t ioy, const float* gout, float* gimg1, float* gimg2, double* ghinv,
                             pysift_stream_t stream) {
    WarpF32Args a = {};
    int rc = warp_args(a, img1, hs, ws, C, img2, h2, w2, cw, ch, hinv_host, ox, oy, iox, ioy);
    if (rc) return rc;
    PYSIFT_CHECK_ARG(gout && gimg1 && gimg2 && ghinv, "NULL gradient buffer");
    a.gout = gout;
    a.gimg1 = gimg1;
    a.gimg2 = gimg2;
    a.ghinv = ghinv;
    k_warp_f32_bwd<<<dim3(ceil_div(cw, 256), ch), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
    PYSIFT_LAUNCH_CHECK("k_warp_f32_bwd");
    return PYSIFT_OK;
}

}  // extern "C"
