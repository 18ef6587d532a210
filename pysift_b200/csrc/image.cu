// image.cu -- colour conversion, CLAHE, homography warp + feather blend.
//
//   k_bgr2gray      cv2.cvtColor(COLOR_BGR2GRAY) for uint8 (pysift/core.py:2546):
//                   (3735 B + 19235 G + 9798 R + 2^14) >> 15
//   k_clahe_lut     cv2.createCLAHE(clip, 8x8).apply, per-tile histogram, clip,
//   k_clahe_apply   redistribution, LUT, bilinear LUT interpolation
//                   (pysift/core.py:2563-2565); bottom/right reflect-101 extension
//                   when the size is not a multiple of the tile grid
//   k_warp_feather  inverse-map bilinear warp of image 1 onto the canvas with the
//                   reference's float32 arithmetic and grid_sample(bilinear, zeros,
//                   align_corners=True) semantics, uint8 truncation
//                   (pysift/core.py:3210-3239), placement of image 2
//                   (pysift/core.py:3794-3800) and a linear feather blend where both
//                   images cover the canvas; per-row/column coverage extents for the
//                   inner-rectangle crop (pysift/core.py:3627-3684)
#include <cstdint>

#include "common.cuh"

namespace pysift {

__global__ void k_bgr2gray(const uint8_t* __restrict__ bgr, int H, int W, long long pitch, uint8_t* __restrict__ gray,
                           int gray_pitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const uint8_t* p = bgr + (long long)y * pitch + 3 * x;
    const int v = (p[0] * 3735 + p[1] * 19235 + p[2] * 9798 + (1 << 14)) >> 15;
    gray[(long long)y * gray_pitch + x] = (uint8_t)v;
}

__device__ __forceinline__ int reflect101(int i, int n) {
    if (n <= 1) return 0;
    while (i < 0 || i >= n) {
        if (i < 0) i = -i;
        if (i >= n) i = 2 * n - 2 - i;
    }
    return i;
}

struct ClaheArgs {
    const uint8_t* src;
    int H, W, pitch;
    int tiles_x, tiles_y, tile_w, tile_h;  // tile size of the (extended) image
    int clip_limit;                        // 0 = no clipping
    float lut_scale;
    uint8_t* lut;  // [tiles_y][tiles_x][256]
    uint8_t* dst;
    int dst_pitch;
};

// One block per tile: 256-bin histogram, clip + redistribution, LUT.
__global__ void __launch_bounds__(256) k_clahe_lut(const ClaheArgs a) {
    __shared__ unsigned int hist[256];
    __shared__ int sh[33];
    __shared__ int s_clipped;
    const int tx = blockIdx.x, ty = blockIdx.y, t = threadIdx.x;
    hist[t] = 0u;
    if (t == 0) s_clipped = 0;
    __syncthreads();
    const int x0 = tx * a.tile_w, y0 = ty * a.tile_h;
    {
        // element i = t + 256 k of the tile, walked without a division per
        // element; loads go out CL_B at a time before their counts
        constexpr int CL_B = 16;
        const int area = a.tile_w * a.tile_h;
        const int sy = 256 / a.tile_w, sx = 256 - sy * a.tile_w;
        int yy = t / a.tile_w, xx = t - yy * a.tile_w;
        const bool inside = y0 + a.tile_h <= a.H && x0 + a.tile_w <= a.W;
        for (int i0 = t; i0 < area; i0 += 256 * CL_B) {
            uint8_t v[CL_B];
#pragma unroll
            for (int k = 0; k < CL_B; ++k) {
                v[k] = 0;
                if (i0 + 256 * k < area) {
                    const int gy = y0 + yy, gx = x0 + xx;
                    const long long off = inside ? (long long)gy * a.pitch + gx
                                                 : (long long)reflect101(gy, a.H) * a.pitch + reflect101(gx, a.W);
                    v[k] = a.src[off];
                }
                xx += sx;
                yy += sy;
                if (xx >= a.tile_w) {
                    xx -= a.tile_w;
                    ++yy;
                }
            }
#pragma unroll
            for (int k = 0; k < CL_B; ++k)
                if (i0 + 256 * k < area) atomicAdd(&hist[v[k]], 1u);
        }
    }
    __syncthreads();
    int h = (int)hist[t];
    if (a.clip_limit > 0) {
        if (h > a.clip_limit) {
            atomicAdd(&s_clipped, h - a.clip_limit);
            h = a.clip_limit;
        }
        __syncthreads();
        const int clipped = s_clipped;
        const int batch = clipped / 256;
        const int resid = clipped - batch * 256;
        h += batch;
        if (resid != 0) {
            const int step = max(256 / resid, 1);
            if (t % step == 0 && t / step < resid) h += 1;
        }
    }
    int total;
    const int cum = block_excl_scan(h, &total, sh) + h;
    float v = (float)cum * a.lut_scale;
    int q = __float2int_rn(v);
    q = q < 0 ? 0 : (q > 255 ? 255 : q);
    a.lut[((long long)ty * a.tiles_x + tx) * 256 + t] = (uint8_t)q;
}

__global__ void k_clahe_apply(const ClaheArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= a.W) return;
    const float inv_tw = 1.0f / (float)a.tile_w, inv_th = 1.0f / (float)a.tile_h;
    const float txf = (float)x * inv_tw - 0.5f;
    int tx1 = (int)floorf(txf);
    int tx2 = tx1 + 1;
    const float xa = txf - (float)tx1, xa1 = 1.0f - xa;
    tx1 = max(tx1, 0);
    tx2 = min(tx2, a.tiles_x - 1);
    const float tyf = (float)y * inv_th - 0.5f;
    int ty1 = (int)floorf(tyf);
    int ty2 = ty1 + 1;
    const float ya = tyf - (float)ty1, ya1 = 1.0f - ya;
    ty1 = max(ty1, 0);
    ty2 = min(ty2, a.tiles_y - 1);
    const int v = a.src[(long long)y * a.pitch + x];
    const uint8_t* l1 = a.lut + (long long)ty1 * a.tiles_x * 256;
    const uint8_t* l2 = a.lut + (long long)ty2 * a.tiles_x * 256;
    const float res = ((float)l1[tx1 * 256 + v] * xa1 + (float)l1[tx2 * 256 + v] * xa) * ya1 +
                      ((float)l2[tx1 * 256 + v] * xa1 + (float)l2[tx2 * 256 + v] * xa) * ya;
    int q = __float2int_rn(res);
    q = q < 0 ? 0 : (q > 255 ? 255 : q);
    a.dst[(long long)y * a.dst_pitch + x] = (uint8_t)q;
}

struct WarpArgs {
    const uint8_t* img1;  // hs x ws x 3
    int hs, ws, pitch1;
    const uint8_t* img2;  // h2 x w2 x 3
    int h2, w2, pitch2;
    int cw, ch;
    float hinv[9];  // float32 inverse homography (canvas - offset -> image 1)
    float ox, oy;   // float32 canvas offset
    int iox, ioy;   // integer placement of image 2
    int feather;    // 1: linear feather where both cover; 0: warped image 1 only
    uint8_t* out;   // ch x cw x 3
    uint8_t* warped;  // optional: warped image 1 alone (ch x cw x 3)
    uint8_t* mask1;   // optional
    uint8_t* mask2;   // optional
    int* row_lo;      // [ch] min x covered, atomics
    int* row_hi;
    int* col_lo;      // [cw] min y covered
    int* col_hi;
};

__global__ void __launch_bounds__(256) k_warp_feather(const WarpArgs a) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= a.cw) return;
    // src = Hinv @ (u - ox, v - oy, 1) in float32 (pysift/core.py:3223-3228)
    const float X = (float)u - a.ox, Y = (float)v - a.oy;
    const float s0 = a.hinv[0] * X + a.hinv[1] * Y + a.hinv[2];
    const float s1 = a.hinv[3] * X + a.hinv[4] * Y + a.hinv[5];
    const float s2 = a.hinv[6] * X + a.hinv[7] * Y + a.hinv[8];
    const float den = s2 < 1e-10f ? 1e-10f : s2;
    const float sx = s0 / den, sy = s1 / den;
    const float sxn = (2.0f * sx / (float)(a.ws - 1)) - 1.0f;
    const float syn = (2.0f * sy / (float)(a.hs - 1)) - 1.0f;
    const bool valid1 = (sxn >= -1.0f) && (sxn <= 1.0f) && (syn >= -1.0f) && (syn <= 1.0f);
    // grid_sample(bilinear, zeros, align_corners=True)
    const float ix = ((sxn + 1.0f) / 2.0f) * (float)(a.ws - 1);
    const float iy = ((syn + 1.0f) / 2.0f) * (float)(a.hs - 1);
    const float fx = floorf(ix), fy = floorf(iy);
    const int ix_nw = (int)fx, iy_nw = (int)fy;
    const float ix_se = fx + 1.0f, iy_se = fy + 1.0f;
    const float w_nw = (ix_se - ix) * (iy_se - iy);
    const float w_ne = (ix - fx) * (iy_se - iy);
    const float w_sw = (ix_se - ix) * (iy - fy);
    const float w_se = (ix - fx) * (iy - fy);
    float c1[3] = {0.0f, 0.0f, 0.0f};
    const bool in_nw = ix_nw >= 0 && ix_nw < a.ws && iy_nw >= 0 && iy_nw < a.hs;
    const bool in_ne = ix_nw + 1 >= 0 && ix_nw + 1 < a.ws && iy_nw >= 0 && iy_nw < a.hs;
    const bool in_sw = ix_nw >= 0 && ix_nw < a.ws && iy_nw + 1 >= 0 && iy_nw + 1 < a.hs;
    const bool in_se = ix_nw + 1 >= 0 && ix_nw + 1 < a.ws && iy_nw + 1 >= 0 && iy_nw + 1 < a.hs;
    const bool finite = isfinite(ix) && isfinite(iy) && fabsf(ix) < 1e9f && fabsf(iy) < 1e9f;
    if (finite) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float acc = 0.0f;
            if (in_nw) acc = fmaf((float)a.img1[(long long)iy_nw * a.pitch1 + 3 * ix_nw + c], w_nw, acc);
            if (in_ne) acc = fmaf((float)a.img1[(long long)iy_nw * a.pitch1 + 3 * (ix_nw + 1) + c], w_ne, acc);
            if (in_sw) acc = fmaf((float)a.img1[(long long)(iy_nw + 1) * a.pitch1 + 3 * ix_nw + c], w_sw, acc);
            if (in_se) acc = fmaf((float)a.img1[(long long)(iy_nw + 1) * a.pitch1 + 3 * (ix_nw + 1) + c], w_se, acc);
            c1[c] = acc;
        }
    }
    uint8_t w1b[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float t = c1[c] < 0.0f ? 0.0f : (c1[c] > 255.0f ? 255.0f : c1[c]);
        w1b[c] = (uint8_t)(int)t;  // numpy astype(uint8) truncation
    }
    const int x2 = u - a.iox, y2 = v - a.ioy;
    const bool valid2 = x2 >= 0 && x2 < a.w2 && y2 >= 0 && y2 < a.h2;
    const long long o = ((long long)v * a.cw + u) * 3;
    if (a.warped) {
#pragma unroll
        for (int c = 0; c < 3; ++c) a.warped[o + c] = w1b[c];
    }
    if (a.mask1) a.mask1[(long long)v * a.cw + u] = valid1;
    if (a.mask2) a.mask2[(long long)v * a.cw + u] = valid2;
    if (a.row_lo) {
        // the lanes of a warp share the row: one min / max per warp for the
        // row extents (same-address atomics serialise), one per pixel for the
        // columns (distinct addresses)
        const bool cov = valid1 || valid2;
        const unsigned am = __activemask();
        const unsigned cm = __ballot_sync(am, cov);
        if (cm) {
            const int lo = __reduce_min_sync(am, cov ? u : 0x7fffffff);
            const int hi = __reduce_max_sync(am, cov ? u : -1);
            if ((int)(threadIdx.x & 31) == __ffs(cm) - 1) {
                atomicMin(&a.row_lo[v], lo);
                atomicMax(&a.row_hi[v], hi);
            }
        }
        if (cov) {
            atomicMin(&a.col_lo[u], v);
            atomicMax(&a.col_hi[u], v);
        }
    }
    if (!a.out) return;
    uint8_t res[3] = {0, 0, 0};
    if (valid1 && valid2 && a.feather) {
        // linear feather: weights = 1 + distance to the nearest border of each image
        const float d1 = 1.0f + fminf(fminf(ix, (float)(a.ws - 1) - ix), fminf(iy, (float)(a.hs - 1) - iy));
        const float d2 = 1.0f + (float)min(min(x2, a.w2 - 1 - x2), min(y2, a.h2 - 1 - y2));
        const uint8_t* p2 = a.img2 + (long long)y2 * a.pitch2 + 3 * x2;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float val = ((float)w1b[c] * d1 + (float)p2[c] * d2) / (d1 + d2);
            float t = val + 0.5f;
            t = t < 0.0f ? 0.0f : (t > 255.0f ? 255.0f : t);
            res[c] = (uint8_t)(int)t;
        }
    } else if (valid2) {
        const uint8_t* p2 = a.img2 + (long long)y2 * a.pitch2 + 3 * x2;
        res[0] = p2[0];
        res[1] = p2[1];
        res[2] = p2[2];
    } else if (valid1) {
        res[0] = w1b[0];
        res[1] = w1b[1];
        res[2] = w1b[2];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) a.out[o + c] = res[c];
}

__global__ void k_fill_int(int* p, int n, int value) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = value;
}

// rank[i] = #{j : (resp_j, j) precedes (resp_i, i)} under descending response,
// ascending index; integer atomics over (i-tile, j-tile) pairs.
__global__ void __launch_bounds__(256) k_resp_rank(const float* __restrict__ resp, int n, int* __restrict__ rank) {
    __shared__ float tile[256];
    const int nt = (n + 255) / 256;
    for (long long t = blockIdx.x; t < (long long)nt * nt; t += gridDim.x) {
        const int ti = (int)(t / nt), tj = (int)(t - (long long)ti * nt);
        __syncthreads();
        const int j = tj * 256 + threadIdx.x;
        if (j < n) tile[threadIdx.x] = resp[j];
        __syncthreads();
        const int i = ti * 256 + threadIdx.x;
        if (i < n) {
            const float me = resp[i];
            const int m = min(256, n - tj * 256);
            int cnt = 0;
            for (int k = 0; k < m; ++k) {
                const float o = tile[k];
                const int jj = tj * 256 + k;
                cnt += (o > me || (o == me && jj < i)) ? 1 : 0;
            }
            if (cnt) atomicAdd(&rank[i], cnt);
        }
    }
}

__global__ void k_topk_scatter(const int* __restrict__ rank, int n, int k, int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && rank[i] < k) out[rank[i]] = i;
}

__global__ void k_gather_points(const float* __restrict__ kpts, const int* __restrict__ pairs,
                                const int* __restrict__ count, int max_pairs, int col, double* __restrict__ pts) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= max_pairs || m >= *count) return;
    const int idx = pairs[2 * m + col];
    pts[2 * m] = (double)kpts[4 * idx];
    pts[2 * m + 1] = (double)kpts[4 * idx + 1];
}

}  // namespace pysift

using namespace pysift;

// OpenCV's uint8 SIFT descriptor: saturate(rint(512 v)) of the L2 / clip 0.2 /
// L2 vector (512 v is exact in float32; rint rounds half to even)
__global__ void k_desc_to_u8(const float* __restrict__ desc, long long n, uint8_t* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = rintf(desc[i] * 512.0f);
    v = v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v);
    out[i] = (uint8_t)(int)v;
}

extern "C" {

int pysift_bgr2gray(const uint8_t* bgr, int32_t H, int32_t W, int64_t pitch_bytes, uint8_t* gray, int32_t gray_pitch,
                    pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(bgr && gray, "NULL pointer argument");
    PYSIFT_CHECK_ARG(H > 0 && W > 0 && pitch_bytes >= 3 * (int64_t)W && gray_pitch >= W, "bad sizes");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_bgr2gray<<<dim3(ceil_div(W, 256), H), 256, 0, st>>>(bgr, H, W, pitch_bytes, gray, gray_pitch);
    PYSIFT_LAUNCH_CHECK("k_bgr2gray");
    return PYSIFT_OK;
}

int pysift_clahe_lut_bytes(int32_t tiles_x, int32_t tiles_y, size_t* bytes) {
    PYSIFT_CHECK_ARG(bytes && tiles_x > 0 && tiles_y > 0, "bad arguments");
    *bytes = (size_t)tiles_x * tiles_y * 256;
    return PYSIFT_OK;
}

int pysift_clahe(const uint8_t* src, int32_t H, int32_t W, int32_t pitch, double clip_limit, int32_t tiles_x,
                 int32_t tiles_y, uint8_t* lut, uint8_t* dst, int32_t dst_pitch, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(src && lut && dst, "NULL pointer argument");
    PYSIFT_CHECK_ARG(H > 0 && W > 0 && pitch >= W && dst_pitch >= W && tiles_x > 0 && tiles_y > 0, "bad sizes");
    ClaheArgs a;
    a.src = src;
    a.H = H;
    a.W = W;
    a.pitch = pitch;
    a.tiles_x = tiles_x;
    a.tiles_y = tiles_y;
    // cv2's CLAHE extends the image (reflect-101) only when a side does not
    // divide by its tile count, and then extends BOTH sides by
    // tiles - size % tiles: a side that divides gains a whole tile count
    const bool exact = (W % tiles_x == 0) && (H % tiles_y == 0);
    const int ew = exact ? W : W + (tiles_x - W % tiles_x);
    const int eh = exact ? H : H + (tiles_y - H % tiles_y);
    a.tile_w = ew / tiles_x;
    a.tile_h = eh / tiles_y;
    const int area = a.tile_w * a.tile_h;
    a.lut_scale = 255.0f / (float)area;
    a.clip_limit = 0;
    if (clip_limit > 0.0) {
        int cl = (int)(clip_limit * area / 256);
        a.clip_limit = cl < 1 ? 1 : cl;
    }
    a.lut = lut;
    a.dst = dst;
    a.dst_pitch = dst_pitch;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_clahe_lut<<<dim3(tiles_x, tiles_y), 256, 0, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_clahe_lut");
    k_clahe_apply<<<dim3(ceil_div(W, 256), H), 256, 0, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_clahe_apply");
    return PYSIFT_OK;
}

int pysift_warp_feather(const uint8_t* img1, int32_t hs, int32_t ws, int32_t pitch1, const uint8_t* img2, int32_t h2,
                        int32_t w2, int32_t pitch2, int32_t cw, int32_t ch, const float* hinv9, float ox, float oy,
                        int32_t iox, int32_t ioy, int32_t feather, uint8_t* out, uint8_t* warped, uint8_t* mask1,
                        uint8_t* mask2, int32_t* row_lo, int32_t* row_hi, int32_t* col_lo, int32_t* col_hi,
                        pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(img1 && img2 && hinv9, "NULL pointer argument");
    PYSIFT_CHECK_ARG(out || (warped && mask1), "no output requested");
    PYSIFT_CHECK_ARG(hs > 1 && ws > 1 && h2 > 0 && w2 > 0 && cw > 0 && ch > 0, "bad sizes");
    PYSIFT_CHECK_ARG((row_lo && row_hi && col_lo && col_hi) || !(row_lo || row_hi || col_lo || col_hi),
                     "extents must be all or none");
    WarpArgs a;
    a.img1 = img1;
    a.hs = hs;
    a.ws = ws;
    a.pitch1 = pitch1;
    a.img2 = img2;
    a.h2 = h2;
    a.w2 = w2;
    a.pitch2 = pitch2;
    a.cw = cw;
    a.ch = ch;
    for (int i = 0; i < 9; ++i) a.hinv[i] = hinv9[i];
    a.ox = ox;
    a.oy = oy;
    a.iox = iox;
    a.ioy = ioy;
    a.feather = feather;
    a.out = out;
    a.warped = warped;
    a.mask1 = mask1;
    a.mask2 = mask2;
    a.row_lo = row_lo;
    a.row_hi = row_hi;
    a.col_lo = col_lo;
    a.col_hi = col_hi;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (row_lo) {
        k_fill_int<<<ceil_div(ch, 256), 256, 0, st>>>(row_lo, ch, 0x7fffffff);
        PYSIFT_LAUNCH_CHECK("k_fill_int");
        k_fill_int<<<ceil_div(ch, 256), 256, 0, st>>>(row_hi, ch, -1);
        PYSIFT_LAUNCH_CHECK("k_fill_int");
        k_fill_int<<<ceil_div(cw, 256), 256, 0, st>>>(col_lo, cw, 0x7fffffff);
        PYSIFT_LAUNCH_CHECK("k_fill_int");
        k_fill_int<<<ceil_div(cw, 256), 256, 0, st>>>(col_hi, cw, -1);
        PYSIFT_LAUNCH_CHECK("k_fill_int");
    }
    k_warp_feather<<<dim3(ceil_div(cw, 256), ch), 256, 0, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_warp_feather");
    return PYSIFT_OK;
}

int pysift_topk_by_response(const float* response, int32_t n, int32_t k, int32_t* rank, int32_t* out_idx,
                            pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(response && rank && out_idx && n >= 0 && k >= 0 && k <= n, "bad arguments");
    if (n == 0 || k == 0) return PYSIFT_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    PYSIFT_CUDA_TRY(cudaMemsetAsync(rank, 0, sizeof(int32_t) * (size_t)n, st));
    k_resp_rank<<<1184, 256, 0, st>>>(response, n, rank);
    PYSIFT_LAUNCH_CHECK("k_resp_rank");
    k_topk_scatter<<<ceil_div(n, 256), 256, 0, st>>>(rank, n, k, out_idx);
    PYSIFT_LAUNCH_CHECK("k_topk_scatter");
    return PYSIFT_OK;
}

int pysift_gather_points(const float* kpts, const int32_t* pairs, const int32_t* count, int32_t max_pairs, int32_t col,
                         double* pts, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(kpts && pairs && count && pts && max_pairs >= 0 && (col == 0 || col == 1), "bad arguments");
    if (max_pairs == 0) return PYSIFT_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_gather_points<<<ceil_div(max_pairs, 256), 256, 0, st>>>(kpts, pairs, count, max_pairs, col, pts);
    PYSIFT_LAUNCH_CHECK("k_gather_points");
    return PYSIFT_OK;
}

int pysift_desc_to_u8(const float* desc, int64_t n_rows, uint8_t* out, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(n_rows >= 0, "bad sizes");
    if (n_rows == 0) return PYSIFT_OK;
    PYSIFT_CHECK_ARG(desc && out, "NULL pointer argument");
    const long long n = (long long)n_rows * 128;
    k_desc_to_u8<<<(unsigned)ceil_div_ll(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(desc, n, out);
    PYSIFT_LAUNCH_CHECK("k_desc_to_u8");
    return PYSIFT_OK;
}

}  // extern "C"
