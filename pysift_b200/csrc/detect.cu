// detect.cu -- SIFT detection + description on one device-resident image.
//
// Pipeline (all launches on the caller's stream, no host synchronisation,
// capturable into a CUDA graph):
//   k_histogram          256-bin histogram + entropy threshold (pysift/core.py:1129-1148)
//   k_prefilter_cols, k_prefilter_rows, k_zoom_interp
//                        2x cubic B-spline upsample (pysift/core.py:1270-1275)
//   k_u8_to_f32          base image when not upsampled (pysift/core.py:1248-1261)
//   k_blur<R>            fused H+V separable blur per level (pysift/core.py:475-608,
//                        1288-1343); the first blur of octave o>0 reads the previous
//                        octave's level S with stride 2 and also stores level 0
//   k_extrema_mask       26-neighbour test on DoG computed on the fly from the Gaussian
//                        levels (pysift/core.py:176-217); one bit per voxel + per-row
//                        integer counts
//   k_rowscan, k_scatter deterministic compaction in (s, r, c) order, cap per octave
//   k_refine             Taylor refinement + contrast + edge (pysift/core.py:343-463)
//   k_refine_compact     valid keypoints in candidate order
//   k_retry_decide       starvation retry at half threshold (pysift/core.py:2066-2071)
//   k_cap                top-cap by response, stable (pysift/core.py:2078-2080)
//   k_orientation        36-bin histogram, peaks (pysift/core.py:228-333)
//   k_expand             orientation expansion + (x, y) sort keys (pysift/core.py:1592-1598)
//   k_br_scan/scatter/rank  rank of each key = output row (pysift/core.py:2128-2134),
//                        and the output-limit order, exactly, through buckets
//   k_descriptor         4x4x8 descriptor (+DSP) + L2/clip/L2 + RootSIFT, written at its
//                        output row (pysift/core.py:693-997, 1870-1873)
#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <atomic>
#include <mutex>

#include "common.cuh"
#include "sift_math.cuh"

namespace pysift {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

// ---------------------------------------------------------------------------
// Device control block (one per run, inside the workspace).
// ---------------------------------------------------------------------------
struct Ctrl {
    double ct;
    float thr[2];
    unsigned int hist[256];
    unsigned int blocks_done;
    int found[PYSIFT_MAX_OCTAVES];
    int ncand[PYSIFT_MAX_OCTAVES];
    int nref[PYSIFT_MAX_OCTAVES];
    int retried;
    int n_total_ref;
    int n_kept;
    int capped;
    int n_oriented;
    int overflow_octs;
    int desc_next;  // next oriented entry a descriptor block takes
    int ori_next;   // next kept keypoint an orientation block takes
};

// buckets of the exact rank kernels (k_br_*)
constexpr int BR_NB = 4096;

struct OctView {
    const float* lev[PYSIFT_MAX_LEVELS];
    int H, W, pitch;
};

// ---------------------------------------------------------------------------
// Workspace layout.
// ---------------------------------------------------------------------------
struct Layout {
    int n_oct, L, S;
    bool doubled;
    int H0, W0, pitch0;  // octave-0 / base image
    int H[PYSIFT_MAX_OCTAVES], W[PYSIFT_MAX_OCTAVES], pitch[PYSIFT_MAX_OCTAVES], wpr[PYSIFT_MAX_OCTAVES];
    size_t off_pyr[PYSIFT_MAX_OCTAVES], off_pyr_r[PYSIFT_MAX_OCTAVES];
    size_t off_mask[PYSIFT_MAX_OCTAVES], off_rowcnt[PYSIFT_MAX_OCTAVES], off_rowoff[PYSIFT_MAX_OCTAVES];
    size_t off_ctrl, off_coef, off_base;
    size_t off_cand, off_rv_valid, off_rv_ri, off_rv_ci, off_rv_si, off_rv_resp;
    size_t off_rf_ri, off_rf_ci, off_rf_si, off_rf_resp;
    size_t off_kp_o, off_kp_si, off_kp_ri, off_kp_ci, off_kp_resp, off_kp_tb;
    size_t off_ang, off_angcnt, off_ent_kp, off_ent_slot, off_keys, off_rank, off_row_resp, off_lrank;
    size_t off_bkt, off_members;  // bucket ranks: [2 orders][cnt | off | cursor][BR_NB], [2][4 kc] members
    size_t off_xblk;              // k_expand block counts
    size_t rowcnt_bytes_total;
    size_t off_rowcnt_base;
    size_t total;
};

static int validate_cfg(const pysift_detect_config* c) {
    PYSIFT_CHECK_ARG(c != nullptr, "config is NULL");
    PYSIFT_CHECK_ARG(c->n_octaves >= 1 && c->n_octaves <= PYSIFT_MAX_OCTAVES, "n_octaves %d outside 1..%d",
                     c->n_octaves, PYSIFT_MAX_OCTAVES);
    PYSIFT_CHECK_ARG(c->n_scales >= 1 && c->n_scales + 3 <= PYSIFT_MAX_LEVELS, "n_scales %d outside 1..%d",
                     c->n_scales, PYSIFT_MAX_LEVELS - 3);
    PYSIFT_CHECK_ARG(c->max_cands_per_octave >= 1 && c->max_cands_per_octave <= (1 << 22),
                     "max_cands_per_octave %d out of range", c->max_cands_per_octave);
    PYSIFT_CHECK_ARG(c->keypoint_cap >= 1 && c->keypoint_cap <= (1 << 20), "keypoint_cap %d out of range",
                     c->keypoint_cap);
    PYSIFT_CHECK_ARG(c->border >= 1 && c->border < 64, "border %d out of range", c->border);
    PYSIFT_CHECK_ARG(c->output_limit >= 0, "output_limit %d is negative", c->output_limit);
    PYSIFT_CHECK_ARG(!c->dsp || (c->n_dsp >= 1 && c->n_dsp <= 8), "n_dsp %d out of range", c->n_dsp);
    for (int i = 0; i < 2 + c->n_scales + 2; ++i)
        PYSIFT_CHECK_ARG(c->blur_radius[i] >= 0 && c->blur_radius[i] <= PYSIFT_MAX_RADIUS,
                         "blur radius %d outside 0..%d", c->blur_radius[i], PYSIFT_MAX_RADIUS);
    for (int s = 1; s <= c->n_scales; ++s) {
        PYSIFT_CHECK_ARG(c->desc_ph[s] >= 1.0f && c->desc_ph[s] <= 200.0f, "desc_ph[%d] out of range", s);
        PYSIFT_CHECK_ARG(c->ori_sigma[s] > 0.0f && c->ori_sigma[s] < 64.0f, "ori_sigma[%d] out of range", s);
    }
    return PYSIFT_OK;
}

static Layout make_layout(const pysift_detect_config* c, int H, int W) {
    Layout l;
    memset(&l, 0, sizeof(l));
    l.n_oct = c->n_octaves;
    l.S = c->n_scales;
    l.L = c->n_scales + 3;
    l.doubled = c->double_image && ((int64_t)H * W < c->double_px_cap);
    l.H0 = l.doubled ? 2 * H : H;
    l.W0 = l.doubled ? 2 * W : W;
    int h = l.H0, w = l.W0;
    for (int o = 0; o < l.n_oct; ++o) {
        l.H[o] = h;
        l.W[o] = w;
        l.pitch[o] = (int)align_up((size_t)w, 32);
        l.wpr[o] = ceil_div(w, 32);
        h = (h + 1) / 2;
        w = (w + 1) / 2;
    }
    l.pitch0 = l.pitch[0];
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t r = off;
        off = align_up(off + bytes, 256);
        return r;
    };
    const size_t cap = (size_t)c->max_cands_per_octave;
    const size_t kc = (size_t)c->keypoint_cap;
    l.off_ctrl = take(sizeof(Ctrl));
    // row counts of all octaves are contiguous so one memset clears them
    l.off_rowcnt_base = off;
    size_t rc = 0;
    for (int o = 0; o < l.n_oct; ++o) rc += (size_t)l.S * l.H[o];
    size_t start = take(rc * sizeof(int));
    l.rowcnt_bytes_total = rc * sizeof(int);
    size_t acc = start;
    for (int o = 0; o < l.n_oct; ++o) {
        l.off_rowcnt[o] = acc;
        acc += (size_t)l.S * l.H[o] * sizeof(int);
    }
    for (int o = 0; o < l.n_oct; ++o) l.off_rowoff[o] = take((size_t)l.S * l.H[o] * sizeof(int));
    for (int o = 0; o < l.n_oct; ++o) l.off_mask[o] = take((size_t)l.S * l.H[o] * l.wpr[o] * sizeof(uint32_t));
    l.off_cand = take(cap * l.n_oct * sizeof(int4));
    l.off_rv_valid = take(cap * l.n_oct * sizeof(int));
    l.off_rv_ri = take(cap * l.n_oct * sizeof(float));
    l.off_rv_ci = take(cap * l.n_oct * sizeof(float));
    l.off_rv_si = take(cap * l.n_oct * sizeof(int));
    l.off_rv_resp = take(cap * l.n_oct * sizeof(float));
    l.off_rf_ri = take(cap * l.n_oct * sizeof(float));
    l.off_rf_ci = take(cap * l.n_oct * sizeof(float));
    l.off_rf_si = take(cap * l.n_oct * sizeof(int));
    l.off_rf_resp = take(cap * l.n_oct * sizeof(float));
    l.off_kp_o = take(kc * sizeof(int));
    l.off_kp_si = take(kc * sizeof(int));
    l.off_kp_ri = take(kc * sizeof(float));
    l.off_kp_ci = take(kc * sizeof(float));
    l.off_kp_resp = take(kc * sizeof(float));
    l.off_kp_tb = take(kc * sizeof(uint32_t));
    l.off_ang = take(kc * 4 * sizeof(float));
    l.off_angcnt = take(kc * sizeof(int));
    l.off_ent_kp = take(kc * 4 * sizeof(int));
    l.off_ent_slot = take(kc * 4 * sizeof(int));
    l.off_keys = take(kc * 4 * sizeof(uint4));
    l.off_rank = take(kc * 4 * sizeof(int));
    l.off_row_resp = take(kc * 4 * sizeof(float));
    l.off_lrank = take(kc * 4 * sizeof(int));
    l.off_bkt = take(2 * 3 * BR_NB * sizeof(int));
    l.off_members = take(2 * kc * 4 * sizeof(int));
    l.off_xblk = take(((size_t)kc / 2048 + 2) * sizeof(int));
    if (l.doubled) l.off_coef = take((size_t)H * W * sizeof(double));
    l.off_base = take((size_t)l.H0 * l.pitch0 * sizeof(float));
    for (int o = 0; o < l.n_oct; ++o) l.off_pyr[o] = take((size_t)l.L * l.H[o] * l.pitch[o] * sizeof(float));
    for (int o = 0; o < l.n_oct; ++o) {
        if (c->fp16_pyramid && o >= 2)
            l.off_pyr_r[o] = take((size_t)l.L * l.H[o] * l.pitch[o] * sizeof(float));
        else
            l.off_pyr_r[o] = l.off_pyr[o];
    }
    l.total = off;
    return l;
}

// ---------------------------------------------------------------------------
// A1: histogram + entropy threshold.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_histogram(const uint8_t* __restrict__ img, int H, int W, long long pitch,
                                                   Ctrl* ctrl, double base, int S) {
    __shared__ unsigned int sh[8][256];
    __shared__ double terms[256];
    __shared__ int is_last;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < 8 * 256; i += 256) (&sh[0][0])[i] = 0u;
    __syncthreads();
    // a warp per row; 16-byte loads when every row starts on a 16-byte
    // boundary, else byte loads in batches of 8, all in flight before the
    // shared-memory counts
    const bool vec = ((reinterpret_cast<uintptr_t>(img) | (uintptr_t)pitch) & 15) == 0;
    const int nw = W >> 4;
    for (int r = blockIdx.x * 8 + warp; r < H; r += gridDim.x * 8) {
        const uint8_t* row = img + (long long)r * pitch;
        int c0 = 0;
        if (vec) {
            for (int q0 = 0; q0 < nw; q0 += 64) {
                uint4 u[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int q = q0 + lane + 32 * k;
                    u[k] = q < nw ? reinterpret_cast<const uint4*>(row)[q] : make_uint4(0u, 0u, 0u, 0u);
                }
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    if (q0 + lane + 32 * k >= nw) continue;
                    const uint32_t w4[4] = {u[k].x, u[k].y, u[k].z, u[k].w};
#pragma unroll
                    for (int e = 0; e < 4; ++e)
#pragma unroll
                        for (int sh8 = 0; sh8 < 32; sh8 += 8) atomicAdd(&sh[warp][(w4[e] >> sh8) & 255u], 1u);
                }
            }
            c0 = nw << 4;
        }
        for (int cb = c0; cb < W; cb += 32 * 8) {
            uint8_t u[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int c = cb + lane + 32 * k;
                u[k] = c < W ? row[c] : 0;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (cb + lane + 32 * k < W) atomicAdd(&sh[warp][u[k]], 1u);
        }
    }
    __syncthreads();
    unsigned int mine = 0;
    for (int w = 0; w < 8; ++w) mine += sh[w][tid];
    if (mine) atomicAdd(&ctrl->hist[tid], mine);
    __threadfence();
    __syncthreads();
    if (tid == 0) is_last = (atomicAdd(&ctrl->blocks_done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const double n = (double)H * (double)W;
    unsigned int h = atomicAdd(&ctrl->hist[tid], 0u);
    double t = 0.0;
    if (h) {
        double p = (double)h / n;
        t = p * sm::log2d_(p);
    }
    terms[tid] = t;
    sh[0][tid] = h;
    __syncthreads();
    if (tid == 0) {
        // ascending bins, one double sum; an empty bin holds +0.0, which
        // leaves a sum that started at +0.0 unchanged, so every term is added
        // and the loads run ahead of the chain
        double ent = 0.0;
#pragma unroll 32
        for (int b = 0; b < 256; ++b) ent = ent + terms[b];
        ent = -ent;
        double scale = 0.8 + ent / 40.0;
        if (scale > 1.0) scale = 1.0;
        double ct = base * scale;
        ctrl->ct = ct;
        ctrl->thr[0] = (float)(ct / (double)S);
        ctrl->thr[1] = (float)((ct * 0.5) / (double)S);
    }
}

// ---------------------------------------------------------------------------
// A2/A3: base image.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float u8_to_unit(uint8_t u, int fp16) {
    float f = (float)u / 255.0f;
    return fp16 ? round_half(f) : f;
}

__global__ void k_u8_to_f32(const uint8_t* __restrict__ img, int H, int W, long long pitch, int fp16,
                            float* __restrict__ out, int out_pitch) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int r = blockIdx.y;
    if (c < W) out[(long long)r * out_pitch + c] = u8_to_unit(img[(long long)r * pitch + c], fp16);
}

// B-spline direct transform (scipy.ndimage.spline_filter, order 3, mirror
// boundary) as a symmetric FIR: on the mirror-extended line the recursive
// prefilter's impulse response is h[k] = (-6 z / (1 - z^2)) z^|k| with
// z = sqrt(3) - 2, truncated at |k| <= SPL_K (|z|^31 < 2e-18).  Taps run
// k = -SPL_K..SPL_K with one fma each.  Columns (axis 0) are filtered first,
// then rows, as scipy does.
constexpr int SPL_K = 30;
constexpr int SPL_TAPS = 2 * SPL_K + 1;

// Taps computed once on the host with the same operation sequence as the
// oracle (IEEE double, no contraction) and passed by value, so that fully
// unrolled loops read them as constant-bank operands.
struct SplTaps {
    double h[SPL_TAPS];
};

static const SplTaps& spline_taps() {
    static const SplTaps taps = [] {
        SplTaps t;
        const double z = sqrt(3.0) - 2.0;
        const double c0 = -6.0 * z / (1.0 - z * z);
        for (int k = -SPL_K; k <= SPL_K; ++k) {
            const int a = k < 0 ? -k : k;
            double zk = 1.0;
            for (int i = 0; i < a; ++i) zk = zk * z;
            t.h[k + SPL_K] = c0 * zk;
        }
        return t;
    }();
    return taps;
}

__device__ __forceinline__ long long mirror_index(long long idx, long long len) {
    if (len <= 1) return 0;
    long long s2 = 2 * len - 2;
    if (idx < 0) {
        idx = s2 * (long long)(-idx / s2) + idx;
        idx = idx <= 1 - len ? idx + s2 : -idx;
    } else if (idx >= len) {
        idx -= s2 * (long long)(idx / s2);
        if (idx >= len) idx = s2 - idx;
    }
    return idx;
}

constexpr int PC_TW = 32, PC_RB = 8, PC_TH = 8 * PC_RB;

// Column FIR straight from the uint8 image: coef[r][x] = sum_k h[k] u[mirror(r+k)][x].
// Each thread produces PC_RB consecutive rows of one column, streaming the
// input window through registers (taps in ascending k for every output).
__global__ void __launch_bounds__(256) k_prefilter_cols(const uint8_t* __restrict__ img, int H, int W,
                                                        long long pitch, int fp16, double* __restrict__ coef,
                                                        const SplTaps taps) {
    __shared__ double tile[(PC_TH + 2 * SPL_K) * PC_TW];
    const int x0 = blockIdx.x * PC_TW, r0 = blockIdx.y * PC_TH;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x = x0 + tx;
    {
        // every load of the window issued before the first conversion
        constexpr int NL = (PC_TH + 2 * SPL_K + 7) / 8;
        uint8_t u[NL];
#pragma unroll
        for (int q = 0; q < NL; ++q) {
            const int rr = ty + 8 * q;
            u[q] = (x < W && rr < PC_TH + 2 * SPL_K) ? img[mirror_index(r0 - SPL_K + rr, H) * pitch + x] : 0;
        }
#pragma unroll
        for (int q = 0; q < NL; ++q) {
            const int rr = ty + 8 * q;
            if (rr < PC_TH + 2 * SPL_K) tile[rr * PC_TW + tx] = x < W ? (double)u8_to_unit(u[q], fp16) : 0.0;
        }
    }
    __syncthreads();
    if (x >= W) return;
    const int y0 = ty * PC_RB;
    double acc[PC_RB];
#pragma unroll
    for (int j = 0; j < PC_RB; ++j) acc[j] = 0.0;
#pragma unroll
    for (int m = 0; m < PC_RB + 2 * SPL_K; ++m) {
        const double t = tile[(y0 + m) * PC_TW + tx];
#pragma unroll
        for (int j = 0; j < PC_RB; ++j) {
            const int k = m - j;
            if (k >= 0 && k < SPL_TAPS) acc[j] = fma(taps.h[k], t, acc[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < PC_RB; ++j) {
        const int r = r0 + y0 + j;
        if (r < H) coef[(long long)r * W + x] = acc[j];
    }
}

// Output-coordinate setup for one axis of scipy's zoom (grid_mode=False,
// mode='constant'): input coordinate k*(in-1)/(out-1), cubic B-spline
// weights, mirror-mapped support; false outside [0, in-1] (cval 0).
__device__ __forceinline__ bool zoom_axis(long long k, long long in_len, long long out_len, long long idx[4],
                                          double w[4]) {
    double zoom = (out_len > 1) ? (double)(in_len - 1) / (double)(out_len - 1) : 1.0;
    double cc = (double)k * zoom;
    if (cc < 0.0 || cc > (double)(in_len - 1)) return false;
    double fl = floor(cc);
    long long start = (long long)fl - 1;
    double y = cc - fl;
    double z = 1.0 - y;
    w[0] = z * z * z / 6.0;
    w[1] = (y * y * (y - 2.0) * 3.0 + 4.0) / 6.0;
    double y1 = 1.0 - y;
    w[2] = (y1 * y1 * (y1 - 2.0) * 3.0 + 4.0) / 6.0;
    w[3] = 1.0 - w[0] - w[1] - w[2];
    for (int h = 0; h < 4; ++h) idx[h] = mirror_index(start + h, in_len);
    return true;
}

// Row FIR in place: coef[r][x] <- sum_k h[k] coef[r][mirror(x-SPL_K+k)], one
// block per row, the row processed in chunks of PR_CW outputs left to right.
// A chunk's window is read before any of its outputs is written; its left
// halo, which the previous chunk has overwritten, comes from a carry of the
// previous chunk's last SPL_K inputs.  Mirrored positions past the right
// end fall at or after the chunk start minus SPL_K once the row spans more
// than one chunk, so the carry and the unwritten part of the row hold every
// input.  The window sits in shared memory with one padding double per 8 so
// that lanes reading 8-output strips hit distinct banks.
constexpr int PR_NT = 256, PR_CW = 2048;
constexpr int PR_EXT = PR_CW + 2 * SPL_K;
__device__ __forceinline__ int pr_phys(int e) { return e + (e >> 3); }

__global__ void __launch_bounds__(PR_NT) k_prefilter_rows(double* __restrict__ coef, int W, const SplTaps taps) {
    // a strip that ends past the chunk reads up to 7 positions beyond the
    // window (values that feed no stored output), so the array covers them
    __shared__ double ext[PR_EXT + 7 + (PR_EXT + 7) / 8 + 1];
    __shared__ double carry[SPL_K];
    double* row = coef + (long long)blockIdx.x * W;
    for (int x0 = 0; x0 < W; x0 += PR_CW) {
        const int len = min(PR_CW, W - x0);
        for (int e = threadIdx.x; e < len + 2 * SPL_K; e += PR_NT) {
            const int m = (int)mirror_index((long long)x0 - SPL_K + e, W);
            if (m >= x0) {
                const unsigned d = (unsigned)__cvta_generic_to_shared(&ext[pr_phys(e)]);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(row + m) : "memory");
            } else {
                ext[pr_phys(e)] = carry[m - (x0 - SPL_K)];
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        if (x0 + PR_CW < W)
            for (int i = threadIdx.x; i < SPL_K; i += PR_NT) carry[i] = ext[pr_phys(PR_CW + i)];
        for (int b = threadIdx.x * 8; b < len; b += PR_NT * 8) {
            double acc[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] = 0.0;
#pragma unroll
            for (int m = 0; m < 8 + 2 * SPL_K; ++m) {
                const double t = ext[pr_phys(b + m)];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int k = m - j;
                    if (k >= 0 && k < SPL_TAPS) acc[j] = fma(taps.h[k], t, acc[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (b + j < len) row[x0 + b + j] = acc[j];
        }
        __syncthreads();
    }
}

// 4x4 cubic interpolation of the prefiltered coefficients on the 2x output
// grid, t = sum_a sum_b (c[a][b] * wy_a) * wx_b in scipy's order, rounded to
// float32.  On the 2x grid the output columns 2k-1 and 2k interpolate the
// same 4 input columns (their input coordinates share the floor k-1), and
// likewise the output rows 2k-1 and 2k.  A tile covers output rows
// oy0-1 .. oy0+30 and columns ox0-1 .. ox0+62, so it splits into 16 x 32
// such 2x2 quads; each thread takes 2 quads, loads the quad's 16
// coefficients once and forms each c * wy_a once per row for both columns.
// A quad whose rows or columns do not share their support (mirrored image
// edges) reads each output's coefficients separately; either way each
// output is the same sequence of products and sums.  The tile touches at
// most 20 input rows and 36 input columns (zoom factor below 1/2).
constexpr int ZI_TW = 64, ZI_TH = 32;
constexpr int ZI_CR = 20, ZI_CC = 36;

__device__ __forceinline__ double zoom_term_sum(const double (*win)[ZI_CC], const int* ry, const double* wy,
                                                const int* cx, const double* wx) {
    double t = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            double coeff = win[ry[a]][cx[b]];
            coeff *= wy[a];
            coeff *= wx[b];
            t += coeff;
        }
    return t;
}

__global__ void __launch_bounds__(256) k_zoom_interp(const double* __restrict__ coef, int H, int W, int fp16,
                                                     float* __restrict__ out, int out_pitch) {
    __shared__ int rvalid[ZI_TH], ridx[4][ZI_TH];
    __shared__ double rw[4][ZI_TH];
    __shared__ int cvalid[ZI_TW], cidx[4][ZI_TW];
    __shared__ double cw[4][ZI_TW];
    __shared__ int s_lo[2], s_hi[2];
    __shared__ double win[ZI_CR][ZI_CC];
    const int OH = 2 * H, OW = 2 * W;
    const int ox0 = blockIdx.x * ZI_TW, oy0 = blockIdx.y * ZI_TH;
    const int tid = threadIdx.x;
    if (tid < 2) {
        s_lo[tid] = 0x7fffffff;
        s_hi[tid] = -1;
    }
    __syncthreads();
    if (tid < ZI_TH) {
        const int r = oy0 - 1 + tid;
        long long idx[4];
        double w[4];
        bool v = (r >= 0 && r < OH) && zoom_axis(r, H, OH, idx, w);
        rvalid[tid] = v;
        if (v) {
            int lo = 0x7fffffff, hi = -1;
            for (int q = 0; q < 4; ++q) {
                ridx[q][tid] = (int)idx[q];
                rw[q][tid] = w[q];
                lo = min(lo, (int)idx[q]);
                hi = max(hi, (int)idx[q]);
            }
            atomicMin(&s_lo[0], lo);
            atomicMax(&s_hi[0], hi);
        }
    } else if (tid >= 32 && tid < 32 + ZI_TW) {
        const int t = tid - 32;
        const int x = ox0 - 1 + t;
        long long idx[4];
        double w[4];
        bool v = (x >= 0 && x < OW) && zoom_axis(x, W, OW, idx, w);
        cvalid[t] = v;
        if (v) {
            int lo = 0x7fffffff, hi = -1;
            for (int q = 0; q < 4; ++q) {
                cidx[q][t] = (int)idx[q];
                cw[q][t] = w[q];
                lo = min(lo, (int)idx[q]);
                hi = max(hi, (int)idx[q]);
            }
            atomicMin(&s_lo[1], lo);
            atomicMax(&s_hi[1], hi);
        }
    }
    __syncthreads();
    const int ylo = s_lo[0], yhi = s_hi[0], xlo = s_lo[1], xhi = s_hi[1];
    const bool any = (yhi >= 0 && xhi >= 0);
    const int ny = any ? yhi - ylo + 1 : 0, nx = any ? xhi - xlo + 1 : 0;
    const bool fits = ny <= ZI_CR && nx <= ZI_CC;
    const int warp = tid >> 5, lane = tid & 31;
    if (any && fits) {
        for (int yy = warp; yy < ny; yy += 8) {
            const double* src = coef + (long long)(ylo + yy) * W + xlo;
            for (int xx = lane; xx < nx; xx += 32) {
                const unsigned d = (unsigned)__cvta_generic_to_shared(&win[yy][xx]);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src + xx) : "memory");
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncthreads();
    // this lane's column pair
    const int ta = 2 * lane, tb = ta + 1;
    const int xa = ox0 - 1 + ta, xb = xa + 1;
    const bool cva = cvalid[ta], cvb = cvalid[tb];
    int cxa[4], cxb[4];
    double wxa[4], wxb[4];
    bool csame = cva && cvb;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        cxa[q] = cva ? cidx[q][ta] - xlo : 0;
        cxb[q] = cvb ? cidx[q][tb] - xlo : 0;
        wxa[q] = cva ? cw[q][ta] : 0.0;
        wxb[q] = cvb ? cw[q][tb] : 0.0;
        csame = csame && cxa[q] == cxb[q];
    }
    const float nan = __int_as_float(0x7fc00000);  // unreachable by construction; visible in parity tests
    for (int pr = warp; pr < ZI_TH / 2; pr += 8) {
        const int ua = 2 * pr, ub = ua + 1;
        const int ra = oy0 - 1 + ua, rb = ra + 1;
        const bool rva = rvalid[ua], rvb = rvalid[ub];
        int rya[4], ryb[4];
        double wya[4], wyb[4];
        bool rsame = rva && rvb;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            rya[q] = rva ? ridx[q][ua] - ylo : 0;
            ryb[q] = rvb ? ridx[q][ub] - ylo : 0;
            wya[q] = rva ? rw[q][ua] : 0.0;
            wyb[q] = rvb ? rw[q][ub] : 0.0;
            rsame = rsame && rya[q] == ryb[q];
        }
        double t00 = 0.0, t01 = 0.0, t10 = 0.0, t11 = 0.0;
        if (fits) {
            if (rsame && csame) {
                double c[4][4];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) c[a][b] = win[rya[a]][cxa[b]];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const double pa = c[a][b] * wya[a];
                        const double pb = c[a][b] * wyb[a];
                        t00 += pa * wxa[b];
                        t01 += pa * wxb[b];
                        t10 += pb * wxa[b];
                        t11 += pb * wxb[b];
                    }
            } else {
                if (rva && cva) t00 = zoom_term_sum(win, rya, wya, cxa, wxa);
                if (rva && cvb) t01 = zoom_term_sum(win, rya, wya, cxb, wxb);
                if (rvb && cva) t10 = zoom_term_sum(win, ryb, wyb, cxa, wxa);
                if (rvb && cvb) t11 = zoom_term_sum(win, ryb, wyb, cxb, wxb);
            }
        }
        const double tq[2][2] = {{t00, t01}, {t10, t11}};
        const bool rv[2] = {rva, rvb}, cv[2] = {cva, cvb};
        const int rr[2] = {ra, rb}, xx[2] = {xa, xb};
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            if (rr[i] < 0 || rr[i] >= OH) continue;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (xx[j] < 0 || xx[j] >= OW) continue;
                float res = 0.0f;
                if (rv[i] && cv[j]) {
                    res = fits ? (float)tq[i][j] : nan;
                    if (fits && fp16) res = round_half(res);
                }
                out[(long long)rr[i] * out_pitch + xx[j]] = res;
            }
        }
    }
}

static int launch_zoom2x(const uint8_t* gray, int H, int W, long long pitch, int fp16, double* coef, float* out,
                         int out_pitch, cudaStream_t st) {
    const SplTaps& taps = spline_taps();
    k_prefilter_cols<<<dim3(ceil_div(W, PC_TW), ceil_div(H, PC_TH)), 256, 0, st>>>(gray, H, W, pitch, fp16, coef,
                                                                                  taps);
    PYSIFT_LAUNCH_CHECK("k_prefilter_cols");
    k_prefilter_rows<<<H, PR_NT, 0, st>>>(coef, W, taps);
    PYSIFT_LAUNCH_CHECK("k_prefilter_rows");
    k_zoom_interp<<<dim3(ceil_div(2 * W + 1, ZI_TW), ceil_div(2 * H + 1, ZI_TH)), 256, 0, st>>>(coef, H, W, fp16,
                                                                                               out, out_pitch);
    PYSIFT_LAUNCH_CHECK("k_zoom_interp");
    return PYSIFT_OK;
}

// ---------------------------------------------------------------------------
// A4/A5: fused separable blur.
// ---------------------------------------------------------------------------
constexpr int BLUR_PAIR_MAX_R = 16;  // radii with a register-blocked kernel

struct BlurArgs {
    const float* in;
    long long in_pitch;
    int step;  // 1, or 2 when reading level S of the previous octave
    float* out;
    float* out_r;  // binary16-rounded copy (fp16 mode), else null
    float* copy0;  // stores the (subsampled) input tile interior, else null
    float* copy0_r;
    int out_pitch;
    int H, W;
    float w[PYSIFT_MAX_TAPS];
    unsigned long long w2[2 * BLUR_PAIR_MAX_R + 1];  // (w[k], w[k]) packed, radii up to BLUR_PAIR_MAX_R
};

// Half-sample-symmetric reflection into [0, n) (period 2n), as the
// reference's reflect() (pysift/core.py:477-483), without integer division.
__device__ __forceinline__ int reflect_idx(int i, int n) {
    while (i < 0 || i >= n) {
        if (i < 0) i = -i - 1;
        if (i >= n) i = 2 * n - 1 - i;
    }
    return i;
}

constexpr int BLUR_TW = 64, BLUR_TH = 32, BLUR_NT = 256;

// Loads input rows [r0-R, r0+TH+R) and columns [c0-RA, c0+TW+RA) (RA >= R,
// a multiple of 4) into tile[ROWS][TWP] with reflection.  Tiles whose
// window lies inside the image, read with stride 1 from a 16-byte aligned
// base and pitch, use float4 loads.
__device__ __forceinline__ void blur_load_tile(const BlurArgs& a, float* tile, int R, int RA, int TWP, int ROWS,
                                               int r0, int c0) {
    const bool interior = a.step == 1 && r0 - R >= 0 && r0 + BLUR_TH + R <= a.H && c0 - RA >= 0 &&
                          c0 + BLUR_TW + RA <= a.W && ((a.in_pitch & 3) == 0) &&
                          ((reinterpret_cast<uintptr_t>(a.in) & 15) == 0);
    if (interior) {
        const int q4 = TWP / 4;
        for (int i = threadIdx.x; i < ROWS * q4; i += BLUR_NT) {
            const int rr = i / q4, q = i - rr * q4;
            const float4 v = *reinterpret_cast<const float4*>(a.in + (long long)(r0 - R + rr) * a.in_pitch + c0 - RA +
                                                              4 * q);
            *reinterpret_cast<float4*>(tile + rr * TWP + 4 * q) = v;
        }
        return;
    }
    for (int i = threadIdx.x; i < ROWS * TWP; i += BLUR_NT) {
        int rr = i / TWP, cc = i - rr * TWP;
        int gr = reflect_idx(r0 - R + rr, a.H), gc = reflect_idx(c0 - RA + cc, a.W);
        float v = a.in[(long long)gr * a.step * a.in_pitch + (long long)gc * a.step];
        tile[i] = v;
        if (a.copy0 && rr >= R && rr < R + BLUR_TH && cc >= RA && cc < RA + BLUR_TW) {
            int orow = r0 + rr - R, ocol = c0 + cc - RA;
            if (orow < a.H && ocol < a.W) {
                a.copy0[(long long)orow * a.out_pitch + ocol] = v;
                if (a.copy0_r) a.copy0_r[(long long)orow * a.out_pitch + ocol] = round_half(v);
            }
        }
    }
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

// Packed single-precision pairs: fma.rn.f32x2 is an IEEE fused multiply-add
// with round-to-nearest on each half, the same result as fmaf per element.
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float lo2(unsigned long long v) { return __uint_as_float((unsigned)(v & 0xffffffffull)); }
__device__ __forceinline__ float hi2(unsigned long long v) { return __uint_as_float((unsigned)(v >> 32)); }

// Tile geometry of k_blur<R, TH>: input rows [r0-R, r0+TH+R) and columns
// [c0-R, c0+TW+R) at a row stride TS = 2 (mod 4) (8-byte aligned rows; lanes
// that own consecutive rows read 8-byte pairs from distinct banks), then the
// row-filtered rows at the stride HS = 66, also 2 (mod 4).
template <int R, int TH>
struct BlurTile {
    static constexpr int ROWS = TH + 2 * R;
    static constexpr int TWR = BLUR_TW + 2 * R;
    static constexpr int TS = (TWR % 4 == 2) ? TWR : TWR + 2;
    static constexpr int HS = BLUR_TW + 2;
    static constexpr size_t bytes = (size_t)(ROWS * TS + ROWS * HS) * sizeof(float);
};

// Row filter of 8 outputs src[0..7] (+R halo each side) of one tile row into
// dst[0..7]: 4 output pairs, one packed fma per pair and tap, taps in
// ascending order.  Pairs at even offsets are loaded as 8-byte words; the
// pairs at odd offsets are formed from their neighbours.
template <int R, typename WF>
__device__ __forceinline__ void blur_row_strip(const float* src, float* dst, const WF& w2) {
    constexpr int NP = 4 + R;
    unsigned long long E[NP], O[NP - 1];
#pragma unroll
    for (int m = 0; m < NP; ++m) E[m] = reinterpret_cast<const unsigned long long*>(src)[m];
#pragma unroll
    for (int m = 0; m < NP - 1; ++m) O[m] = pack2(hi2(E[m]), lo2(E[m + 1]));
    unsigned long long A[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
    for (int k = 0; k <= 2 * R; ++k) {
        const unsigned long long wk = w2(k);
#pragma unroll
        for (int p = 0; p < 4; ++p) A[p] = ffma2((k & 1) ? O[p + (k >> 1)] : E[p + (k >> 1)], wk, A[p]);
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) reinterpret_cast<unsigned long long*>(dst)[p] = A[p];
}

// The source, destination and geometry of one blurred level, as a tile of
// it sees them (the fields of BlurArgs without the weights).
struct TileIO {
    const float* in;
    long long in_pitch;
    int step;
    float* out;
    float* out_r;
    float* copy0;
    float* copy0_r;
    int out_pitch;
    int H, W;
};

// Fused H+V separable blur of one 64 x TH output tile (tile column bx, tile
// row by).  The tile and its reflected halo are filled with cp.async (every
// load in flight at once; reflection computed once per row and once per
// column).  Row pass: a lane per tile row (the rows past the first 32 packed
// densely onto the first warps), 8 outputs per lane.  Column pass: each
// thread filters a pair of adjacent columns over TH / 8 rows.  Both passes
// use packed fma pairs; each output is the same fmaf chain over the taps in
// ascending order.  w2(k) is tap k's weight packed twice.  The caller
// synchronises the block before smem is reused.
template <int R, int TH, typename WF>
__device__ __forceinline__ void blur_tile(const TileIO& a, int bx, int by, float* smem, const WF& w2) {
    using T = BlurTile<R, TH>;
    constexpr int TW = BLUR_TW, ROWS = T::ROWS, TWR = T::TWR, TS = T::TS, HS = T::HS;
    constexpr int RP = TH / 8;  // column-pass rows per thread
    constexpr int CQ = (TWR + 31) / 32;
    static_assert(BLUR_NT / 32 == TW / 8, "one warp per 8-column strip in the row pass");
    static_assert(TH % 8 == 0 && BLUR_NT == (TW / 2) * 8, "one thread per column pair and TH / 8 rows in the column pass");
    float* tile = smem;
    float* hb = smem + ROWS * TS;
    const int c0 = bx * TW, r0 = by * TH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        long long gcs[CQ];
#pragma unroll
        for (int q = 0; q < CQ; ++q) {
            const int cc = lane + 32 * q;
            gcs[q] = (long long)reflect_idx(c0 - R + (cc < TWR ? cc : 0), a.W) * a.step;
        }
        for (int rr = warp; rr < ROWS; rr += BLUR_NT / 32) {
            const float* rowp = a.in + (long long)reflect_idx(r0 - R + rr, a.H) * a.step * a.in_pitch;
#pragma unroll
            for (int q = 0; q < CQ; ++q) {
                const int cc = lane + 32 * q;
                if (cc < TWR) cp_async4(tile + rr * TS + cc, rowp + gcs[q]);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncthreads();
    if (a.copy0) {
        for (int i = threadIdx.x; i < TH * TW; i += BLUR_NT) {
            const int y = i / TW, x = i - y * TW;
            const int orow = r0 + y, ocol = c0 + x;
            if (orow < a.H && ocol < a.W) {
                const float v = tile[(y + R) * TS + x + R];
                a.copy0[(long long)orow * a.out_pitch + ocol] = v;
                if (a.copy0_r) a.copy0_r[(long long)orow * a.out_pitch + ocol] = round_half(v);
            }
        }
    }
    {
        constexpr int NF = ROWS / 32, N2 = ROWS % 32;
#pragma unroll
        for (int round = 0; round < NF; ++round) {
            const int rr = round * 32 + lane;
            blur_row_strip<R>(tile + rr * TS + warp * 8, hb + rr * HS + warp * 8, w2);
        }
        if constexpr (N2 > 0) {
            if (threadIdx.x < N2 * 8) {
                const int rr = NF * 32 + threadIdx.x % N2, x0 = (threadIdx.x / N2) * 8;
                blur_row_strip<R>(tile + rr * TS + x0, hb + rr * HS + x0, w2);
            }
        }
    }
    __syncthreads();
    {
        const int cp = lane, y0 = warp * RP;
        constexpr int NV = RP + 2 * R;
        unsigned long long V[NV];
#pragma unroll
        for (int m = 0; m < NV; ++m) V[m] = reinterpret_cast<const unsigned long long*>(hb + (y0 + m) * HS)[cp];
        unsigned long long A[RP];
#pragma unroll
        for (int j = 0; j < RP; ++j) A[j] = 0ull;
#pragma unroll
        for (int k = 0; k <= 2 * R; ++k) {
            const unsigned long long wk = w2(k);
#pragma unroll
            for (int j = 0; j < RP; ++j) A[j] = ffma2(V[j + k], wk, A[j]);
        }
        const int gc = c0 + 2 * cp;
        const bool vec = gc + 1 < a.W && (a.out_pitch & 1) == 0;
#pragma unroll
        for (int j = 0; j < RP; ++j) {
            const int gr = r0 + y0 + j;
            if (gr >= a.H || gc >= a.W) continue;
            const float v0 = lo2(A[j]), v1 = hi2(A[j]);
            const long long off = (long long)gr * a.out_pitch + gc;
            if (vec) {
                *reinterpret_cast<float2*>(a.out + off) = make_float2(v0, v1);
                if (a.out_r) *reinterpret_cast<float2*>(a.out_r + off) = make_float2(round_half(v0), round_half(v1));
            } else {
                a.out[off] = v0;
                if (a.out_r) a.out_r[off] = round_half(v0);
                if (gc + 1 < a.W) {
                    a.out[off + 1] = v1;
                    if (a.out_r) a.out_r[off + 1] = round_half(v1);
                }
            }
        }
    }
}

// Interior tiles: the window [r0-R, r0+TH+R) x [c0-RA, c0+64+RA) (RA = R
// rounded up to 4) lies inside the level, the source is read with stride 1
// from 16-byte aligned rows and no copy of the input is stored.  Then the
// fill is one 16-byte cp.async per 4 floats, a warp per row, with no
// reflection; the row stride TSF = 4 (mod 8) lets the lane-per-row row pass
// read 16-byte words without bank conflicts; the stores need no bounds
// checks.  Same arithmetic as blur_tile, so the same results.
template <int R>
struct BlurFast {
    static constexpr int RA = (R + 3) / 4 * 4;
    static constexpr int D = RA - R;                          // first needed column of a strip, within its quad
    static constexpr int TWF = BLUR_TW + 2 * RA;              // floats per tile row
    static constexpr int TSF = (TWF % 8 == 4) ? TWF : TWF + 4;  // row stride = 4 (mod 8)
    static constexpr int NQ = (D + 8 + 2 * R + 3) / 4;        // 16-byte words a strip reads
    static_assert(TWF / 4 <= 32, "one warp fills a tile row");
};

template <int R, int TH>
__host__ __device__ constexpr size_t blur_fast_bytes() {
    return (size_t)((TH + 2 * R) * BlurFast<R>::TSF + (TH + 2 * R) * (BLUR_TW + 2)) * sizeof(float);
}

__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ bool blur_tile_is_fast(const TileIO& a, int R, int RA, int TH, int bx, int by) {
    const int c0 = bx * BLUR_TW, r0 = by * TH;
    return a.step == 1 && !a.copy0 && r0 - R >= 0 && r0 + TH + R <= a.H && c0 - RA >= 0 &&
           c0 + BLUR_TW + RA <= a.W && (a.in_pitch & 3) == 0 && (reinterpret_cast<uintptr_t>(a.in) & 15) == 0 &&
           (a.out_pitch & 1) == 0 && (reinterpret_cast<uintptr_t>(a.out) & 7) == 0 &&
           (reinterpret_cast<uintptr_t>(a.out_r) & 7) == 0;
}

// Row filter of one strip from 16-byte words q[0..NQ): output pair p, tap k
// reads floats D + 2p + k and D + 2p + k + 1 of the strip's words.
template <int R, typename WF>
__device__ __forceinline__ void blur_row_strip_q(const float* src, float* dst, const WF& w2) {
    using F = BlurFast<R>;
    constexpr int NF = 4 * F::NQ;
    float v[NF];
#pragma unroll
    for (int i = 0; i < F::NQ; ++i) {
        const float4 t = reinterpret_cast<const float4*>(src)[i];
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
    }
    unsigned long long A[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
    for (int k = 0; k <= 2 * R; ++k) {
        const unsigned long long wk = w2(k);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int e = F::D + 2 * p + k;
            A[p] = ffma2(pack2(v[e], v[e + 1]), wk, A[p]);
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) reinterpret_cast<unsigned long long*>(dst)[p] = A[p];
}

template <int R, int TH, typename WF>
__device__ __forceinline__ void blur_tile_fast(const TileIO& a, int bx, int by, float* smem, const WF& w2) {
    using F = BlurFast<R>;
    constexpr int TW = BLUR_TW, ROWS = TH + 2 * R, TSF = F::TSF, HS = BLUR_TW + 2;
    constexpr int RP = TH / 8;
    float* tile = smem;
    float* hb = smem + ROWS * TSF;
    const int c0 = bx * TW, r0 = by * TH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        const bool act = lane < F::TWF / 4;
        const float* src = a.in + (long long)(r0 - R + warp) * a.in_pitch + (c0 - F::RA) + 4 * lane;
        float* dst = tile + warp * TSF + 4 * lane;
        const long long gstep = 8 * a.in_pitch;
        for (int rr = warp; rr < ROWS; rr += BLUR_NT / 32) {
            if (act) cp_async16(dst, src);
            src += gstep;
            dst += 8 * TSF;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncthreads();
    {
        constexpr int NR = ROWS / 32, N2 = ROWS % 32;
#pragma unroll
        for (int round = 0; round < NR; ++round) {
            const int rr = round * 32 + lane;
            blur_row_strip_q<R>(tile + rr * TSF + warp * 8, hb + rr * HS + warp * 8, w2);
        }
        if constexpr (N2 > 0) {
            if (threadIdx.x < N2 * 8) {
                const int rr = NR * 32 + threadIdx.x % N2, x0 = (threadIdx.x / N2) * 8;
                blur_row_strip_q<R>(tile + rr * TSF + x0, hb + rr * HS + x0, w2);
            }
        }
    }
    __syncthreads();
    {
        const int cp = lane, y0 = warp * RP;
        constexpr int NV = RP + 2 * R;
        unsigned long long V[NV];
#pragma unroll
        for (int m = 0; m < NV; ++m) V[m] = reinterpret_cast<const unsigned long long*>(hb + (y0 + m) * HS)[cp];
        unsigned long long A[RP];
#pragma unroll
        for (int j = 0; j < RP; ++j) A[j] = 0ull;
#pragma unroll
        for (int k = 0; k <= 2 * R; ++k) {
            const unsigned long long wk = w2(k);
#pragma unroll
            for (int j = 0; j < RP; ++j) A[j] = ffma2(V[j + k], wk, A[j]);
        }
        const long long off = (long long)(r0 + y0) * a.out_pitch + c0 + 2 * cp;
        unsigned long long* o = reinterpret_cast<unsigned long long*>(a.out + off);
        const int op2 = a.out_pitch >> 1;
#pragma unroll
        for (int j = 0; j < RP; ++j) o[j * op2] = A[j];
        if (a.out_r) {
            float2* orr = reinterpret_cast<float2*>(a.out_r + off);
#pragma unroll
            for (int j = 0; j < RP; ++j) orr[j * op2] = make_float2(round_half(lo2(A[j])), round_half(hi2(A[j])));
        }
    }
}

template <int R, int TH>
__host__ __device__ constexpr size_t blur_smem_bytes_rt() {
    return BlurTile<R, TH>::bytes > blur_fast_bytes<R, TH>() ? BlurTile<R, TH>::bytes : blur_fast_bytes<R, TH>();
}

template <int R, int TH>
__global__ void __launch_bounds__(BLUR_NT, TH == 40 ? 7 : 1) k_blur(const BlurArgs a) {
    extern __shared__ __align__(16) float smem[];
    const TileIO io{a.in, a.in_pitch, a.step, a.out, a.out_r, a.copy0, a.copy0_r, a.out_pitch, a.H, a.W};
    auto w = [&](int k) { return a.w2[k]; };
    if (blur_tile_is_fast(io, R, BlurFast<R>::RA, TH, blockIdx.x, blockIdx.y))
        blur_tile_fast<R, TH>(io, blockIdx.x, blockIdx.y, smem, w);
    else
        blur_tile<R, TH>(io, blockIdx.x, blockIdx.y, smem, w);
}

// Any radius up to PYSIFT_MAX_RADIUS (no register blocking); radius 0 copies.
__global__ void __launch_bounds__(BLUR_NT) k_blur_generic(const BlurArgs a, int R) {
    const int RA = (R + 3) / 4 * 4;
    const int TWP = BLUR_TW + 2 * RA, ROWS = BLUR_TH + 2 * R;
    extern __shared__ float smem[];
    float* tile = smem + (RA - R);
    float* hb = smem + ROWS * TWP + 4;
    const int c0 = blockIdx.x * BLUR_TW, r0 = blockIdx.y * BLUR_TH;
    blur_load_tile(a, smem, R, RA, TWP, ROWS, r0, c0);
    __syncthreads();
    for (int i = threadIdx.x; i < ROWS * BLUR_TW; i += BLUR_NT) {
        int rr = i / BLUR_TW, x = i - rr * BLUR_TW;
        float acc = 0.0f;
        if (R == 0) acc = tile[rr * TWP + x];
        else
            for (int k = 0; k <= 2 * R; ++k) acc = fmaf(tile[rr * TWP + x + k], a.w[k], acc);
        hb[i] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < BLUR_TH * BLUR_TW; i += BLUR_NT) {
        int y = i / BLUR_TW, x = i - y * BLUR_TW;
        float acc = 0.0f;
        if (R == 0) acc = hb[y * BLUR_TW + x];
        else
            for (int k = 0; k <= 2 * R; ++k) acc = fmaf(hb[(y + k) * BLUR_TW + x], a.w[k], acc);
        int gr = r0 + y, gc = c0 + x;
        if (gr < a.H && gc < a.W) {
            a.out[(long long)gr * a.out_pitch + gc] = acc;
            if (a.out_r) a.out_r[(long long)gr * a.out_pitch + gc] = round_half(acc);
        }
    }
}

static size_t blur_smem_bytes(int R) {
    const int RA = (R + 3) / 4 * 4;
    return (size_t)((BLUR_TH + 2 * R) * (BLUR_TW + 2 * RA) + (BLUR_TH + 2 * R) * BLUR_TW + 4) * sizeof(float);
}

typedef void (*BlurKernel)(const BlurArgs);

static int num_sms();

// Register-blocked blur variants: radius 1..16 x tile height 16, 32, 40.
constexpr int BLUR_NV = 3;
constexpr int BLUR_THS[BLUR_NV] = {16, 32, 40};
struct BlurVariant {
    BlurKernel fn;
    size_t smem;
};
static_assert(BlurTile<16, 40>::bytes <= 48 * 1024 && blur_fast_bytes<16, 40>() <= 48 * 1024,
              "k_blur<R, TH> stays within the default dynamic shared memory");

template <int R>
static BlurVariant blur_variant_r(int v) {
    switch (v) {
        case 0: return {k_blur<R, 16>, blur_smem_bytes_rt<R, 16>()};
        case 1: return {k_blur<R, 32>, blur_smem_bytes_rt<R, 32>()};
        default: return {k_blur<R, 40>, blur_smem_bytes_rt<R, 40>()};
    }
}

static BlurVariant blur_variant(int R, int v) {
    switch (R) {
        case 1: return blur_variant_r<1>(v);
        case 2: return blur_variant_r<2>(v);
        case 3: return blur_variant_r<3>(v);
        case 4: return blur_variant_r<4>(v);
        case 5: return blur_variant_r<5>(v);
        case 6: return blur_variant_r<6>(v);
        case 7: return blur_variant_r<7>(v);
        case 8: return blur_variant_r<8>(v);
        case 9: return blur_variant_r<9>(v);
        case 10: return blur_variant_r<10>(v);
        case 11: return blur_variant_r<11>(v);
        case 12: return blur_variant_r<12>(v);
        case 13: return blur_variant_r<13>(v);
        case 14: return blur_variant_r<14>(v);
        case 15: return blur_variant_r<15>(v);
        case 16: return blur_variant_r<16>(v);
        default: return {nullptr, 0};
    }
}

// Resident CTAs per SM of every variant, queried once per device.
static int blur_occupancy(int R, int v) {
    constexpr int MAXDEV = 64;
    static std::once_flag once[MAXDEV];
    static int occ[MAXDEV][BLUR_PAIR_MAX_R + 1][BLUR_NV];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAXDEV) return 1;
    std::call_once(once[dev], [dev] {
        for (int r = 1; r <= BLUR_PAIR_MAX_R; ++r)
            for (int k = 0; k < BLUR_NV; ++k) {
                const BlurVariant bv = blur_variant(r, k);
                int n = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bv.fn, BLUR_NT, bv.smem) != cudaSuccess) n = 1;
                occ[dev][r][k] = n > 0 ? n : 1;
            }
    });
    return occ[dev][R][v];
}

// pysift_set_blur_tile_rows: a forced variant (testing), -1 = automatic
static std::atomic<int> g_blur_forced{-1};

// pysift_set_blur_tile_table: a measured variant per (radius, level size
// class), -1 = the cost rule below.  Size class: floor(log2(H W)) - 10,
// clamped to 0 .. BLUR_SIZE_CLASSES - 1.
constexpr int BLUR_SIZE_CLASSES = 16;
static std::atomic<int> g_blur_table[BLUR_PAIR_MAX_R + 1][BLUR_SIZE_CLASSES];
static std::once_flag g_blur_table_once;

static int blur_size_class(int H, int W) {
    const long long px = (long long)H * W;
    int lg = 0;
    while (lg < 62 && (2LL << lg) <= px) ++lg;
    return std::max(0, std::min(BLUR_SIZE_CLASSES - 1, lg - 10));
}

static void blur_table_init() {
    std::call_once(g_blur_table_once, [] {
        for (auto& row : g_blur_table)
            for (auto& e : row) e.store(-1, std::memory_order_relaxed);
    });
}

// The tile height: forced, else tuned, else the one with the fewest (rounds
// of resident CTAs) x (tile rows + halo): big levels avoid a short last
// round, small ones a long CTA.
static int blur_pick(int R, int H, int W) {
    const int forced = g_blur_forced.load(std::memory_order_relaxed);
    if (forced >= 0) return forced;
    blur_table_init();
    const int tuned = g_blur_table[R][blur_size_class(H, W)].load(std::memory_order_relaxed);
    if (tuned >= 0) return tuned;
    int best = 1;
    long long best_cost = -1;
    for (int v = 0; v < BLUR_NV; ++v) {
        const long long blocks = (long long)ceil_div(W, BLUR_TW) * ceil_div(H, BLUR_THS[v]);
        const long long slots = (long long)num_sms() * blur_occupancy(R, v);
        const long long rounds = (blocks + slots - 1) / slots;
        const long long cost = rounds * (BLUR_THS[v] + 2 * R);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = v;
        }
    }
    return best;
}

static int ensure_blur_attrs() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        cudaError_t e = cudaFuncSetAttribute(k_blur_generic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)blur_smem_bytes(PYSIFT_MAX_RADIUS));
        if (e != cudaSuccess) err = e;
    });
    if (err != cudaSuccess) {
        set_error("cudaFuncSetAttribute(k_blur_generic): %s", cudaGetErrorString(err));
        return PYSIFT_ERR_CUDA;
    }
    return PYSIFT_OK;
}

static int launch_blur(BlurArgs& a, int R, const float* w, cudaStream_t st) {
    for (int k = 0; k <= 2 * R; ++k) a.w[k] = w[k];
    for (int k = 0; k <= 2 * R && k <= 2 * BLUR_PAIR_MAX_R; ++k) {
        unsigned u = 0;
        memcpy(&u, &w[k], sizeof(u));
        a.w2[k] = ((unsigned long long)u << 32) | u;
    }
    if (R >= 1 && R <= BLUR_PAIR_MAX_R) {
        const int v = blur_pick(R, a.H, a.W);
        const BlurVariant bv = blur_variant(R, v);
        dim3 grid(ceil_div(a.W, BLUR_TW), ceil_div(a.H, BLUR_THS[v]));
        bv.fn<<<grid, BLUR_NT, bv.smem, st>>>(a);
        PYSIFT_LAUNCH_CHECK("k_blur");
    } else {
        dim3 grid(ceil_div(a.W, BLUR_TW), ceil_div(a.H, BLUR_TH));
        int rc = ensure_blur_attrs();
        if (rc) return rc;
        k_blur_generic<<<grid, BLUR_NT, blur_smem_bytes(R), st>>>(a, R);
        PYSIFT_LAUNCH_CHECK("k_blur_generic");
    }
    return PYSIFT_OK;
}

// ---------------------------------------------------------------------------
// A7: extrema bitmask + per-row counts, then deterministic compaction.
// ---------------------------------------------------------------------------
struct ExtArgs {
    OctView oct[PYSIFT_MAX_OCTAVES];
    int n_oct, S, border, thr_idx, retry_mode, cap;
    int blk_off[PYSIFT_MAX_OCTAVES + 1];
    uint32_t* mask[PYSIFT_MAX_OCTAVES];
    int* rowcnt[PYSIFT_MAX_OCTAVES];
    int* rowoff[PYSIFT_MAX_OCTAVES];
    int wpr[PYSIFT_MAX_OCTAVES];
    int4* cand;
};

__device__ __forceinline__ float dog_at(const OctView& v, int s, int r, int c) {
    long long off = (long long)r * v.pitch + c;
    return v.lev[s + 1][off] - v.lev[s][off];
}

__device__ __forceinline__ int find_octave(const int* blk_off, int n_oct, int b) {
    int o = 0;
    while (o + 1 < n_oct && b >= blk_off[o + 1]) ++o;
    return o;
}

// One block = 32 rows x 32 columns of one octave (a warp per 4 rows, a mask
// word per row and scale).  The block stages the DoG levels of its tile and
// a one-pixel halo in shared memory (D_s = G_{s+1} - G_s, computed once per
// position from the NL Gaussian levels, every load of the tile issued before
// the first subtraction), then tests its pixels: |D| > threshold inside the
// border and D >= all 26 neighbours or D <= all 26 neighbours.  Each lane k
// < 4*S of a warp finally writes the mask word (row k / S, scale k % S + 1)
// and adds its population to the row's count.
constexpr int EX_ROWS = 32;
constexpr int EX_SR = EX_ROWS + 2, EX_SW = 34, EX_SC = 35;  // staged rows, columns, padded stride

template <int NL>
__global__ void __launch_bounds__(256) k_extrema_mask(const ExtArgs a, Ctrl* ctrl) {
    constexpr int S = NL - 3, ND = NL - 1;
    constexpr int NQ = (EX_SR * EX_SW + 255) / 256;
    __shared__ float sDm[ND * EX_SR * EX_SC];
    if (a.retry_mode && !ctrl->retried) return;
    auto sD = [&](int s, int rr, int cc) -> float& { return sDm[(s * EX_SR + rr) * EX_SC + cc]; };
    const float thr = ctrl->thr[a.thr_idx];
    const int o = find_octave(a.blk_off, a.n_oct, blockIdx.x);
    const OctView& v = a.oct[o];
    const int wpr = a.wpr[o];
    const int bl = blockIdx.x - a.blk_off[o];
    const int by = bl / wpr, wc = bl - by * wpr;
    const int r0 = by * EX_ROWS, c0 = wc * 32;
    {
        float g[NQ][NL];
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
            const int q = threadIdx.x + 256 * k;
            const int rr = q / EX_SW, cc = q - rr * EX_SW;
            const int r = r0 - 1 + rr, c = c0 - 1 + cc;
            const bool in = q < EX_SR * EX_SW && r >= 0 && r < v.H && c >= 0 && c < v.W;
            const long long off = in ? (long long)r * v.pitch + c : 0;
#pragma unroll
            for (int l = 0; l < NL; ++l) g[k][l] = in ? v.lev[l][off] : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
            const int q = threadIdx.x + 256 * k;
            if (q >= EX_SR * EX_SW) break;
            const int rr = q / EX_SW, cc = q - rr * EX_SW;
#pragma unroll
            for (int s = 0; s < ND; ++s) sD(s, rr, cc) = g[k][s + 1] - g[k][s];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = c0 + lane;
    const int B = a.border;
    unsigned mine = 0;  // the mask word this lane writes
#pragma unroll
    for (int i = 0; i < EX_ROWS / 8; ++i) {
        const int lr = warp + 8 * i, r = r0 + lr;
        const bool inb = (r >= B && r < v.H - B && c >= B && c < v.W - B);
#pragma unroll
        for (int s = 1; s <= S; ++s) {
            bool ext = false;
            if (inb) {
                const float val = sD(s, lr + 1, lane + 1);
                if (fabsf(val) > thr) {
                    bool is_max = true, is_min = true;
#pragma unroll
                    for (int ds = -1; ds <= 1; ++ds)
#pragma unroll
                        for (int dr = 0; dr < 3; ++dr)
#pragma unroll
                            for (int dc = 0; dc < 3; ++dc) {
                                if (ds == 0 && dr == 1 && dc == 1) continue;
                                const float nb = sD(s + ds, lr + dr, lane + dc);
                                is_max = is_max && (val >= nb);
                                is_min = is_min && (val <= nb);
                            }
                    ext = is_max || is_min;
                }
            }
            const unsigned m = __ballot_sync(FULL_MASK, ext);
            if (lane == i * S + (s - 1)) mine = m;
        }
    }
    if (lane < (EX_ROWS / 8) * S) {
        const int i = lane / S, s = lane - i * S + 1;
        const int r = r0 + warp + 8 * i;
        if (r < v.H) {
            a.mask[o][((long long)(s - 1) * v.H + r) * wpr + wc] = mine;
            if (mine) atomicAdd(&a.rowcnt[o][(s - 1) * v.H + r], __popc(mine));
        }
    }
}

typedef void (*ExtremaKernel)(const ExtArgs, Ctrl*);

static ExtremaKernel extrema_kernel(int S) {
    switch (S + 3) {
        case 4: return k_extrema_mask<4>;
        case 5: return k_extrema_mask<5>;
        case 6: return k_extrema_mask<6>;
        case 7: return k_extrema_mask<7>;
        case 8: return k_extrema_mask<8>;
        default: return nullptr;
    }
}
static_assert(PYSIFT_MAX_LEVELS == 8, "extrema_kernel covers n_scales 1..5");

__global__ void __launch_bounds__(1024) k_rowscan(const ExtArgs a, Ctrl* ctrl) {
    if (a.retry_mode && !ctrl->retried) return;
    __shared__ int sh[33];
    const int o = blockIdx.x;
    const int n = a.S * a.oct[o].H;
    const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int beg = threadIdx.x * per;
    int local = 0;
    for (int i = 0; i < per && beg + i < n; ++i) local += a.rowcnt[o][beg + i];
    int total;
    int off = block_excl_scan(local, &total, sh);
    for (int i = 0; i < per && beg + i < n; ++i) {
        int cnt = a.rowcnt[o][beg + i];
        a.rowoff[o][beg + i] = off;
        off += cnt;
    }
    if (threadIdx.x == 0) {
        ctrl->found[o] = total;
        ctrl->ncand[o] = total < a.cap ? total : a.cap;
        if (total > a.cap) atomicAdd(&ctrl->overflow_octs, 1);
    }
}

__global__ void __launch_bounds__(256) k_scatter(const ExtArgs a, Ctrl* ctrl) {
    if (a.retry_mode && !ctrl->retried) return;
    const int o = find_octave(a.blk_off, a.n_oct, blockIdx.x);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int H = a.oct[o].H;
    const int unit = (blockIdx.x - a.blk_off[o]) * 8 + warp;  // (s-1)*H + r
    if (unit >= a.S * H) return;
    if (a.rowcnt[o][unit] == 0) return;
    const int s = unit / H + 1, r = unit - (s - 1) * H;
    const int wpr = a.wpr[o];
    int base = a.rowoff[o][unit];
    const uint32_t* mrow = a.mask[o] + (long long)unit * wpr;
    int4* out = a.cand + (long long)o * a.cap;
    for (int w0 = 0; w0 < wpr; w0 += 32) {
        uint32_t word = (w0 + lane < wpr) ? mrow[w0 + lane] : 0u;
        int tot;
        int pos = base + warp_excl_scan(__popc(word), &tot);
        while (word) {
            int b = __ffs(word) - 1;
            word &= word - 1;
            if (pos < a.cap) out[pos] = make_int4(s, r, (w0 + lane) * 32 + b, 0);
            ++pos;
        }
        base += tot;
    }
}

// ---------------------------------------------------------------------------
// A8: refinement.
// ---------------------------------------------------------------------------
struct RefArgs {
    OctView oct[PYSIFT_MAX_OCTAVES];
    int n_oct, S, border, cap, thr_idx, retry_mode;
    float edge_score;
    const int4* cand;
    int* rv_valid;
    float* rv_ri;
    float* rv_ci;
    int* rv_si;
    float* rv_resp;
    float* rf_ri;
    float* rf_ci;
    int* rf_si;
    float* rf_resp;
};

__global__ void __launch_bounds__(256) k_refine(const RefArgs a, Ctrl* ctrl) {
    if (a.retry_mode && !ctrl->retried) return;
    const float cthr = ctrl->thr[a.thr_idx];
    const long long nslots = (long long)a.n_oct * a.cap;
    for (long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x; slot < nslots;
         slot += (long long)gridDim.x * blockDim.x) {
        const int o = (int)(slot / a.cap);
        const int j = (int)(slot - (long long)o * a.cap);
        if (j >= ctrl->ncand[o]) continue;
        const OctView& v = a.oct[o];
        const int4 cd = a.cand[slot];
        int si = cd.x, row = cd.y, col = cd.z;
        const int H = v.H, W = v.W, S = a.S, B = a.border;
        float ox = 0.0f, oy = 0.0f, os_ = 0.0f;
        bool converged = false;
        for (int iter = 0; iter < 5; ++iter) {
            if (si < 1 || si > S || row < B || row >= H - B || col < B || col >= W - B) break;
            float cval = dog_at(v, si, row, col);
            float cxp = dog_at(v, si, row, col + 1), cxm = dog_at(v, si, row, col - 1);
            float cyp = dog_at(v, si, row + 1, col), cym = dog_at(v, si, row - 1, col);
            float sp = dog_at(v, si + 1, row, col), smn = dog_at(v, si - 1, row, col);
            float dx = (cxp - cxm) * 0.5f;
            float dy = (cyp - cym) * 0.5f;
            float ds = (sp - smn) * 0.5f;
            float dxx = cxp - 2.0f * cval + cxm;
            float dyy = cyp - 2.0f * cval + cym;
            float dss = sp - 2.0f * cval + smn;
            float dxy = (dog_at(v, si, row + 1, col + 1) - dog_at(v, si, row + 1, col - 1) -
                         dog_at(v, si, row - 1, col + 1) + dog_at(v, si, row - 1, col - 1)) *
                        0.25f;
            float dxs = (dog_at(v, si + 1, row, col + 1) - dog_at(v, si + 1, row, col - 1) -
                         dog_at(v, si - 1, row, col + 1) + dog_at(v, si - 1, row, col - 1)) *
                        0.25f;
            float dys = (dog_at(v, si + 1, row + 1, col) - dog_at(v, si + 1, row - 1, col) -
                         dog_at(v, si - 1, row + 1, col) + dog_at(v, si - 1, row - 1, col)) *
                        0.25f;
            float det = dxx * (dyy * dss - dys * dys) - dxy * (dxy * dss - dys * dxs) + dxs * (dxy * dys - dyy * dxs);
            if (fabsf(det) < 1e-12f) break;
            float inv_det = 1.0f / det;
            float p = -dx, q = -dy, rv = -ds;
            ox = (p * (dyy * dss - dys * dys) - dxy * (q * dss - dys * rv) + dxs * (q * dys - dyy * rv)) * inv_det;
            oy = (dxx * (q * dss - dys * rv) - p * (dxy * dss - dys * dxs) + dxs * (dxy * rv - q * dxs)) * inv_det;
            os_ = (dxx * (dyy * rv - q * dys) - dxy * (dxy * rv - q * dxs) + p * (dxy * dys - dyy * dxs)) * inv_det;
            if (fabsf(ox) < 0.5f && fabsf(oy) < 0.5f && fabsf(os_) < 0.5f) {
                converged = true;
                break;
            }
            col += (ox >= 0.0f) ? (int)(ox + 0.5f) : (int)(ox - 0.5f);
            row += (oy >= 0.0f) ? (int)(oy + 0.5f) : (int)(oy - 0.5f);
            si += (os_ >= 0.0f) ? (int)(os_ + 0.5f) : (int)(os_ - 0.5f);
        }
        int valid = 0;
        float response = 0.0f;
        if (converged && !(si < 1 || si > S || row < B || row >= H - B || col < B || col >= W - B)) {
            float cval = dog_at(v, si, row, col);
            float cxp = dog_at(v, si, row, col + 1), cxm = dog_at(v, si, row, col - 1);
            float cyp = dog_at(v, si, row + 1, col), cym = dog_at(v, si, row - 1, col);
            float dx_ = (cxp - cxm) * 0.5f;
            float dy_ = (cyp - cym) * 0.5f;
            float ds_ = (dog_at(v, si + 1, row, col) - dog_at(v, si - 1, row, col)) * 0.5f;
            response = fabsf(cval + 0.5f * (dx_ * ox + dy_ * oy + ds_ * os_));
            if (response >= cthr) {
                float dxx = cxp - 2.0f * cval + cxm;
                float dyy = cyp - 2.0f * cval + cym;
                float dxy = (dog_at(v, si, row + 1, col + 1) - dog_at(v, si, row + 1, col - 1) -
                             dog_at(v, si, row - 1, col + 1) + dog_at(v, si, row - 1, col - 1)) *
                            0.25f;
                float trace = dxx + dyy;
                float det2d = dxx * dyy - dxy * dxy;
                if (!(det2d <= 0.0f || (trace * trace / det2d) >= a.edge_score)) valid = 1;
            }
        }
        a.rv_valid[slot] = valid;
        if (valid) {
            a.rv_ri[slot] = (float)row + oy;
            a.rv_ci[slot] = (float)col + ox;
            a.rv_si[slot] = si;
            a.rv_resp[slot] = response;
        }
    }
}

// Ordered compaction of the valid refined candidates of one octave.
struct RefinedRow {
    float ri, ci, resp;
    int si, valid;
};
__global__ void __launch_bounds__(1024) k_refine_compact(const RefArgs a, Ctrl* ctrl) {
    if (a.retry_mode && !ctrl->retried) return;
    __shared__ int sh[33];
    const int o = blockIdx.x;
    const int n = ctrl->ncand[o];
    const long long base = (long long)o * a.cap;
    const int total = block_compact<8, RefinedRow>(
        n,
        [&](int j) {
            RefinedRow r;
            r.valid = a.rv_valid[base + j];
            r.ri = a.rv_ri[base + j];
            r.ci = a.rv_ci[base + j];
            r.si = a.rv_si[base + j];
            r.resp = a.rv_resp[base + j];
            return r;
        },
        [](const RefinedRow& r) { return r.valid != 0; },
        [&](int pos, const RefinedRow& r) {
            a.rf_ri[base + pos] = r.ri;
            a.rf_ci[base + pos] = r.ci;
            a.rf_si[base + pos] = r.si;
            a.rf_resp[base + pos] = r.resp;
        },
        sh);
    if (threadIdx.x == 0) ctrl->nref[o] = total;
}

__global__ void k_retry_decide(Ctrl* ctrl, int n_oct, int starvation_min) {
    int t = 0;
    for (int o = 0; o < n_oct; ++o) t += ctrl->nref[o];
    ctrl->retried = (t < starvation_min) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// A9: keypoint cap (top `cap` by response, stable).
// ---------------------------------------------------------------------------
struct CapArgs {
    int n_oct, cap_cand, kp_cap;
    const float* rf_ri;
    const float* rf_ci;
    const int* rf_si;
    const float* rf_resp;
    int* kp_o;
    int* kp_si;
    float* kp_ri;
    float* kp_ci;
    float* kp_resp;
    uint32_t* kp_tb;
};

__device__ __forceinline__ void global_to_local(const int* nref_pref, int n_oct, int g, int* o, int* j) {
    int oo = 0;
    while (oo + 1 < n_oct && g >= nref_pref[oo + 1]) ++oo;
    *o = oo;
    *j = g - nref_pref[oo];
}

// Keys of up to CAP_SMEM_KEYS refined keypoints are staged in shared memory
// for the radix passes; larger sets are read from global memory each pass.
constexpr int CAP_SMEM_KEYS = 40960;
constexpr int CAP_T = 1024;
constexpr size_t CAP_SMEM_BYTES = (size_t)(32 * 256 + CAP_SMEM_KEYS) * sizeof(unsigned int);

__global__ void __launch_bounds__(CAP_T) k_cap(const CapArgs a, Ctrl* ctrl) {
    extern __shared__ unsigned int cap_smem[];
    unsigned int* whist = cap_smem;              // [32 warps][256] private digit histograms
    unsigned int* s_keys = cap_smem + 32 * 256;  // staged keys
    __shared__ int sh[33];
    __shared__ int pref[PYSIFT_MAX_OCTAVES + 1];
    __shared__ unsigned int hist[256];
    __shared__ unsigned int s_prefix, s_mask;
    __shared__ int s_need;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        pref[0] = 0;
        for (int o = 0; o < a.n_oct; ++o) pref[o + 1] = pref[o] + ctrl->nref[o];
    }
    __syncthreads();
    const int total = pref[a.n_oct];
    const bool capped = total > a.kp_cap;
    auto load = [&](int g, int* o, int* j) {
        global_to_local(pref, a.n_oct, g, o, j);
        return (long long)(*o) * a.cap_cand + *j;
    };
    if (!capped) {
        for (int g = tid; g < total; g += CAP_T) {
            int o, j;
            long long src = load(g, &o, &j);
            a.kp_o[g] = o;
            a.kp_si[g] = a.rf_si[src];
            a.kp_ri[g] = a.rf_ri[src];
            a.kp_ci[g] = a.rf_ci[src];
            a.kp_resp[g] = a.rf_resp[src];
            a.kp_tb[g] = 0u;
        }
        if (tid == 0) {
            ctrl->n_total_ref = total;
            ctrl->n_kept = total;
            ctrl->capped = 0;
        }
        return;
    }
    const bool in_smem = total <= CAP_SMEM_KEYS;
    if (in_smem) {
        for (int g = tid; g < total; g += CAP_T) {
            int o, j;
            s_keys[g] = __float_as_uint(a.rf_resp[load(g, &o, &j)]);
        }
    }
    auto key_at = [&](int g) {
        if (in_smem) return s_keys[g];
        int o, j;
        return __float_as_uint(a.rf_resp[load(g, &o, &j)]);
    };
    // radix select of the kp_cap-th largest response (non-negative float bits)
    if (tid == 0) {
        s_prefix = 0u;
        s_mask = 0u;
        s_need = a.kp_cap;
    }
    for (int pass = 3; pass >= 0; --pass) {
        for (int i = tid; i < 32 * 256; i += CAP_T) whist[i] = 0u;
        __syncthreads();
        const unsigned int prefix = s_prefix, mask = s_mask;
        for (int g = tid; g < total; g += CAP_T) {
            const unsigned int key = key_at(g);
            if ((key & mask) == prefix) atomicAdd(&whist[warp * 256 + ((key >> (8 * pass)) & 255u)], 1u);
        }
        __syncthreads();
        for (int d = tid; d < 256; d += CAP_T) {
            unsigned int s = 0u;
#pragma unroll 8
            for (int w = 0; w < 32; ++w) s += whist[w * 256 + d];
            hist[d] = s;
        }
        __syncthreads();
        if (warp == 0) {
            // digit d with cum(> d) < need <= cum(>= d): warp suffix sums over 8-digit groups
            int grp = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) grp += (int)hist[lane * 8 + q];
            int suf = grp;  // inclusive suffix sum over lanes lane..31
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int v = __shfl_down_sync(FULL_MASK, suf, off);
                if (lane + off < 32) suf += v;
            }
            const int need = s_need;
            const int above = suf - grp;  // keys in higher groups
            const unsigned int who = __ballot_sync(FULL_MASK, above < need && need <= suf);
            if (lane == (who ? __ffs(who) - 1 : 0)) {
                int cum = above, d = lane * 8 + 7;
                for (; d > lane * 8; --d) {
                    if (cum + (int)hist[d] >= need) break;
                    cum += (int)hist[d];
                }
                s_need = need - cum;
                s_prefix = prefix | ((unsigned int)d << (8 * pass));
                s_mask = mask | (255u << (8 * pass));
            }
        }
        __syncthreads();
    }
    const unsigned int T = s_prefix;
    const int need_eq = s_need;
    // kept = every key > T and the first need_eq keys == T (index order), at
    // position #greater-before + min(#equal-before, need_eq); warp ballots of
    // both conditions and one packed scan of the warp counts per chunk
    constexpr int K = 8;
    const unsigned below = (1u << lane) - 1u;
    int gt_base = 0, eq_base = 0;
    for (int c0 = 0; c0 < total; c0 += CAP_T * K) {
        const int wbase = c0 + warp * 32 * K;
        unsigned int key[K], bgt[K], beq[K];
        int so[K], ssi[K];
        float sri[K], sci[K], sresp[K];
        // every load of the chunk first (coalesced within an octave), then the stores
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int g = wbase + k * 32 + lane;
            so[k] = 0;
            ssi[k] = 0;
            sri[k] = sci[k] = sresp[k] = 0.0f;
            if (g < total) {
                int o, j;
                const long long src = load(g, &o, &j);
                so[k] = o;
                ssi[k] = a.rf_si[src];
                sri[k] = a.rf_ri[src];
                sci[k] = a.rf_ci[src];
                sresp[k] = a.rf_resp[src];
            }
            key[k] = __float_as_uint(sresp[k]);
        }
        int cg = 0, ce = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int g = wbase + k * 32 + lane;
            bgt[k] = __ballot_sync(FULL_MASK, g < total && key[k] > T);
            beq[k] = __ballot_sync(FULL_MASK, g < total && key[k] == T);
            cg += __popc(bgt[k]);
            ce += __popc(beq[k]);
        }
        int tot;
        const int pre = block_warp_excl_scan(cg | (ce << 16), &tot, sh);
        int pg = gt_base + (pre & 0xffff), pe = eq_base + (pre >> 16);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const bool is_gt = (bgt[k] >> lane) & 1u, is_eq = (beq[k] >> lane) & 1u;
            const int gb = pg + __popc(bgt[k] & below), eb = pe + __popc(beq[k] & below);
            if (is_gt || (is_eq && eb < need_eq)) {
                const int pos = gb + min(eb, need_eq);
                a.kp_o[pos] = so[k];
                a.kp_si[pos] = ssi[k];
                a.kp_ri[pos] = sri[k];
                a.kp_ci[pos] = sci[k];
                a.kp_resp[pos] = sresp[k];
                a.kp_tb[pos] = ~key[k];
            }
            pg += __popc(bgt[k]);
            pe += __popc(beq[k]);
        }
        gt_base += tot & 0xffff;
        eq_base += tot >> 16;
    }
    if (tid == 0) {
        ctrl->n_total_ref = total;
        ctrl->n_kept = gt_base + min(eq_base, need_eq);
        ctrl->capped = 1;
    }
}

// ---------------------------------------------------------------------------
// A10: orientation.
// ---------------------------------------------------------------------------
struct OriArgs {
    OctView oct[PYSIFT_MAX_OCTAVES];
    float ori_sigma[PYSIFT_MAX_LEVELS];
    const int* kp_o;
    const int* kp_si;
    const float* kp_ri;
    const float* kp_ci;
    float* ang;
    int* angcnt;
};

// Exact, order-independent orientation histograms: each non-negative float32
// contribution is rounded to a multiple of 2^-40 (round to nearest even) and
// added as a 64-bit integer; a bin's value is the integer sum rounded to
// float32 and scaled back.  Contributions are below 2.2 (gradient magnitudes
// of pyramid values in [-0.28, 1.28]), so sums stay far below 2^63.  This makes the histograms independent of which thread adds
// what when, so any number of threads can share a keypoint.
__device__ __forceinline__ unsigned long long fix40(float c) {
    return (unsigned long long)__float2ll_rn(c * 0x1p40f);
}
__device__ __forceinline__ float unfix40(unsigned long long s) { return __ll2float_rn((long long)s) * 0x1p-40f; }

// Warp-private fixed-point orientation histograms with native 32-bit
// shared atomics.  A value q < 2^42 is added as two limbs, q mod 2^21 into
// lo[bin] and q >> 21 into hi[bin]; every FOLD_STEPS warp steps (at most 4
// values per lane and bin per step) the limbs are folded into a 64-bit total
// and cleared, so neither limb can overflow.  Integer sums keep the totals
// exact and independent of the order of the atomics.
constexpr int FOLD_STEPS = 8;

struct WarpHist {
    unsigned int* lo;
    unsigned int* hi;
    unsigned long long* tot;
    int nbins;
    __device__ __forceinline__ int phys(int bin) const { return bin; }
    __device__ __forceinline__ void add(int bin, unsigned long long q) const {
        const int p = phys(bin);
        atomicAdd(lo + p, (unsigned int)(q & 0x1fffffull));
        atomicAdd(hi + p, (unsigned int)(q >> 21));
    }
    // all lanes of the warp call fold() together
    __device__ __forceinline__ void fold() const {
        __syncwarp();
        for (int b = (int)(threadIdx.x & 31); b < nbins; b += 32) {
            const int p = phys(b);
            tot[b] += ((unsigned long long)hi[p] << 21) + (unsigned long long)lo[p];
            lo[p] = 0u;
            hi[p] = 0u;
        }
        __syncwarp();
    }
};

// fmodf(x, 360.0f) for x in (-360, 720): the remainder is exact in both forms
// (Sterbenz), so this matches fmodf bit for bit on the ranges the orientation
// (x in [180, 540]) and descriptor (x in (-180, 540]) formulas produce.
__device__ __forceinline__ float mod360(float x) { return x >= 360.0f ? x - 360.0f : x; }

constexpr int ORI_T = 64;
constexpr int ORI_W = ORI_T / 32;

// One ORI_T-thread block per kept keypoint at a time: the first is the
// block index, later ones come from a counter (windows differ in size), the
// next index requested when a keypoint starts and read when it ends.
__global__ void __launch_bounds__(ORI_T) k_orientation(const OriArgs a, Ctrl* ctrl) {
    __shared__ unsigned int wlo[ORI_W][36], whi[ORI_W][36];
    __shared__ unsigned long long whist[ORI_W][36];
    __shared__ float h0[36], h1[36];
    __shared__ int s_next[2];  // alternates, so a late reader never sees the next keypoint
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = ctrl->n_kept;
    int i = blockIdx.x;
    for (int it = 0; i < n; ++it) {
        int next = 0;
        if (tid == 0) next = (int)gridDim.x + atomicAdd(&ctrl->ori_next, 1);
        for (int b = tid; b < ORI_W * 36; b += ORI_T) {
            (&whist[0][0])[b] = 0ull;
            (&wlo[0][0])[b] = 0u;
            (&whi[0][0])[b] = 0u;
        }
        __syncthreads();
        const int o = a.kp_o[i], si = a.kp_si[i];
        const float ri = a.kp_ri[i], ci = a.kp_ci[i];
        const float sigma = a.ori_sigma[si];
        const OctView& v = a.oct[o];
        const int H = v.H, W = v.W;
        int radius = (int)(4.5f * sigma + 0.5f);
        if (radius < 1) radius = 1;
        const float sigma_w = 1.5f * sigma;
        const float inv_2sw2 = 1.0f / (2.0f * sigma_w * sigma_w + 1e-12f);
        int r_min = (int)ri - radius;
        if (r_min < 1) r_min = 1;
        int r_max = (int)ri + radius;
        if (r_max > H - 2) r_max = H - 2;
        int c_min = (int)ci - radius;
        if (c_min < 1) c_min = 1;
        int c_max = (int)ci + radius;
        if (c_max > W - 2) c_max = W - 2;
        int n_cols = c_max - c_min + 1;
        if (n_cols < 1) n_cols = 1;
        int nr = r_max - r_min + 1;
        if (nr < 0) nr = 0;
        const float* g = v.lev[si];
        const long long P = v.pitch;
        const WarpHist hw{wlo[warp], whi[warp], whist[warp], 36};
        // 8x4 pixel blocks per warp step
        const int tcols = (n_cols + 7) >> 3, trows = (nr + 3) >> 2;
        const int ntiles = tcols * trows;
        int steps = 0;
        // tile t -> (t / tcols, t % tcols), advanced ORI_W tiles at a time
        const int dty = ORI_W / tcols, dtx = ORI_W - dty * tcols;
        int ty = warp / tcols, tx = warp - ty * tcols;
        for (int t = warp; t < ntiles; t += ORI_W) {
            const int pr = ty * 4 + (lane >> 3), pc = tx * 8 + (lane & 7);
            tx += dtx;
            ty += dty;
            if (tx >= tcols) {
                tx -= tcols;
                ++ty;
            }
            const bool act = pr < nr && pc < n_cols;
            if (act) {
                const int r = r_min + pr, c = c_min + pc;
                const float* gp = g + r * P + c;
                float dx = gp[1] - gp[-1];
                float dy = gp[P] - gp[-P];
                float mag = sqrtf(dx * dx + dy * dy);
                float ori = mod360(sm::atan2f_(dy, dx) * 57.29577951f + 360.0f);
                float fr = (float)r - ri, fc = (float)c - ci;
                float wt = sm::expf_(-(fr * fr + fc * fc) * inv_2sw2);
                float bin_f = ori * 0.1f;
                const int b0 = ((int)bin_f) % 36;
                const int b1 = (b0 + 1) % 36;
                float frac = bin_f - floorf(bin_f);
                float mw = mag * wt;
                hw.add(b0, fix40(mw * (1.0f - frac)));
                hw.add(b1, fix40(mw * frac));
            }
            if (++steps == FOLD_STEPS) {
                hw.fold();
                steps = 0;
            }
        }
        hw.fold();
        __syncthreads();
        // smoothing and peaks in warp 0: lane l owns bins l and l + 32 (l < 4),
        // same arithmetic per bin; the peak height is a maximum (order-free)
        if (warp == 0) {
            for (int b = lane; b < 36; b += 32) {
                unsigned long long s = 0ull;
                for (int w = 0; w < ORI_W; ++w) s += whist[w][b];
                h0[b] = unfix40(s);
            }
            __syncwarp();
            for (int b = lane; b < 36; b += 32)
                h1[b] = 0.25f * h0[(b + 35) % 36] + 0.5f * h0[b] + 0.25f * h0[(b + 1) % 36];
            __syncwarp();
            for (int b = lane; b < 36; b += 32)
                h0[b] = 0.25f * h1[(b + 35) % 36] + 0.5f * h1[b] + 0.25f * h1[(b + 1) % 36];
            __syncwarp();
            float peak = 0.0f;
            for (int b = lane; b < 36; b += 32) peak = fmaxf(peak, h0[b]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) peak = fmaxf(peak, __shfl_xor_sync(FULL_MASK, peak, o));
            const float thr = 0.8f * peak;
            bool pk[2] = {false, false};
            float ang2[2] = {0.0f, 0.0f};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int b = lane + 32 * h;
                if (b >= 36) continue;
                const float hb = h0[b];
                if (hb >= thr) {
                    const float l = h0[(b + 35) % 36], rv = h0[(b + 1) % 36];
                    if (hb >= l && hb >= rv) {
                        pk[h] = true;
                        const float denom = l - 2.0f * hb + rv;
                        const float fine = (float)b + (fabsf(denom) > 1e-12f ? 0.5f * (l - rv) / denom : 0.0f);
                        ang2[h] = fmodf(fine / 36.0f * 360.0f + 360.0f, 360.0f);
                    }
                }
            }
            const unsigned m0 = __ballot_sync(FULL_MASK, pk[0]), m1 = __ballot_sync(FULL_MASK, pk[1]) & 0xfu;
            const unsigned below = (1u << lane) - 1u;
            const int before0 = __popc(m0 & below), before1 = __popc(m0) + __popc(m1 & below);
            if (pk[0] && before0 < 4) a.ang[i * 4 + before0] = ang2[0];
            if (pk[1] && before1 < 4) a.ang[i * 4 + before1] = ang2[1];
            if (lane == 0) {
                const int cnt = min(4, __popc(m0) + __popc(m1));
                a.angcnt[i] = cnt;
                for (int k = cnt; k < 4; ++k) a.ang[i * 4 + k] = -1.0f;
            }
        }
        if (tid == 0) s_next[it & 1] = next;
        __syncthreads();
        i = s_next[it & 1];
    }
}

// ---------------------------------------------------------------------------
// Expansion into oriented keypoints + output sort keys.
// ---------------------------------------------------------------------------
struct ExpArgs {
    const int* kp_o;
    const int* kp_si;
    const float* kp_ri;
    const float* kp_ci;
    const uint32_t* kp_tb;
    const int* angcnt;
    int* ent_kp;
    int* ent_slot;
    uint4* keys;
    float coord_scale[PYSIFT_MAX_OCTAVES];  // 2^o * (0.5 if doubled else 1)
    int* xy_cnt;                             // per-bucket counts of the (x, y) order (zeroed)
    int* blk_cnt;                            // entries per k_expand block
    float xy_bscale;                         // BR_NB / image width
};

// Bucket of an (x, y) sort key: its x (a non-negative float) scaled to
// BR_NB bins over the image width.  Non-decreasing in x, hence in the key
// order (x first).
__device__ __forceinline__ int br_bucket_xy(const uint4& k, float bscale) {
    const float t = __uint_as_float(k.x) * bscale;
    return t < (float)(BR_NB - 1) ? (int)t : BR_NB - 1;
}
// Bucket of a response in the output-limit order (larger first): BR_NB - 1
// minus the float's exponent and top 8 mantissa bits, offset so that the
// BR_NB buckets span [2^-12, 2^4) (256 per octave) and clamped at both ends.
// Non-decreasing in that order for non-negative responses.
__device__ __forceinline__ int br_bucket_resp(float r) {
    constexpr int OFF = (127 - 12) << 8;  // the bucket of 2^-12
    const int f = (int)(__float_as_uint(r) >> 15) - OFF;
    return BR_NB - 1 - (f < 0 ? 0 : (f > BR_NB - 1 ? BR_NB - 1 : f));
}

// Expansion of the kept keypoints into their oriented entries (1..4 each),
// in keypoint order, over EXP_T x EXP_K keypoints per block: k_expand_count
// writes each block's entry count; in k_expand each block adds up the counts
// of the blocks before it (there are few) for its first entry, and a block
// scan places its own entries.  The last block stores the total.
constexpr int EXP_K = 8;
constexpr int EXP_T = 256;
constexpr int EXP_PER_BLOCK = EXP_T * EXP_K;

__global__ void __launch_bounds__(EXP_T) k_expand_count(const ExpArgs a, const Ctrl* ctrl) {
    __shared__ int sh[33];
    const int n = ctrl->n_kept;
    const int i0 = blockIdx.x * EXP_PER_BLOCK + (int)threadIdx.x * EXP_K;
    int local = 0;
#pragma unroll
    for (int k = 0; k < EXP_K; ++k)
        if (i0 + k < n) local += a.angcnt[i0 + k];
    int tot;
    block_excl_scan(local, &tot, sh);
    if (threadIdx.x == 0) a.blk_cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(EXP_T) k_expand(const ExpArgs a, Ctrl* ctrl) {
    __shared__ int sh[33];
    __shared__ int s_base;
    const int n = ctrl->n_kept;
    if (threadIdx.x < 32) {
        int sum = 0;
        for (int b = (int)threadIdx.x; b < (int)blockIdx.x; b += 32) sum += a.blk_cnt[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL_MASK, sum, o);
        if (threadIdx.x == 0) s_base = sum;
    }
    const int i0 = blockIdx.x * EXP_PER_BLOCK + (int)threadIdx.x * EXP_K;
    int cnt[EXP_K];
    uint32_t kx[EXP_K], ky[EXP_K], tb[EXP_K];
    int local = 0;
#pragma unroll
    for (int k = 0; k < EXP_K; ++k) {
        const int i = i0 + k;
        cnt[k] = 0;
        kx[k] = ky[k] = tb[k] = 0u;
        if (i < n) {
            cnt[k] = a.angcnt[i];
            const float sc = a.coord_scale[a.kp_o[i]];
            kx[k] = __float_as_uint(a.kp_ci[i] * sc);
            ky[k] = __float_as_uint(a.kp_ri[i] * sc);
            tb[k] = a.kp_tb[i];
        }
        local += cnt[k];
    }
    int tot;
    const int excl = block_excl_scan(local, &tot, sh);  // its barriers also publish s_base
    int pos = s_base + excl;
#pragma unroll
    for (int k = 0; k < EXP_K; ++k) {
        const int i = i0 + k;
        for (int q = 0; q < cnt[k]; ++q) {
            a.ent_kp[pos + q] = i;
            a.ent_slot[pos + q] = q;
            const uint4 key = make_uint4(kx[k], ky[k], tb[k], (uint32_t)(i * 4 + q));
            a.keys[pos + q] = key;
            atomicAdd(&a.xy_cnt[br_bucket_xy(key, a.xy_bscale)], 1);
        }
        pos += cnt[k];
    }
    if (threadIdx.x == 0 && blockIdx.x == gridDim.x - 1) ctrl->n_oriented = s_base + tot;
}

__device__ __forceinline__ bool key_less(const uint4& p, const uint4& q) {
    if (p.x != q.x) return p.x < q.x;
    if (p.y != q.y) return p.y < q.y;
    if (p.z != q.z) return p.z < q.z;
    return p.w < q.w;
}

// Exact ranks through buckets.  Keys follow a strict total order; a bucket
// function that never decreases along the order gives
//   rank[i] = #{keys in lower buckets} + #{keys of i's bucket ordered before i},
// the same count as comparing every pair.  Counts come from the kernel that
// writes the keys; k_br_scan turns them into bucket starts, k_br_scatter
// lists each bucket's members (in any order: the in-bucket count does not
// depend on it) and k_br_rank counts.  ORD 0: the (x, y) sort keys, rank =
// output row.  ORD 1: the rows' responses, larger first, ties by lower row
// (the output-limit order); nothing to do unless there are more rows than
// the limit.
struct BRArgs {
    const uint4* keys;      // ORD 0
    const float* row_resp;  // ORD 1
    float xy_bscale;
    int limit;              // ORD 1
    int* cnt;               // [BR_NB] counts
    int* off;               // [BR_NB] bucket starts
    int* cursor;            // [BR_NB] fill positions
    int* members;
    int* rank;
};

template <int ORD>
__device__ __forceinline__ bool br_skip(const BRArgs& a, int n) {
    return ORD == 1 && n <= a.limit;
}
template <int ORD>
__device__ __forceinline__ int br_bucket(const BRArgs& a, int i) {
    if (ORD == 0) return br_bucket_xy(a.keys[i], a.xy_bscale);
    return br_bucket_resp(a.row_resp[i]);
}

template <int ORD>
__global__ void __launch_bounds__(1024) k_br_scan(const BRArgs a, const Ctrl* ctrl) {
    __shared__ int sh[33];
    if (br_skip<ORD>(a, ctrl->n_oriented)) return;
    constexpr int PER = BR_NB / 1024;
    int c[PER], local = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        c[k] = a.cnt[threadIdx.x * PER + k];
        local += c[k];
    }
    int tot;
    int pos = block_excl_scan(local, &tot, sh);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        a.off[threadIdx.x * PER + k] = pos;
        a.cursor[threadIdx.x * PER + k] = pos;
        pos += c[k];
    }
}

template <int ORD>
__global__ void k_br_scatter(const BRArgs a, const Ctrl* ctrl) {
    const int n = ctrl->n_oriented;
    if (br_skip<ORD>(a, n)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a.members[atomicAdd(&a.cursor[br_bucket<ORD>(a, i)], 1)] = i;
}

template <int ORD>
__global__ void k_br_rank(const BRArgs a, const Ctrl* ctrl) {
    const int n = ctrl->n_oriented;
    if (br_skip<ORD>(a, n)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = br_bucket<ORD>(a, i);
        const int s0 = a.off[b], s1 = s0 + a.cnt[b];
        int r = s0;
        if (ORD == 0) {
            const uint4 me = a.keys[i];
            for (int s = s0; s < s1; ++s) r += key_less(a.keys[a.members[s]], me) ? 1 : 0;
        } else {
            const float me = a.row_resp[i];
            for (int s = s0; s < s1; ++s) {
                const int j = a.members[s];
                const float o = a.row_resp[j];
                r += (o > me || (o == me && j < i)) ? 1 : 0;
            }
        }
        a.rank[i] = r;
    }
}

// ---------------------------------------------------------------------------
// A11: descriptor.
// ---------------------------------------------------------------------------
struct DescArgs {
    OctView oct[PYSIFT_MAX_OCTAVES];
    float desc_ph[PYSIFT_MAX_LEVELS];
    float kp_size[PYSIFT_MAX_OCTAVES][PYSIFT_MAX_LEVELS];
    float coord_scale[PYSIFT_MAX_OCTAVES];
    float dsp_scales[8];
    int n_dsp;  // 0 = single scale
    int rootsift;
    const int* kp_o;
    const int* kp_si;
    const float* kp_ri;
    const float* kp_ci;
    const float* kp_resp;
    const float* ang;
    const int* ent_kp;
    const int* ent_slot;
    const int* rank;
    const int* lrank;  // rank by response of each output row (output_limit > 0)
    int limit;
    float* out_kpts;
    float* out_resp;
    int* out_oct;
    float* out_desc;
};

constexpr int DESC_T = 256;
constexpr int DESC_W = DESC_T / 32;
// Lane layout of a descriptor warp step: the 32 lanes form DESC_GR x DESC_GC
// groups of DESC_L consecutive pixels of one row; the groups sit in
// different row bands and column bands of the patch (a band is 1/DESC_GR of
// the patch height, 1/DESC_GC of its width), so lanes of different groups
// fall in different spatial bins and their histogram updates do not
// serialise on one shared-memory word, while each group's loads stay
// contiguous.
#ifndef DESC_GR
#define DESC_GR 4
#endif
#ifndef DESC_GC
#define DESC_GC 2
#endif
constexpr int DESC_L = 32 / (DESC_GR * DESC_GC);
static_assert(DESC_GR * DESC_GC * DESC_L == 32, "descriptor lane groups must tile a warp");

// Descriptor histograms: exact fixed point at a quantum of 2^-24, one 32-bit
// shared word per bin and warp (one atomic per corner).  Pyramid values lie
// in [-0.28, 1.28] (u8/255, widened by the cubic spline of the 2x base), so
// a gradient magnitude is below 2.2 and a pixel's eight corner weights sum
// to at most that; a warp step adds at most 32 * 2.2 * 2^24 + 64 < 1.19e9 to
// one bin, and folding the words into 64-bit totals every DESC_FOLD_STEPS = 3
// steps keeps them below 2^32.  Bin b sits at b ^ (ycell << 3), so the
// y-cell moves a bin to another bank.
constexpr int DESC_FOLD_STEPS = 3;
__device__ __forceinline__ unsigned fix24(float c) { return __float2uint_rn(c * 0x1p24f); }
__device__ __forceinline__ float unfix24(unsigned long long s) { return __ull2float_rn(s) * 0x1p-24f; }

struct DescHist {
    unsigned* h;               // [128] words of this warp
    unsigned long long* tot;   // [128] totals of this warp
    __device__ static __forceinline__ int phys(int bin) { return bin ^ (((bin >> 5) & 3) << 3); }
    // all lanes of the warp call fold() together
    __device__ __forceinline__ void fold() const {
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int b = (int)(threadIdx.x & 31) + 32 * i;
            const int p = phys(b);
            tot[b] += (unsigned long long)h[p];
            h[p] = 0u;
        }
        __syncwarp();
    }
};

__device__ __forceinline__ void desc_accumulate(const float* __restrict__ g, long long P, int H, int W, float ri,
                                                float ci, float cos_a, float sin_a, float ang_rad, int ph,
                                                const DescHist& hw, int tid) {
    const float scale_sp = 4.0f / (2.0f * (float)ph);
    const float sigma_d = (float)ph * 0.5657f;
    const float inv_2s2 = 1.0f / (2.0f * sigma_d * sigma_d + 1e-12f);
    const int side = 2 * ph + 1;
    const int r0 = (int)ri, c0 = (int)ci;
    const int lane = tid & 31, warp = tid >> 5;
    const int k = lane % DESC_L, grp = lane / DESC_L;
    const int gi = grp / DESC_GC, gj = grp - gi * DESC_GC;
    const int band_r = (side + DESC_GR - 1) / DESC_GR;  // rows per row band
    const int band_c = (side + DESC_GC - 1) / DESC_GC;  // columns per column band
    const int runs = (band_c + DESC_L - 1) / DESC_L;    // DESC_L-pixel runs per band row
    const int nsteps = band_r * runs;
    // step t -> (u, v) = (t / runs, t % runs), advanced by DESC_W steps at a
    // time with one carry instead of a division per step
    const int du = DESC_W / runs, dv = DESC_W - du * runs;
    int u = warp / runs, v = warp - u * runs;
    const int pr0 = gi * band_r, pc0 = gj * band_c + k;
    unsigned* const hb = hw.h;
    int steps = 0;
    for (int t = warp; t < nsteps; t += DESC_W) {
        const int pr = pr0 + u, pcb = v * DESC_L + k, pc = pc0 + v * DESC_L;
        v += dv;
        u += du;
        if (v >= runs) {
            v -= runs;
            ++u;
        }
        const int r_off = pr - ph, c_off = pc - ph;
        const int rr = r0 + r_off, cc = c0 + c_off;
        bool act = pr < side && pcb < band_c && pc < side && !(rr < 1 || rr >= H - 1 || cc < 1 || cc >= W - 1);
        float fc = (float)c_off, fr = (float)r_off;
        float xr = cos_a * fc - sin_a * fr;
        float yr = sin_a * fc + cos_a * fr;
        float xb = xr * scale_sp + 1.5f;
        float yb = yr * scale_sp + 1.5f;
        act = act && !(xb < -0.5f || xb >= 3.5f || yb < -0.5f || yb >= 3.5f);
        if (act) {
            const float* gp = g + rr * P + cc;
            float dx = gp[1] - gp[-1];
            float dy = gp[P] - gp[-P];
            float mag = sqrtf(dx * dx + dy * dy);
            float ori_deg = mod360((sm::atan2f_(dy, dx) - ang_rad) * 57.29577951f + 360.0f);
            float gw = sm::expf_(-(xr * xr + yr * yr) * inv_2s2);
            const float wmag = mag * gw;
            float ob = ori_deg * 0.02222222f;
            int oi0 = (int)floorf(ob);
            float df = ob - (float)oi0;
            int xi0 = (int)floorf(xb), yi0 = (int)floorf(yb);
            float dx_b = xb - (float)xi0, dy_b = yb - (float)yi0;
            const int xi0c = max(0, min(xi0, 3));
            const int yi0c = max(0, min(yi0, 3));
            const int xi1c = max(0, min(xi0 + 1, 3));
            const int yi1c = max(0, min(yi0 + 1, 3));
            // orientation bins mod 8 (two's complement & 7 is the
            // non-negative remainder for every int)
            const int oi0w = oi0 & 7, oi1w = (oi0 + 1) & 7;
            float w_y0 = 1.0f - dy_b, w_y1 = dy_b;
            float w_x0 = 1.0f - dx_b, w_x1 = dx_b;
            float w_o0 = 1.0f - df, w_o1 = df;
            // shared-memory word of bin y*32 + x*8 + o: the descriptor
            // histograms store it at y*32 + ((x ^ y) << 3) + o
            const int b00 = yi0c * 32 + ((xi0c ^ yi0c) << 3), b01 = yi0c * 32 + ((xi1c ^ yi0c) << 3);
            const int b10 = yi1c * 32 + ((xi0c ^ yi1c) << 3), b11 = yi1c * 32 + ((xi1c ^ yi1c) << 3);
            const unsigned q[8] = {
                fix24(w_y0 * w_x0 * w_o0 * wmag), fix24(w_y0 * w_x0 * w_o1 * wmag),
                fix24(w_y0 * w_x1 * w_o0 * wmag), fix24(w_y0 * w_x1 * w_o1 * wmag),
                fix24(w_y1 * w_x0 * w_o0 * wmag), fix24(w_y1 * w_x0 * w_o1 * wmag),
                fix24(w_y1 * w_x1 * w_o0 * wmag), fix24(w_y1 * w_x1 * w_o1 * wmag)};
            const int pb[8] = {b00 + oi0w, b00 + oi1w, b01 + oi0w, b01 + oi1w,
                               b10 + oi0w, b10 + oi1w, b11 + oi0w, b11 + oi1w};
#pragma unroll
            for (int c = 0; c < 8; ++c) atomicAdd(hb + pb[c], q[c]);
        }
        if (++steps == DESC_FOLD_STEPS) {
            hw.fold();
            steps = 0;
        }
    }
    hw.fold();
}

__device__ __forceinline__ float warp_tree_sum(float v) {
    v += __shfl_down_sync(FULL_MASK, v, 16);
    v += __shfl_down_sync(FULL_MASK, v, 8);
    v += __shfl_down_sync(FULL_MASK, v, 4);
    v += __shfl_down_sync(FULL_MASK, v, 2);
    v += __shfl_down_sync(FULL_MASK, v, 1);
    return v;
}

// Sum over the 128 bins (thread = bin) in the reference's order: a warp
// shuffle tree per 32 bins, then the four warp partials in order.
// Called by threads 0..127 only (named barrier 1 over those 4 warps).
__device__ __forceinline__ float bins_sum(float x, float* part) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float w = warp_tree_sum(x);
    if (lane == 0) part[warp] = w;
    asm volatile("bar.sync 1, 128;" ::: "memory");
    float s = part[0] + part[1] + part[2] + part[3];
    asm volatile("bar.sync 1, 128;" ::: "memory");
    return s;
}

// One DESC_T-thread block per oriented keypoint at a time; a block takes its
// next entry from a counter (entries differ in patch size, so blocks stay
// busy until the list is done; every entry writes its own output row).
// Warps accumulate into private fixed-point histograms; threads 0..127 then
// own one bin each for the merge, normalisation and RootSIFT.
__global__ void __launch_bounds__(DESC_T, 5) k_descriptor(const DescArgs a, Ctrl* ctrl) {
    __shared__ unsigned int wh32[DESC_W][128];
    __shared__ unsigned long long whist[DESC_W][128];
    __shared__ float part[4];
    __shared__ int s_entry[2];  // alternates, so a late reader never sees the next entry
    const int tid = threadIdx.x, warp = tid >> 5;
    const int n = ctrl->n_oriented;
    // the first entry is the block index, later ones come from the counter;
    // the next index is requested when an entry starts and read when it ends
    int e = blockIdx.x;
    for (int it = 0; e < n; ++it) {
        int next = 0;
        if (tid == 0) next = (int)gridDim.x + atomicAdd(&ctrl->desc_next, 1);
        for (int b = tid; b < DESC_W * 128; b += DESC_T) {
            (&whist[0][0])[b] = 0ull;
            (&wh32[0][0])[b] = 0u;
        }
        __syncthreads();
        int row = a.rank[e];
        if (a.limit > 0 && n > a.limit) row = a.lrank[row];
        if (!(a.limit > 0 && n > a.limit) || row < a.limit) {  // else the whole block skips this entry
            const int kp = a.ent_kp[e], slot = a.ent_slot[e];
            const int o = a.kp_o[kp], si = a.kp_si[kp];
            const float ri = a.kp_ri[kp], ci = a.kp_ci[kp];
            const float angle = a.ang[kp * 4 + slot];
            const float ang_rad = angle * (float)(3.14159265358979323846 / 180.0);
            const float phf = a.desc_ph[si];
            const OctView& v = a.oct[o];
            float sin_a, cos_a;
            sm::sincosf_(ang_rad, &sin_a, &cos_a);
            const float* g = v.lev[si];
            const DescHist hw{wh32[warp], whist[warp]};
            if (a.n_dsp > 0) {
                for (int dd = 0; dd < a.n_dsp; ++dd) {
                    int ph = (int)(phf * a.dsp_scales[dd] + 0.5f);
                    if (ph < 4) ph = 4;
                    desc_accumulate(g, v.pitch, v.H, v.W, ri, ci, cos_a, sin_a, ang_rad, ph, hw, tid);
                }
            } else {
                desc_accumulate(g, v.pitch, v.H, v.W, ri, ci, cos_a, sin_a, ang_rad, (int)phf, hw, tid);
            }
            __syncthreads();
            if (tid < 128) {
                unsigned long long s = 0ull;
    #pragma unroll
                for (int w = 0; w < DESC_W; ++w) s += whist[w][tid];
                float val = unfix24(s);
                if (a.n_dsp > 0) val = val * (1.0f / (float)a.n_dsp);
                float inv = 1.0f / sqrtf(bins_sum(val * val, part) + 1e-14f);
                float t = val * inv;
                val = t > 0.2f ? 0.2f : t;
                inv = 1.0f / sqrtf(bins_sum(val * val, part) + 1e-14f);
                val = val * inv;
                if (a.rootsift) {
                    const float den = bins_sum(fabsf(val), part) + 1e-7f;
                    float q = val / den;
                    if (q < 0.0f) q = 0.0f;
                    val = sqrtf(q);
                }
                a.out_desc[(long long)row * 128 + tid] = val;
                if (tid == 0) {
                    const float sc = a.coord_scale[o];
                    a.out_kpts[row * 4 + 0] = ci * sc;
                    a.out_kpts[row * 4 + 1] = ri * sc;
                    a.out_kpts[row * 4 + 2] = a.kp_size[o][si];
                    a.out_kpts[row * 4 + 3] = angle;
                    a.out_resp[row] = a.kp_resp[kp];
                    a.out_oct[row] = o;
                }
            }
        }
        if (tid == 0) s_entry[it & 1] = next;
        __syncthreads();
        e = s_entry[it & 1];
    }
}

// Response of every output row (rows are the (x, y) ranks of the oriented
// entries), counted into the output-limit order's buckets.
__global__ void k_row_resp(const int* __restrict__ ent_kp, const float* __restrict__ kp_resp,
                           const int* __restrict__ rank, float* __restrict__ row_resp, int* __restrict__ resp_cnt,
                           const Ctrl* ctrl) {
    const int n = ctrl->n_oriented;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float r = kp_resp[ent_kp[e]];
        row_resp[rank[e]] = r;
        atomicAdd(&resp_cnt[br_bucket_resp(r)], 1);
    }
}

__global__ void k_finalize(const Ctrl* ctrl, int32_t* stats, int n_oct, int doubled, int limit) {
    int t = threadIdx.x;
    if (t < PYSIFT_STAT_COUNT) stats[t] = 0;
    __syncthreads();
    if (t == 0) {
        int nref = 0;
        for (int o = 0; o < n_oct; ++o) nref += ctrl->nref[o];
        stats[PYSIFT_STAT_N_KEYPOINTS] = (limit > 0 && ctrl->n_oriented > limit) ? limit : ctrl->n_oriented;
        stats[PYSIFT_STAT_N_REFINED] = nref;
        stats[PYSIFT_STAT_N_KEPT] = ctrl->n_kept;
        stats[PYSIFT_STAT_RETRIED] = ctrl->retried;
        stats[PYSIFT_STAT_CAPPED] = ctrl->capped;
        stats[PYSIFT_STAT_DOUBLED] = doubled;
        stats[PYSIFT_STAT_CAND_OVERFLOW] = ctrl->overflow_octs;
        for (int o = 0; o < n_oct; ++o) {
            stats[PYSIFT_STAT_CANDS + o] = ctrl->found[o];
            stats[PYSIFT_STAT_REFINED_OCT + o] = ctrl->nref[o];
        }
        stats[PYSIFT_STAT_THRESH_BITS] = (int32_t)__float_as_uint(ctrl->thr[ctrl->retried ? 1 : 0]);
    }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
template <typename T>
static T* at(void* ws, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(ws) + off);
}

static void fill_oct_views(const Layout& l, void* ws, bool rounded, OctView* out) {
    for (int o = 0; o < l.n_oct; ++o) {
        size_t off = rounded ? l.off_pyr_r[o] : l.off_pyr[o];
        float* base = at<float>(ws, off);
        for (int s = 0; s < PYSIFT_MAX_LEVELS; ++s)
            out[o].lev[s] = (s < l.L) ? base + (size_t)s * l.H[o] * l.pitch[o] : nullptr;
        out[o].H = l.H[o];
        out[o].W = l.W[o];
        out[o].pitch = l.pitch[o];
    }
}

static int g_num_sms = 0;

static int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        g_num_sms = n > 0 ? n : 148;
    }
    return g_num_sms;
}

// A second stream paired with each caller stream (per host thread and
// device), with events reused from call to call: work that only depends on
// part of the pyramid (the entropy histogram; levels S+1 and S+2 of each
// octave, which no later octave reads) runs there, forked from and joined
// back into the caller's stream, inside a CUDA graph capture too.  The pair
// is created on the first call made with that caller stream outside a
// capture; a call that captures on a stream without a pair returns null
// here and runs everything on the caller's stream (no objects are created
// while a capture is open).
struct SidePair {
    int dev;
    cudaStream_t main, side;
    cudaEvent_t ev[PYSIFT_MAX_OCTAVES + 2];
};

static SidePair* side_pair(cudaStream_t st) {
    constexpr int MAXP = 64;
    thread_local SidePair pairs[MAXP];
    thread_local int n = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_error("side_pair: no current device");
        return nullptr;
    }
    for (int i = 0; i < n; ++i)
        if (pairs[i].dev == dev && pairs[i].main == st) return &pairs[i];
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    if (n == MAXP) return nullptr;
    SidePair p{};
    p.dev = dev;
    p.main = st;
    if (cudaStreamCreateWithFlags(&p.side, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("side_pair: cudaStreamCreateWithFlags failed");
        return nullptr;
    }
    for (auto& e : p.ev) {
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            set_error("side_pair: cudaEventCreateWithFlags failed");
            return nullptr;
        }
    }
    pairs[n] = p;
    return &pairs[n++];
}

static int record_stage(void* const* ev, int i, cudaStream_t st) {
    if (ev && ev[i]) PYSIFT_CUDA_TRY(cudaEventRecord(reinterpret_cast<cudaEvent_t>(ev[i]), st));
    return PYSIFT_OK;
}

#define PYSIFT_STAGE(i)                              \
    do {                                             \
        int rc_ = record_stage(stage_events, i, st); \
        if (rc_) return rc_;                         \
    } while (0)

static int run_detect(const pysift_detect_config* cfg, const uint8_t* gray, int H, int W, long long pitch,
                      void* ws, const Layout& l, float* kpts, float* resp, int32_t* octv, float* desc,
                      int32_t* stats, void* const* stage_events, cudaStream_t st) {
    PYSIFT_STAGE(0);
    const int S = l.S, n_oct = l.n_oct;
    const int cap = cfg->max_cands_per_octave, kcap = cfg->keypoint_cap;
    Ctrl* ctrl = at<Ctrl>(ws, l.off_ctrl);
    PYSIFT_CUDA_TRY(cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st));
    SidePair* sp = side_pair(st);  // null: everything on st
    const cudaStream_t side = sp ? sp->side : st;
    if (sp) {
        PYSIFT_CUDA_TRY(cudaEventRecord(sp->ev[0], st));
        PYSIFT_CUDA_TRY(cudaStreamWaitEvent(side, sp->ev[0], 0));
    }
    // A1 (side stream; read by the extrema test after the join)
    {
        const int blocks = std::max(1, std::min(ceil_div(H, 8), num_sms() * 2));
        k_histogram<<<blocks, 256, 0, side>>>(gray, H, W, pitch, ctrl, cfg->contrast_thresh, S);
        PYSIFT_LAUNCH_CHECK("k_histogram");
    }
    // A2/A3: base image
    float* base = at<float>(ws, l.off_base);
    if (l.doubled) {
        double* coef = at<double>(ws, l.off_coef);
        int rc = launch_zoom2x(gray, H, W, pitch, cfg->fp16_pyramid, coef, base, l.pitch0, st);
        if (rc) return rc;
    } else {
        k_u8_to_f32<<<dim3(ceil_div(W, 256), H), 256, 0, st>>>(gray, H, W, pitch, cfg->fp16_pyramid, base,
                                                               l.pitch0);
        PYSIFT_LAUNCH_CHECK("k_u8_to_f32");
    }
    PYSIFT_STAGE(1);
    // A4/A5: pyramid
    {
        static thread_local BlurArgs a;  // large (weights by value); not on the stack
        for (int o = 0; o < n_oct; ++o) {
            float* pyr = at<float>(ws, l.off_pyr[o]);
            float* pyr_r = (l.off_pyr_r[o] != l.off_pyr[o]) ? at<float>(ws, l.off_pyr_r[o]) : nullptr;
            const size_t lev = (size_t)l.H[o] * l.pitch[o];
            // level 0
            memset(&a, 0, sizeof(a));
            a.H = l.H[o];
            a.W = l.W[o];
            a.out_pitch = l.pitch[o];
            if (o == 0) {
                int k = l.doubled ? 0 : 1;
                a.in = base;
                a.in_pitch = l.pitch0;
                a.step = 1;
                a.out = pyr;
                a.out_r = pyr_r;
                int rc = launch_blur(a, cfg->blur_radius[k], cfg->blur_weights[k], st);
                if (rc) return rc;
            }
            for (int s = 0; s < S + 2; ++s) {
                // levels S+1 and S+2 on the side stream, once level S exists
                cudaStream_t ls = st;
                if (s >= S) {
                    ls = side;
                    if (s == S && sp) {
                        PYSIFT_CUDA_TRY(cudaEventRecord(sp->ev[1 + o], st));
                        PYSIFT_CUDA_TRY(cudaStreamWaitEvent(side, sp->ev[1 + o], 0));
                    }
                }
                memset(&a, 0, sizeof(a));
                a.H = l.H[o];
                a.W = l.W[o];
                a.out_pitch = l.pitch[o];
                if (s == 0 && o > 0) {
                    const float* prev = at<float>(ws, l.off_pyr[o - 1]) + (size_t)S * l.H[o - 1] * l.pitch[o - 1];
                    a.in = prev;
                    a.in_pitch = l.pitch[o - 1];
                    a.step = 2;
                    a.copy0 = pyr;
                    a.copy0_r = pyr_r;
                } else {
                    a.in = pyr + (size_t)s * lev;
                    a.in_pitch = l.pitch[o];
                    a.step = 1;
                }
                a.out = pyr + (size_t)(s + 1) * lev;
                a.out_r = pyr_r ? pyr_r + (size_t)(s + 1) * lev : nullptr;
                int rc = launch_blur(a, cfg->blur_radius[2 + s], cfg->blur_weights[2 + s], ls);
                if (rc) return rc;
            }
        }
    }
    if (sp) {
        PYSIFT_CUDA_TRY(cudaEventRecord(sp->ev[PYSIFT_MAX_OCTAVES + 1], side));
        PYSIFT_CUDA_TRY(cudaStreamWaitEvent(st, sp->ev[PYSIFT_MAX_OCTAVES + 1], 0));
    }
    PYSIFT_STAGE(2);
    // A7/A8 (+ retry)
    static thread_local ExtArgs ea;
    static thread_local RefArgs ra;
    memset(&ea, 0, sizeof(ea));
    memset(&ra, 0, sizeof(ra));
    fill_oct_views(l, ws, true, ea.oct);
    fill_oct_views(l, ws, true, ra.oct);
    ea.n_oct = ra.n_oct = n_oct;
    ea.S = ra.S = S;
    ea.border = ra.border = cfg->border;
    ea.cap = ra.cap = cap;
    ea.cand = at<int4>(ws, l.off_cand);
    ra.cand = ea.cand;
    int mask_blocks = 0, row_blocks = 0;
    int row_off[PYSIFT_MAX_OCTAVES + 1];
    for (int o = 0; o < n_oct; ++o) {
        ea.blk_off[o] = mask_blocks;
        mask_blocks += ceil_div(l.H[o], EX_ROWS) * l.wpr[o];
        row_off[o] = row_blocks;
        row_blocks += ceil_div(S * l.H[o], 8);
        ea.mask[o] = at<uint32_t>(ws, l.off_mask[o]);
        ea.rowcnt[o] = at<int>(ws, l.off_rowcnt[o]);
        ea.rowoff[o] = at<int>(ws, l.off_rowoff[o]);
        ea.wpr[o] = l.wpr[o];
    }
    ea.blk_off[n_oct] = mask_blocks;
    row_off[n_oct] = row_blocks;
    ra.edge_score = cfg->edge_score;
    ra.rv_valid = at<int>(ws, l.off_rv_valid);
    ra.rv_ri = at<float>(ws, l.off_rv_ri);
    ra.rv_ci = at<float>(ws, l.off_rv_ci);
    ra.rv_si = at<int>(ws, l.off_rv_si);
    ra.rv_resp = at<float>(ws, l.off_rv_resp);
    ra.rf_ri = at<float>(ws, l.off_rf_ri);
    ra.rf_ci = at<float>(ws, l.off_rf_ci);
    ra.rf_si = at<int>(ws, l.off_rf_si);
    ra.rf_resp = at<float>(ws, l.off_rf_resp);
    const int refine_blocks = (int)std::min<long long>(ceil_div_ll((long long)n_oct * cap, 256), num_sms() * 8);
    for (int pass = 0; pass < 2; ++pass) {
        ea.thr_idx = ra.thr_idx = pass;
        ea.retry_mode = ra.retry_mode = pass;
        PYSIFT_CUDA_TRY(cudaMemsetAsync(at<char>(ws, l.off_rowcnt_base), 0, l.rowcnt_bytes_total, st));
        extrema_kernel(S)<<<mask_blocks, 256, 0, st>>>(ea, ctrl);
        PYSIFT_LAUNCH_CHECK("k_extrema_mask");
        if (pass == 0) PYSIFT_STAGE(3);
        k_rowscan<<<n_oct, 1024, 0, st>>>(ea, ctrl);
        PYSIFT_LAUNCH_CHECK("k_rowscan");
        // k_scatter indexes blocks by (s, r) rows: reuse blk_off for its own table
        ExtArgs& sa = ea;
        int saved[PYSIFT_MAX_OCTAVES + 1];
        memcpy(saved, sa.blk_off, sizeof(saved));
        memcpy(sa.blk_off, row_off, sizeof(row_off));
        k_scatter<<<row_blocks, 256, 0, st>>>(sa, ctrl);
        PYSIFT_LAUNCH_CHECK("k_scatter");
        memcpy(sa.blk_off, saved, sizeof(saved));
        k_refine<<<refine_blocks, 256, 0, st>>>(ra, ctrl);
        PYSIFT_LAUNCH_CHECK("k_refine");
        k_refine_compact<<<n_oct, 1024, 0, st>>>(ra, ctrl);
        PYSIFT_LAUNCH_CHECK("k_refine_compact");
        if (pass == 0) {
            k_retry_decide<<<1, 1, 0, st>>>(ctrl, n_oct, cfg->starvation_min);
            PYSIFT_LAUNCH_CHECK("k_retry_decide");
        }
    }
    // A9
    CapArgs ca;
    ca.n_oct = n_oct;
    ca.cap_cand = cap;
    ca.kp_cap = kcap;
    ca.rf_ri = ra.rf_ri;
    ca.rf_ci = ra.rf_ci;
    ca.rf_si = ra.rf_si;
    ca.rf_resp = ra.rf_resp;
    ca.kp_o = at<int>(ws, l.off_kp_o);
    ca.kp_si = at<int>(ws, l.off_kp_si);
    ca.kp_ri = at<float>(ws, l.off_kp_ri);
    ca.kp_ci = at<float>(ws, l.off_kp_ci);
    ca.kp_resp = at<float>(ws, l.off_kp_resp);
    ca.kp_tb = at<uint32_t>(ws, l.off_kp_tb);
    {
        PYSIFT_CUDA_TRY(
            cudaFuncSetAttribute(k_cap, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CAP_SMEM_BYTES));
        k_cap<<<1, CAP_T, CAP_SMEM_BYTES, st>>>(ca, ctrl);
    }
    PYSIFT_LAUNCH_CHECK("k_cap");
    PYSIFT_STAGE(4);
    // A10
    static thread_local OriArgs oa;
    memset(&oa, 0, sizeof(oa));
    fill_oct_views(l, ws, true, oa.oct);
    for (int s = 0; s < PYSIFT_MAX_LEVELS; ++s) oa.ori_sigma[s] = cfg->ori_sigma[s];
    oa.kp_o = ca.kp_o;
    oa.kp_si = ca.kp_si;
    oa.kp_ri = ca.kp_ri;
    oa.kp_ci = ca.kp_ci;
    oa.ang = at<float>(ws, l.off_ang);
    oa.angcnt = at<int>(ws, l.off_angcnt);
    k_orientation<<<std::min(kcap, num_sms() * 32), ORI_T, 0, st>>>(oa, ctrl);
    PYSIFT_LAUNCH_CHECK("k_orientation");
    // expansion + keys + rank
    ExpArgs xa;
    memset(&xa, 0, sizeof(xa));
    xa.kp_o = ca.kp_o;
    xa.kp_si = ca.kp_si;
    xa.kp_ri = ca.kp_ri;
    xa.kp_ci = ca.kp_ci;
    xa.kp_tb = ca.kp_tb;
    xa.angcnt = oa.angcnt;
    xa.ent_kp = at<int>(ws, l.off_ent_kp);
    xa.ent_slot = at<int>(ws, l.off_ent_slot);
    xa.keys = at<uint4>(ws, l.off_keys);
    for (int o = 0; o < n_oct; ++o) xa.coord_scale[o] = (float)((double)(1 << o) * (l.doubled ? 0.5 : 1.0));
    int* bkt = at<int>(ws, l.off_bkt);  // [order][cnt | off | cursor][BR_NB]
    PYSIFT_CUDA_TRY(cudaMemsetAsync(bkt, 0, sizeof(int) * 2 * 3 * BR_NB, st));
    xa.xy_cnt = bkt;
    xa.xy_bscale = (float)BR_NB / (float)W;
    xa.blk_cnt = at<int>(ws, l.off_xblk);
    const int exp_blocks = ceil_div(kcap, EXP_PER_BLOCK);
    k_expand_count<<<exp_blocks, EXP_T, 0, st>>>(xa, ctrl);
    k_expand<<<exp_blocks, EXP_T, 0, st>>>(xa, ctrl);
    PYSIFT_LAUNCH_CHECK("k_expand");
    int* rank = at<int>(ws, l.off_rank);
    const int br_blocks = std::max(1, std::min(ceil_div(4 * kcap, 256), num_sms() * 4));
    BRArgs bx{};
    bx.keys = xa.keys;
    bx.xy_bscale = xa.xy_bscale;
    bx.cnt = bkt;
    bx.off = bkt + BR_NB;
    bx.cursor = bkt + 2 * BR_NB;
    bx.members = at<int>(ws, l.off_members);
    bx.rank = rank;
    k_br_scan<0><<<1, 1024, 0, st>>>(bx, ctrl);
    k_br_scatter<0><<<br_blocks, 256, 0, st>>>(bx, ctrl);
    k_br_rank<0><<<br_blocks, 256, 0, st>>>(bx, ctrl);
    PYSIFT_LAUNCH_CHECK("k_br (x, y)");
    PYSIFT_STAGE(5);
    // A11
    static thread_local DescArgs da;
    memset(&da, 0, sizeof(da));
    fill_oct_views(l, ws, true, da.oct);
    for (int s = 0; s < PYSIFT_MAX_LEVELS; ++s) da.desc_ph[s] = cfg->desc_ph[s];
    for (int o = 0; o < n_oct; ++o) {
        for (int s = 0; s < PYSIFT_MAX_LEVELS; ++s) da.kp_size[o][s] = cfg->kp_size[l.doubled ? 1 : 0][o][s];
        da.coord_scale[o] = xa.coord_scale[o];
    }
    da.n_dsp = cfg->dsp ? cfg->n_dsp : 0;
    for (int d = 0; d < 8; ++d) da.dsp_scales[d] = cfg->dsp_scales[d];
    da.rootsift = cfg->rootsift;
    da.kp_o = ca.kp_o;
    da.kp_si = ca.kp_si;
    da.kp_ri = ca.kp_ri;
    da.kp_ci = ca.kp_ci;
    da.kp_resp = ca.kp_resp;
    da.ang = oa.ang;
    da.ent_kp = xa.ent_kp;
    da.ent_slot = xa.ent_slot;
    da.rank = rank;
    da.limit = cfg->output_limit;
    da.lrank = at<int>(ws, l.off_lrank);
    if (cfg->output_limit > 0) {
        float* row_resp = at<float>(ws, l.off_row_resp);
        BRArgs br{};
        br.row_resp = row_resp;
        br.limit = cfg->output_limit;
        br.cnt = bkt + 3 * BR_NB;
        br.off = bkt + 4 * BR_NB;
        br.cursor = bkt + 5 * BR_NB;
        br.members = at<int>(ws, l.off_members) + 4 * (size_t)kcap;
        br.rank = at<int>(ws, l.off_lrank);
        k_row_resp<<<br_blocks, 256, 0, st>>>(xa.ent_kp, ca.kp_resp, rank, row_resp, br.cnt, ctrl);
        PYSIFT_LAUNCH_CHECK("k_row_resp");
        k_br_scan<1><<<1, 1024, 0, st>>>(br, ctrl);
        k_br_scatter<1><<<br_blocks, 256, 0, st>>>(br, ctrl);
        k_br_rank<1><<<br_blocks, 256, 0, st>>>(br, ctrl);
        PYSIFT_LAUNCH_CHECK("k_br (response)");
    }
    da.out_kpts = kpts;
    da.out_resp = resp;
    da.out_oct = octv;
    da.out_desc = desc;
    k_descriptor<<<std::min(4 * kcap, num_sms() * 5), DESC_T, 0, st>>>(da, ctrl);
    PYSIFT_LAUNCH_CHECK("k_descriptor");
    k_finalize<<<1, 32, 0, st>>>(ctrl, stats, n_oct, l.doubled ? 1 : 0, cfg->output_limit);
    PYSIFT_LAUNCH_CHECK("k_finalize");
    PYSIFT_STAGE(6);
    return PYSIFT_OK;
}

}  // namespace pysift

using namespace pysift;

extern "C" {

const char* pysift_last_error(void) { return g_last_error.c_str(); }

const char* pysift_b200_version(void) { return "pysift_b200 0.1.0 (sm_100a)"; }

size_t pysift_detect_config_size(void) { return sizeof(pysift_detect_config); }

int64_t pysift_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

void pysift_count_launches(int64_t n) { g_launches.fetch_add((long long)n, std::memory_order_relaxed); }

int pysift_detect_workspace_size(const pysift_detect_config* cfg, int32_t H, int32_t W, size_t* bytes) {
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    PYSIFT_CHECK_ARG(H > 0 && W > 0, "image size %dx%d must be positive", H, W);
    PYSIFT_CHECK_ARG(bytes != nullptr, "bytes is NULL");
    Layout l = make_layout(cfg, H, W);
    *bytes = l.total;
    return PYSIFT_OK;
}

int32_t pysift_detect_max_keypoints(const pysift_detect_config* cfg) {
    if (!cfg) return 0;
    return 4 * cfg->keypoint_cap;
}

int pysift_detect_workspace_view(const pysift_detect_config* cfg, int32_t H, int32_t W, int32_t what, int32_t octave,
                                 int32_t level, size_t* offset, int32_t* rows, int32_t* cols, int32_t* pitch_floats) {
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    PYSIFT_CHECK_ARG(H > 0 && W > 0, "image size %dx%d must be positive", H, W);
    PYSIFT_CHECK_ARG(offset && rows && cols && pitch_floats, "NULL output pointer");
    Layout l = make_layout(cfg, H, W);
    if (what == 0) {
        PYSIFT_CHECK_ARG(octave >= 0 && octave < l.n_oct && level >= 0 && level < l.L, "octave/level out of range");
        *offset = l.off_pyr_r[octave] + (size_t)level * l.H[octave] * l.pitch[octave] * sizeof(float);
        *rows = l.H[octave];
        *cols = l.W[octave];
        *pitch_floats = l.pitch[octave];
    } else if (what == 1) {
        *offset = l.off_base;
        *rows = l.H0;
        *cols = l.W0;
        *pitch_floats = l.pitch0;
    } else {
        set_error("unknown view %d", what);
        return PYSIFT_ERR_INVALID_ARG;
    }
    return PYSIFT_OK;
}

int pysift_detect_and_compute(const pysift_detect_config* cfg, const uint8_t* gray, int32_t H, int32_t W,
                              int64_t pitch_bytes, void* workspace, size_t workspace_bytes, float* kpts,
                              float* response, int32_t* octave, float* desc, int32_t max_out, int32_t* stats,
                              void* const* stage_events, pysift_stream_t stream) {
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    PYSIFT_CHECK_ARG(H > 0 && W > 0, "image size %dx%d must be positive", H, W);
    PYSIFT_CHECK_ARG(pitch_bytes >= W, "pitch %lld smaller than width %d", (long long)pitch_bytes, W);
    PYSIFT_CHECK_ARG(gray && workspace && kpts && response && octave && desc && stats, "NULL pointer argument");
    Layout l = make_layout(cfg, H, W);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    if (max_out < 4 * cfg->keypoint_cap) {
        set_error("max_out %d < 4 * keypoint_cap (%d)", max_out, 4 * cfg->keypoint_cap);
        return PYSIFT_ERR_CAPACITY;
    }
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) {
        set_error("workspace must be 256-byte aligned");
        return PYSIFT_ERR_INVALID_ARG;
    }
    return run_detect(cfg, gray, H, W, pitch_bytes, workspace, l, kpts, response, octave, desc, stats,
                      stage_events, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_gauss_blur(const float* in, int32_t in_pitch, float* out, int32_t out_pitch, int32_t H, int32_t W,
                      const float* weights, int32_t radius, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(in && out && weights, "NULL pointer argument");
    PYSIFT_CHECK_ARG(H > 0 && W > 0 && in_pitch >= W && out_pitch >= W, "bad sizes");
    PYSIFT_CHECK_ARG(radius >= 0 && radius <= PYSIFT_MAX_RADIUS, "radius %d outside 0..%d", radius,
                     PYSIFT_MAX_RADIUS);
    static thread_local BlurArgs a;
    memset(&a, 0, sizeof(a));
    a.in = in;
    a.in_pitch = in_pitch;
    a.step = 1;
    a.out = out;
    a.out_pitch = out_pitch;
    a.H = H;
    a.W = W;
    return launch_blur(a, radius, weights, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_set_blur_tile_rows(int32_t rows) {
    int v = -1;
    for (int k = 0; k < BLUR_NV; ++k)
        if (rows == BLUR_THS[k]) v = k;
    PYSIFT_CHECK_ARG(rows == 0 || v >= 0, "tile rows %d: 0 (automatic), 16, 32 or 40", rows);
    g_blur_forced.store(rows == 0 ? -1 : v, std::memory_order_relaxed);
    return PYSIFT_OK;
}

int pysift_blur_size_class(int32_t H, int32_t W) { return (H > 0 && W > 0) ? blur_size_class(H, W) : -1; }

int pysift_set_blur_tile_table(const int32_t* rows, int32_t n) {
    constexpr int N = (BLUR_PAIR_MAX_R + 1) * BLUR_SIZE_CLASSES;
    PYSIFT_CHECK_ARG(n == 0 || (rows && n == N), "the table has %d entries (0 clears it)", N);
    int v[N];
    for (int i = 0; i < n; ++i) {
        v[i] = -1;
        for (int k = 0; k < BLUR_NV; ++k)
            if (rows[i] == BLUR_THS[k]) v[i] = k;
        PYSIFT_CHECK_ARG(rows[i] == 0 || v[i] >= 0, "entry %d: tile rows %d: 0 (rule), 16, 32 or 40", i, rows[i]);
    }
    blur_table_init();
    for (int i = 0; i < N; ++i)
        g_blur_table[i / BLUR_SIZE_CLASSES][i % BLUR_SIZE_CLASSES].store(n ? v[i] : -1, std::memory_order_relaxed);
    return PYSIFT_OK;
}

int pysift_zoom2x_u8(const uint8_t* gray, int32_t H, int32_t W, int64_t pitch_bytes, int32_t fp16_round,
                     double* coef, float* out, int32_t out_pitch, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(gray && coef && out, "NULL pointer argument");
    PYSIFT_CHECK_ARG(H > 0 && W > 0 && pitch_bytes >= W && out_pitch >= 2 * W, "bad sizes");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    return launch_zoom2x(gray, H, W, pitch_bytes, fp16_round, coef, out, out_pitch, st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of pysift_zoom2x_u8.
//
// Some callers cannot allocate device memory at the call site: for example a
// plugin loaded into a host application that owns the whole device heap and
// forbids cudaMalloc inside plugins, or code that runs under a fixed device
// memory budget with no allocator handle to pass in.  For them this entry
// point keeps the spline-coefficient scratch in a file-scope device array of
// PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS doubles (8 MiB), which every GPU that
// loads the library holds until the process exits.
//
// Host code cannot pass g_zoom2x_scratch to a kernel directly (in host code
// the name is a host-side stand-in, not a device address), so the device
// address is looked up with cudaGetSymbolAddress once per device, on the
// first call made with that device current, and cached.
// ---------------------------------------------------------------------------
namespace pysift {

static __device__ __align__(256) double g_zoom2x_scratch[PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS];

static int zoom2x_scratch_ptr(double** out) {
    constexpr int MAX_DEVICES = 64;
    static std::mutex mu;
    static double* ptrs[MAX_DEVICES] = {nullptr};
    int dev = 0;
    PYSIFT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) {
        set_error("device ordinal %d not supported by the allocation-free entry point", dev);
        return PYSIFT_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_zoom2x_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error("cudaGetSymbolAddress(g_zoom2x_scratch) on device %d failed: %s", dev,
                      cudaGetErrorString(e));
            return PYSIFT_ERR_CUDA;
        }
        ptrs[dev] = static_cast<double*>(p);
    }
    *out = ptrs[dev];
    return PYSIFT_OK;
}

}  // namespace pysift

extern "C" int pysift_zoom2x_u8_noalloc(const uint8_t* gray, int32_t H, int32_t W, int64_t pitch_bytes,
                                        int32_t fp16_round, float* out, int32_t out_pitch,
                                        pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(gray && out, "NULL pointer argument");
    PYSIFT_CHECK_ARG(H > 0 && W > 0 && pitch_bytes >= W && out_pitch >= 2 * W, "bad sizes");
    if ((int64_t)H * W > (int64_t)PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS) {
        set_error("pysift_zoom2x_u8_noalloc: %dx%d = %lld pixels exceeds the fixed scratch of %d pixels; "
                  "use pysift_zoom2x_u8 with caller-provided scratch",
                  H, W, (long long)H * W, (int)PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS);
        return PYSIFT_ERR_CAPACITY;
    }
    double* coef = nullptr;
    int rc = zoom2x_scratch_ptr(&coef);
    if (rc) return rc;
    // Every scratch element the kernels read is written earlier in this same
    // call (k_prefilter_cols fills all H*W coefficients), so nothing needs
    // clearing between calls.
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    return launch_zoom2x(gray, H, W, pitch_bytes, fp16_round, coef, out, out_pitch, st);
}
