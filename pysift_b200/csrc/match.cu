// match.cu -- brute-force ratio-test matching on the 5th-generation tensor cores.
//
// One CTA computes a 128 x 128 tile of S = A * B^T with tcgen05.mma
// (kind::f16, fp16 or bf16 operands staged in shared memory in the
// no-swizzle K-major core-matrix layout, fp32 accumulators in tensor memory),
// then reduces the tile in its epilogue to per-row and per-column top-2
// candidates.  A second kernel merges the per-tile candidates, applies the
// ratio test in both directions and keeps mutual matches
// (pysift/core.py:2574-2701, 2840-2940).
//
// Two scoring modes share the kernel:
//   SIM_F16   reference semantics: fp16 inputs, the fp32 tile rounded to fp16
//             (torch.mm under fp16 autocast, core.py:2604-2605), larger is better,
//             d^2 = max(0, 2 - 2 s), pass iff d2^2 > 1e-10 and d1^2 < r^2 d2^2 in float32.
//   DIST_BF16 exact L2 on uint8-valued descriptors: bf16 holds 0..255 exactly and
//             every partial sum of 128 products stays below 2^24, so the fp32
//             accumulator is the exact integer dot product; d^2 = |a|^2 + |b|^2 - 2 a.b,
//             smaller is better, pass iff d2^2 > 0 and d1^2 < r^2 d2^2 (exact).
// Ties are broken towards the lower index in every direction.
#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include <cuda_bf16.h>

namespace pysift {

constexpr int MT = 128;           // tile rows (queries) = UMMA M
constexpr int NT = 128;           // tile cols (train)   = UMMA N
constexpr int MATCH_THREADS = 128;
constexpr unsigned SPIN_LIMIT = 1u << 26;  // bounded wait on the MMA barrier

enum MatchMode { SIM_F16 = 0, DIST_BF16 = 1 };

struct Cand {  // top-2, "larger key is better", ties to the lower index
    float k1, k2;
    int i1, i2;
};

__device__ __forceinline__ bool better(float ka, int ia, float kb, int ib) {
    return ka > kb || (ka == kb && ia < ib);
}

__device__ __forceinline__ void cand_push(Cand& c, float k, int i) {
    if (better(k, i, c.k1, c.i1)) {
        c.k2 = c.k1;
        c.i2 = c.i1;
        c.k1 = k;
        c.i1 = i;
    } else if (better(k, i, c.k2, c.i2)) {
        c.k2 = k;
        c.i2 = i;
    }
}

__device__ __forceinline__ Cand cand_empty() {
    Cand c;
    c.k1 = c.k2 = -INFINITY;
    c.i1 = c.i2 = 0x7fffffff;
    return c;
}

// byte offset of 16-byte chunk c (8 elements along K) of row r in the
// no-swizzle K-major layout: core matrices of 8 rows x 16 bytes, adjacent
// along K at 128 bytes (LBO), 8-row groups at K/8 * 128 bytes (SBO).
__device__ __forceinline__ uint32_t core_off(int r, int c, int kchunks) {
    return (uint32_t)(((r >> 3) * kchunks + c) * 128 + (r & 7) * 16);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    // base offset 0, legacy LBO mode, layout type 0 = SWIZZLE_NONE
    return d;
}

// kind::f16 instruction descriptor: D = f32, A/B = f16 (0) or bf16 (1),
// both K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(int ab_format) {
    return (1u << 4) | ((uint32_t)ab_format << 7) | ((uint32_t)ab_format << 10) | ((uint32_t)(NT >> 3) << 17) |
           ((uint32_t)(MT >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

struct MatchTileArgs {
    const uint16_t* a;  // n_a x K (fp16 or bf16 bits), row stride K
    const uint16_t* b;  // n_b x K
    int n_a, n_b, K;
    const int* norm_a;  // DIST_BF16: |a|^2 per row
    const int* norm_b;
    Cand* row_part;     // [n_a][n_tiles_b]
    Cand* col_part;     // [n_b][n_tiles_a]
    int* error;         // set when the MMA wait gives up
};

template <int MODE, int K>
__global__ void __launch_bounds__(MATCH_THREADS) k_match_tile(const MatchTileArgs args) {
    constexpr int KC = K / 8;                  // 16-byte chunks per row
    constexpr uint32_t TILE_BYTES = MT * K * 2;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem;
    uint8_t* sB = smem + TILE_BYTES;
    float* sT = reinterpret_cast<float*>(smem);  // reused after the MMA: 128 x 129 floats
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int ta = blockIdx.y, tb = blockIdx.x;
    const int row0 = ta * MT, col0 = tb * NT;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
    }
    // stage the operand tiles (rows beyond n_a / n_b are zero)
    for (int q = tid; q < MT * KC; q += MATCH_THREADS) {
        const int r = q / KC, c = q - r * KC;
        uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
        if (row0 + r < args.n_a) va = *reinterpret_cast<const uint4*>(args.a + (size_t)(row0 + r) * K + c * 8);
        if (col0 + r < args.n_b) vb = *reinterpret_cast<const uint4*>(args.b + (size_t)(col0 + r) * K + c * 8);
        *reinterpret_cast<uint4*>(sA + core_off(r, c, KC)) = va;
        *reinterpret_cast<uint4*>(sB + core_off(r, c, KC)) = vb;
    }
    // make the generic-proxy shared-memory writes visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    if (tid == 0) {
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
        constexpr uint32_t idesc = umma_idesc(MODE == SIM_F16 ? 0 : 1);
#pragma unroll
        for (int s = 0; s < K / 16; ++s) {
            const uint64_t da = umma_desc(a0 + s * 256, 128, KC * 128);
            const uint64_t db = umma_desc(b0 + s * 256, 128, KC * 128);
            const uint32_t acc = s > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(&mbar)));
    }
    // bounded wait for the MMAs (phase 0)
    {
        unsigned done = 0, spins = 0;
        while (!done) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(&mbar)), "r"(0));
            if (!done && ++spins > SPIN_LIMIT) {
                s_fail = 1;
                break;
            }
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    const bool ok = (s_fail == 0);
    if (!ok && tid == 0) atomicExch(args.error, 1);

    // epilogue: thread = tile row (TMEM lane 32*warp + lane)
    const int row = row0 + tid;
    Cand rc = cand_empty();
    const int na_r = (MODE == DIST_BF16 && row < args.n_a) ? args.norm_a[row] : 0;
#pragma unroll
    for (int chunk = 0; chunk < NT / 32; ++chunk) {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(chunk * 32);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const int col = col0 + chunk * 32 + j;
            float key;
            if (MODE == SIM_F16) {
                key = __half2float(__float2half_rn(__uint_as_float(v[j])));
            } else {
                const int dot = (int)__uint_as_float(v[j]);
                const int nb = col < args.n_b ? args.norm_b[col] : 0;
                key = -(float)(na_r + nb - 2 * dot);
            }
            if (!ok) key = -INFINITY;
            sT[tid * (NT + 1) + chunk * 32 + j] = key;
            if (col < args.n_b) cand_push(rc, key, col);
        }
    }
    const int n_tb = gridDim.x, n_ta = gridDim.y;
    if (row < args.n_a) args.row_part[(size_t)row * n_tb + tb] = rc;
    __syncthreads();
    // column candidates: thread = tile column
    {
        const int col = col0 + tid;
        Cand cc = cand_empty();
        const int nrows = min(MT, args.n_a - row0);
        for (int r = 0; r < nrows; ++r) cand_push(cc, sT[r * (NT + 1) + tid], row0 + r);
        if (col < args.n_b) args.col_part[(size_t)col * n_ta + ta] = cc;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT));
}

// Merge per-tile candidates of one side, ratio test.  best/pass per element.
template <int MODE>
__global__ void k_match_merge(const Cand* __restrict__ part, int n, int ntiles, float ratio_sq, int* __restrict__ best,
                              int* __restrict__ pass, float* __restrict__ dist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Cand c = cand_empty();
    for (int t = 0; t < ntiles; ++t) {
        const Cand p = part[(size_t)i * ntiles + t];
        if (p.i1 != 0x7fffffff) cand_push(c, p.k1, p.i1);
        if (p.i2 != 0x7fffffff) cand_push(c, p.k2, p.i2);
    }
    int ok = 0;
    float d = 0.0f;
    if (c.i2 != 0x7fffffff) {
        if (MODE == SIM_F16) {
            // pysift/core.py:2676-2680 (float32)
            float db = 2.0f - 2.0f * c.k1;
            float ds = 2.0f - 2.0f * c.k2;
            db = db < 0.0f ? 0.0f : db;
            ds = ds < 0.0f ? 0.0f : ds;
            ok = (ds > 1e-10f) && (db < ratio_sq * ds);
            d = sqrtf(db);
        } else {
            const double d1 = -(double)c.k1, d2 = -(double)c.k2;  // exact integers
            ok = (d2 > 0.0) && (d1 < (double)ratio_sq * d2);
            d = sqrtf((float)d1);
        }
    }
    best[i] = c.i1 == 0x7fffffff ? -1 : c.i1;
    pass[i] = ok;
    if (dist) dist[i] = d;
}

// Mutual matches in query order: fwd[i] = j passes, bwd[j] = i passes.
__global__ void __launch_bounds__(1024) k_match_mutual(const int* __restrict__ fbest, const int* __restrict__ fpass,
                                                       const float* __restrict__ fdist, const int* __restrict__ bbest,
                                                       const int* __restrict__ bpass, int n1, int2* __restrict__ pairs,
                                                       float* __restrict__ pdist, int* __restrict__ count) {
    __shared__ int sh[33];
    int base = 0;
    for (int c0 = 0; c0 < n1; c0 += blockDim.x) {
        const int i = c0 + threadIdx.x;
        int keep = 0, j = -1;
        if (i < n1 && fpass[i]) {
            j = fbest[i];
            keep = (j >= 0 && bpass[j] && bbest[j] == i) ? 1 : 0;
        }
        int tot;
        const int pos = base + block_excl_scan(keep, &tot, sh);
        if (keep) {
            pairs[pos] = make_int2(i, j);
            pdist[pos] = fdist[i];
        }
        base += tot;
    }
    if (threadIdx.x == 0) *count = base;
}

__global__ void k_row_norms_u8(const uint8_t* __restrict__ d, int n, int D, int* __restrict__ norms,
                               uint16_t* __restrict__ bf) {
    const int i = blockIdx.x * blockDim.y + threadIdx.y;
    if (i >= n) return;
    int s = 0;
    for (int k = threadIdx.x; k < D; k += 32) {
        const int v = d[(size_t)i * D + k];
        s += v * v;
        bf[(size_t)i * D + k] = __bfloat16_as_ushort(__float2bfloat16_rn((float)v));
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL_MASK, s, o);
    if (threadIdx.x == 0) norms[i] = s;
}

template <int MODE, int K>
static int launch_tiles(const MatchTileArgs& a, cudaStream_t st) {
    // operand tiles, later reused for the 128 x 129 float key tile
    const size_t smem_launch = std::max(2 * (size_t)MT * K * 2, (size_t)MT * (NT + 1) * 4);
    PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_match_tile<MODE, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_launch));
    dim3 grid(ceil_div(a.n_b, NT), ceil_div(a.n_a, MT));
    k_match_tile<MODE, K><<<grid, MATCH_THREADS, smem_launch, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_match_tile");
    return PYSIFT_OK;
}

struct MatchLayout {
    size_t off_rowp, off_colp, off_fbest, off_fpass, off_fdist, off_bbest, off_bpass, off_bdist, off_err;
    size_t off_na, off_nb, off_bfa, off_bfb;
    size_t total;
};

static MatchLayout match_layout(int n1, int n2, int D, bool exact) {
    MatchLayout l;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t r = off;
        off = align_up(off + bytes, 256);
        return r;
    };
    const size_t ta = ceil_div(n1, MT), tb = ceil_div(n2, NT);
    l.off_rowp = take((size_t)n1 * tb * sizeof(Cand));
    l.off_colp = take((size_t)n2 * ta * sizeof(Cand));
    l.off_fbest = take((size_t)n1 * 4);
    l.off_fpass = take((size_t)n1 * 4);
    l.off_fdist = take((size_t)n1 * 4);
    l.off_bbest = take((size_t)n2 * 4);
    l.off_bpass = take((size_t)n2 * 4);
    l.off_bdist = take((size_t)n2 * 4);
    l.off_err = take(4);
    l.off_na = l.off_nb = l.off_bfa = l.off_bfb = 0;
    if (exact) {
        l.off_na = take((size_t)n1 * 4);
        l.off_nb = take((size_t)n2 * 4);
        l.off_bfa = take((size_t)n1 * D * 2);
        l.off_bfb = take((size_t)n2 * D * 2);
    }
    l.total = off;
    return l;
}

template <typename T>
static T* wsp(void* ws, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(ws) + off);
}

static int run_match(int mode, const uint16_t* a, int n1, const uint16_t* b, int n2, int D, float ratio_sq,
                     const MatchLayout& l, void* ws, int* fbest_out, int* fpass_out, int* bbest_out, int* bpass_out,
                     int32_t* pairs, float* pdist, int32_t* count, cudaStream_t st) {
    MatchTileArgs ta;
    ta.a = a;
    ta.b = b;
    ta.n_a = n1;
    ta.n_b = n2;
    ta.K = D;
    ta.norm_a = mode == DIST_BF16 ? wsp<int>(ws, l.off_na) : nullptr;
    ta.norm_b = mode == DIST_BF16 ? wsp<int>(ws, l.off_nb) : nullptr;
    ta.row_part = wsp<Cand>(ws, l.off_rowp);
    ta.col_part = wsp<Cand>(ws, l.off_colp);
    ta.error = wsp<int>(ws, l.off_err);
    PYSIFT_CUDA_TRY(cudaMemsetAsync(ta.error, 0, 4, st));
    int rc;
    if (mode == SIM_F16)
        rc = (D == 64) ? launch_tiles<SIM_F16, 64>(ta, st) : launch_tiles<SIM_F16, 128>(ta, st);
    else
        rc = (D == 64) ? launch_tiles<DIST_BF16, 64>(ta, st) : launch_tiles<DIST_BF16, 128>(ta, st);
    if (rc) return rc;
    int* fbest = fbest_out ? fbest_out : wsp<int>(ws, l.off_fbest);
    int* fpass = fpass_out ? fpass_out : wsp<int>(ws, l.off_fpass);
    int* bbest = bbest_out ? bbest_out : wsp<int>(ws, l.off_bbest);
    int* bpass = bpass_out ? bpass_out : wsp<int>(ws, l.off_bpass);
    float* fdist = wsp<float>(ws, l.off_fdist);
    float* bdist = wsp<float>(ws, l.off_bdist);
    const int ntb = ceil_div(n2, NT), nta = ceil_div(n1, MT);
    if (mode == SIM_F16) {
        k_match_merge<SIM_F16><<<ceil_div(n1, 256), 256, 0, st>>>(ta.row_part, n1, ntb, ratio_sq, fbest, fpass, fdist);
        PYSIFT_LAUNCH_CHECK("k_match_merge");
        k_match_merge<SIM_F16><<<ceil_div(n2, 256), 256, 0, st>>>(ta.col_part, n2, nta, ratio_sq, bbest, bpass, bdist);
    } else {
        k_match_merge<DIST_BF16><<<ceil_div(n1, 256), 256, 0, st>>>(ta.row_part, n1, ntb, ratio_sq, fbest, fpass,
                                                                    fdist);
        PYSIFT_LAUNCH_CHECK("k_match_merge");
        k_match_merge<DIST_BF16><<<ceil_div(n2, 256), 256, 0, st>>>(ta.col_part, n2, nta, ratio_sq, bbest, bpass,
                                                                    bdist);
    }
    PYSIFT_LAUNCH_CHECK("k_match_merge");
    k_match_mutual<<<1, 1024, 0, st>>>(fbest, fpass, fdist, bbest, bpass, n1, reinterpret_cast<int2*>(pairs), pdist,
                                       count);
    PYSIFT_LAUNCH_CHECK("k_match_mutual");
    return PYSIFT_OK;
}

}  // namespace pysift

using namespace pysift;

extern "C" {

int pysift_match_workspace_size(int32_t n1, int32_t n2, int32_t D, int32_t exact_u8, size_t* bytes) {
    PYSIFT_CHECK_ARG(bytes != nullptr, "bytes is NULL");
    PYSIFT_CHECK_ARG(n1 >= 0 && n2 >= 0 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    *bytes = match_layout(n1, n2, D, exact_u8 != 0).total;
    return PYSIFT_OK;
}

int pysift_match_fp16(const uint16_t* d1, int32_t n1, const uint16_t* d2, int32_t n2, int32_t D, float ratio,
                      void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                      int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist, int32_t* pair_count,
                      pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(d1 && d2 && workspace && pairs && pair_dist && pair_count, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n1 >= 1 && n2 >= 1 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    PYSIFT_CHECK_ARG((reinterpret_cast<uintptr_t>(d1) & 15) == 0 && (reinterpret_cast<uintptr_t>(d2) & 15) == 0,
                     "descriptor arrays must be 16-byte aligned");
    MatchLayout l = match_layout(n1, n2, D, false);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    const float ratio_sq = (float)((double)ratio * (double)ratio);
    return run_match(SIM_F16, d1, n1, d2, n2, D, ratio_sq, l, workspace, fwd_best, fwd_pass, bwd_best, bwd_pass, pairs,
                     pair_dist, pair_count, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_match_u8_exact(const uint8_t* d1, int32_t n1, const uint8_t* d2, int32_t n2, int32_t D, float ratio,
                          void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                          int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                          int32_t* pair_count, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(d1 && d2 && workspace && pairs && pair_dist && pair_count, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n1 >= 1 && n2 >= 1 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    MatchLayout l = match_layout(n1, n2, D, true);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint16_t* bfa = wsp<uint16_t>(workspace, l.off_bfa);
    uint16_t* bfb = wsp<uint16_t>(workspace, l.off_bfb);
    k_row_norms_u8<<<ceil_div(n1, 8), dim3(32, 8), 0, st>>>(d1, n1, D, wsp<int>(workspace, l.off_na), bfa);
    PYSIFT_LAUNCH_CHECK("k_row_norms_u8");
    k_row_norms_u8<<<ceil_div(n2, 8), dim3(32, 8), 0, st>>>(d2, n2, D, wsp<int>(workspace, l.off_nb), bfb);
    PYSIFT_LAUNCH_CHECK("k_row_norms_u8");
    const float ratio_sq = (float)((double)ratio * (double)ratio);
    return run_match(DIST_BF16, bfa, n1, bfb, n2, D, ratio_sq, l, workspace, fwd_best, fwd_pass, bwd_best, bwd_pass,
                     pairs, pair_dist, pair_count, st);
}

}  // extern "C"
