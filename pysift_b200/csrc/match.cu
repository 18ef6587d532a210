// match.cu -- brute-force ratio-test matching on the 5th-generation tensor cores.
//
// Matching runs as two row scans: queries against the train set (forward
// top-2) and the train set against the queries (backward top-2).  Both sets
// are first written in a tiled operand layout (128-row tiles of 16 KB slabs
// in the no-swizzle K-major core-matrix layout).  Each CTA of k_match_rows
// keeps a 128-row query tile resident in shared memory; a loader thread
// streams the train slabs into a ring with one bulk copy each, an MMA thread
// issues tcgen05.mma (kind::f16 / f8f6f4 / i8, fp32 or s32 accumulator in
// tensor memory, two accumulators of 128 columns) and eight warps reduce the
// finished accumulator, read back with tcgen05.ld (two warps per TMEM lane
// quadrant, each half of the tile's columns); mbarriers link the three roles.  Train tiles are split into segments so that the grid fills the
// SMs; a merge kernel combines the segments of each row and applies the ratio
// test; k_match_mutual keeps mutual matches (pysift/core.py:2574-2701,
// 2840-2940).
//
// The reduction works on 32-column chunks: a chunk's key is its largest
// column key (a tree of 31 max operations, no per-column index), and each
// row keeps the three best chunks in (key desc, first column asc) order with
// the first two chunks' positions (Top3 at chunk level).  The merge then
// recomputes the candidate chunks' columns exactly, one warp per row:
//   SIM_F16   reference semantics: fp16 inputs, the similarity rounded to fp16
//             (torch.mm under fp16 autocast, core.py:2604-2605), larger is better,
//             d^2 = max(0, 2 - 2 s), pass iff d2^2 > 1e-10 and d1^2 < r^2 d2^2 in float32.
//             The canonical similarity is the fp16 rounding (nearest, ties to
//             even) of the EXACT dot product.  The tensor cores' fp32
//             accumulation is within e = D 2^-21 |a| max|b| of it.  The merge
//             recomputes every column of the two best chunks exactly (float64
//             sums of the exact fp16 products: every partial sum is a multiple
//             of 2^-48 below 2^5 in magnitude for rows of norm <= 1, hence
//             exact in any order) and accepts the row when no column of the
//             other chunks can reach the exact second value
//             (fp16(third chunk key + e) <= second, and < best); the other rows
//             are recomputed over every column by k_match_recheck_f16.
//   DIST_U8   exact L2 on uint8 descriptors: kind::i8 with unsigned 8-bit
//             operands and an s32 accumulator gives the exact integer dot
//             product (below 128 * 255^2 < 2^24).  Rows rank train
//             entries by 2 a.b - |b|^2 (exact in fp32: |2 a.b| < 2^24), which orders
//             them as -|a - b|^2; d^2 = |a|^2 - key, pass iff d2^2 > 0 and
//             d1^2 < r^2 d2^2 (exact).  The merge recomputes the best chunk
//             from the uint8 rows (integer dot products): the first column
//             with the chunk's key is the best, the second key the larger of
//             the chunk's second and the next chunk's key.
//   SPLIT_FP8 the same keys through split-nibble e4m3 planes.
//   SIM_I8    int8 similarities divided by the row scales, per column (the
//             division does not commute with the maximum): column-level top-2.
// Ties are broken towards the lower index in every direction: a scan visits
// train entries in increasing index order and replaces the best only on a
// strictly larger key; segments merge in index order.
#include <algorithm>
#include <climits>
#include <cstdint>

#include "common.cuh"
#include <cuda_fp8.h>

namespace pysift {

constexpr int MT = 128;           // query rows per CTA = UMMA M = TMEM lanes
constexpr int NT = 128;           // train rows per tile = UMMA N
constexpr int MATCH_THREADS = 256;  // the scan's reducer threads: 2 warps per TMEM lane quadrant, each half the tile's columns
constexpr unsigned SPIN_LIMIT = 1u << 22;  // bounded waits on the pipeline barriers

enum MatchMode { SIM_F16 = 0, DIST_U8 = 1, SPLIT_FP8 = 2, SIM_I8 = 3 };

struct Top2 {  // best key and index, second-best key
    float k1, k2;
    int i1, pad;
};

// SIM_F16 scan state of one row: the best and second raw keys with their
// indices (order: larger key first, the lower index on equal keys) and the
// third-largest key of the columns seen.
struct Top3 {
    float k1, k2, k3;
    int i1, i2;
    int pad[3];
};

__device__ __forceinline__ void top3_init(Top3& t) {
    t.k1 = t.k2 = t.k3 = -INFINITY;
    t.i1 = t.i2 = 0x7fffffff;
}

// Column c with key x, visited in increasing column order within the state.
__device__ __forceinline__ void top3_push(Top3& t, float x, int c) {
    t.k3 = fmaxf(t.k3, fminf(x, t.k2));
    const bool g1 = x > t.k1, g2 = x > t.k2;
    t.i2 = g2 ? (g1 ? t.i1 : c) : t.i2;
    t.k2 = fmaxf(t.k2, fminf(x, t.k1));
    t.i1 = g1 ? c : t.i1;
    t.k1 = fmaxf(t.k1, x);
}

__device__ __forceinline__ bool key_before(float ka, int ia, float kb, int ib) {
    return ka > kb || (ka == kb && ia < ib);
}

// Union of two states over disjoint column sets (in any index relation):
// the two first entries in (key desc, index asc) order, and the third-largest
// key of the union.
__device__ __forceinline__ void top3_merge(Top3& a, const Top3& b) {
    Top3 r;
    if (key_before(a.k1, a.i1, b.k1, b.i1)) {
        r.k1 = a.k1;
        r.i1 = a.i1;
        if (key_before(a.k2, a.i2, b.k1, b.i1)) {
            r.k2 = a.k2;
            r.i2 = a.i2;
            r.k3 = fmaxf(a.k3, b.k1);
        } else {
            r.k2 = b.k1;
            r.i2 = b.i1;
            r.k3 = fmaxf(a.k2, b.k2);
        }
    } else {
        r.k1 = b.k1;
        r.i1 = b.i1;
        if (key_before(b.k2, b.i2, a.k1, a.i1)) {
            r.k2 = b.k2;
            r.i2 = b.i2;
            r.k3 = fmaxf(b.k3, a.k1);
        } else {
            r.k2 = a.k1;
            r.i2 = a.i1;
            r.k3 = fmaxf(a.k2, b.k2);
        }
    }
    a.k1 = r.k1;
    a.k2 = r.k2;
    a.k3 = r.k3;
    a.i1 = r.i1;
    a.i2 = r.i2;
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

// kind::i8 instruction descriptor: D = s32 (2), A/B = signed (1) or
// unsigned (0) 8-bit, both K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc_i8(bool is_signed) {
    return (2u << 4) | ((is_signed ? 1u : 0u) << 7) | ((is_signed ? 1u : 0u) << 10) | ((uint32_t)(NT >> 3) << 17) |
           ((uint32_t)(MT >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Tiled operand layout (global memory and shared memory alike).  A tile is
// 128 rows of RB bytes; it is stored as RB / (16 SW) slabs of SW 16-byte
// chunks along K (SW = min(RB / 16, 8)), each slab in the no-swizzle K-major
// core-matrix layout: core matrices of 8 rows x 16 bytes, adjacent along K
// at 128 bytes (LBO), 8-row groups at SW * 128 bytes (SBO).  A slab is one
// contiguous block, so one bulk copy moves it; rows past the set are zero.
template <int RB>
struct TileGeom {
    static constexpr int KC = RB / 16;              // 16-byte chunks per row
    static constexpr int SW = KC < 8 ? KC : 8;      // chunks per slab
    static constexpr int NSL = KC / SW;             // slabs per tile
    static constexpr uint32_t SLAB = MT * SW * 16;  // bytes per slab
    static constexpr uint32_t TILE = MT * RB;       // bytes per tile
    // slabs in the shared-memory ring: query tile + ring within 96 KB
    static constexpr int NS = (96 * 1024 - (int)TILE) / (int)SLAB;
    static_assert(NS >= 2, "ring too small");
};

// Byte offset of 16-byte chunk c of row r (RB-byte rows) in the tiled layout.
__host__ __device__ __forceinline__ size_t tiled_off(int r, int c, int RB) {
    const int KC = RB / 16, SW = KC < 8 ? KC : 8;
    const int rr = r & (MT - 1), slab = c / SW, cs = c - slab * SW;
    return (size_t)(r / MT) * MT * RB + (size_t)slab * MT * SW * 16 + (size_t)(((rr >> 3) * SW + cs) * 128 + (rr & 7) * 16);
}

// Row-major rows of RB bytes (16-byte aligned) into the tiled layout, rows
// n .. n_pad-1 zero.  One thread per 16-byte chunk.
__global__ void k_tile_rows(const uint8_t* __restrict__ src, int n, int n_pad, int RB, uint8_t* __restrict__ dst) {
    const int KC = RB / 16;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)n_pad * KC) return;
    const int r = (int)(q / KC), c = (int)(q - (long long)r * KC);
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r < n) v = *reinterpret_cast<const uint4*>(src + (size_t)r * RB + (size_t)c * 16);
    *reinterpret_cast<uint4*>(dst + tiled_off(r, c, RB)) = v;
}

// Bounded mbarrier wait that also gives up once another role of the CTA has
// raised the abort flag.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int* abort_flag) {
    uint32_t done = 0;
    for (unsigned spins = 0; spins < SPIN_LIMIT; ++spins) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (abort_flag && *abort_flag) return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// One contiguous global -> shared bulk copy into this CTA's own shared
// memory, completing on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Arrives on bar once every tcgen05.mma this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

struct RowScanArgs {
    const uint8_t* q;    // n_q rows of RB bytes (fp16 / uint8 / int8 / e4m3 codes), tiled
    const uint8_t* t;    // n_t rows of RB bytes
    int n_q, n_t;
    const float* norm_t;   // SPLIT_FP8: |t|^2 per train row (exact in float32), padded to whole tiles
    const int* norm_ti;    // DIST_U8: |t|^2 per train row as int32, padded to whole tiles
    const float* scale_q;  // SIM_I8: quantisation scale per query row
    const float* scale_t;  //         and per train row
    int seg_tiles;       // train tiles per segment (blockIdx.y)
    void* part;          // [n_q][gridDim.y] Top3 (chunk level; SIM_I8: Top2 of columns)
    int* error;          // set when an MMA wait gives up
};

// SIM_I8 running top-2 of one 32-column chunk: even columns into (k1, k2,
// i1), odd columns into (m1, m2, j1) (two independent chains); each partial
// visits its columns in increasing index order and replaces its best only
// on a strictly larger key.
__device__ __forceinline__ void scan_chunk_i8(const uint32_t (&v)[32], int col0, int lim, int nb_lane, float sq,
                                              float& k1, float& k2, int& i1, float& m1, float& m2, int& j1) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        // torch._int_mm(...).float() / (s1 * s2.T) (pysift/core.py:2908-2910):
        // the int32 dot product is exact (|.| < 2^24, so exact in float32)
        const float st = __int_as_float(__shfl_sync(FULL_MASK, nb_lane, j));
        float key = __fdiv_rn((float)(int)v[j], __fmul_rn(sq, st));
        if (j >= lim) key = -INFINITY;
        if (j & 1) {
            m2 = fmaxf(m2, fminf(key, m1));
            j1 = key > m1 ? col0 + j : j1;
            m1 = fmaxf(m1, key);
        } else {
            k2 = fmaxf(k2, fminf(key, k1));
            i1 = key > k1 ? col0 + j : i1;
            k1 = fmaxf(k1, key);
        }
    }
}

// Largest key of a 32-column chunk (SIM_F16: the raw fp32 accumulator;
// DIST_U8 / SPLIT_FP8: 2 a.b - |b|^2, exact), columns >= lim excluded.
// A pairwise tree of 31 max operations; the chunk's position in the row is
// kept by the caller, so no per-column index is tracked.
template <int MODE>
__device__ __forceinline__ float chunk_max(uint32_t (&v)[32], int lim, const float* __restrict__ nb,
                                           const int* __restrict__ nbi) {
    if constexpr (MODE == DIST_U8) {
        // integer keys 2 a.b - |b|^2 from the s32 accumulator (|key| < 2^24):
        // an integer max tree, one conversion per chunk (exact)
        int y[32];
        const int4* n4 = reinterpret_cast<const int4*>(nbi);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int4 n = n4[q];  // the same address in every lane: one broadcast
            y[4 * q + 0] = 2 * (int)v[4 * q + 0] - n.x;
            y[4 * q + 1] = 2 * (int)v[4 * q + 1] - n.y;
            y[4 * q + 2] = 2 * (int)v[4 * q + 2] - n.z;
            y[4 * q + 3] = 2 * (int)v[4 * q + 3] - n.w;
        }
        if (lim < 32) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j >= lim) y[j] = INT_MIN;
        }
#pragma unroll
        for (int w = 16; w > 0; w >>= 1) {
#pragma unroll
            for (int j = 0; j < w; ++j) y[j] = max(y[j], y[j + w]);
        }
        return y[0] == INT_MIN ? -INFINITY : (float)y[0];
    }
    float x[32];
    if constexpr (MODE == SIM_F16) {
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = __uint_as_float(v[j]);
    } else {
        const float4* n4 = reinterpret_cast<const float4*>(nb);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 n = n4[q];  // the same address in every lane: one broadcast
            // 2 a.b and |b|^2 are integers below 2^24: the fused result is exact
            x[4 * q + 0] = __fmaf_rn(2.0f, __uint_as_float(v[4 * q + 0]), -n.x);
            x[4 * q + 1] = __fmaf_rn(2.0f, __uint_as_float(v[4 * q + 1]), -n.y);
            x[4 * q + 2] = __fmaf_rn(2.0f, __uint_as_float(v[4 * q + 2]), -n.z);
            x[4 * q + 3] = __fmaf_rn(2.0f, __uint_as_float(v[4 * q + 3]), -n.w);
        }
    }
    if (lim < 32) {  // the last tile only; the same in every lane
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (j >= lim) x[j] = -INFINITY;
    }
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
#pragma unroll
        for (int j = 0; j < w; ++j) x[j] = fmaxf(x[j], x[j + w]);
    }
    return x[0];
}

// Top-2 of the union of two disjoint column sets: the best is the larger
// best (the lower index on equal keys, i.e. its first occurrence in index
// order), the second the largest of the smaller best and the two seconds --
// the result a single scan in index order would give.
__device__ __forceinline__ void top2_merge(float& k1, float& k2, int& i1, float bk1, float bk2, int bi1) {
    k2 = fmaxf(fmaxf(k2, bk2), fminf(k1, bk1));
    i1 = bk1 > k1 ? bi1 : (bk1 == k1 ? min(i1, bi1) : i1);
    k1 = fmaxf(k1, bk1);
}

// Warp roles of k_match_rows: warps 0..7 reduce (two per TMEM lane
// quadrant, each half of a tile's columns), warp 8 lane 0 loads (bulk
// copies of the query tile and of the train slabs into a ring of NS slabs),
// warp 9 lane 0 issues the MMAs.  Barriers: full[s] (slab landed), empty[s]
// (the MMAs reading slab s completed), acc_full[a] (accumulator a holds a
// finished tile), acc_empty[a] (the reducers have read accumulator a).  No
// block-wide barrier in the loop; every wait is bounded and gives up once a
// role raised the abort flag (the scan then reports an error).
constexpr int EPI_WARPS = MATCH_THREADS / 32;
constexpr int SCAN_THREADS = MATCH_THREADS + 64;

template <int MODE, int RB>
__global__ void __launch_bounds__(SCAN_THREADS, 2) k_match_rows(const RowScanArgs args) {
    using G = TileGeom<RB>;
    constexpr int NS = G::NS;
    // SIM_F16, DIST_U8, SPLIT_FP8: chunk-level state (the key of each
    // 32-column chunk is its largest); SIM_I8: column-level top-2
    constexpr bool CHUNKED = MODE != SIM_I8;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sQ = smem;                // the query tile (NSL slabs)
    uint8_t* sRing = smem + G::TILE;   // NS train slabs
    __shared__ __align__(8) uint64_t bar_full[NS], bar_empty[NS], bar_acc_full[2], bar_acc_empty[2], bar_q, bar_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int s_abort;
    __shared__ Top3 s_half[MT];  // Top2 in the first 16 bytes for SIM_I8

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n_tt = (args.n_t + NT - 1) / NT;
    const int t_begin = blockIdx.y * args.seg_tiles;
    const int nt = min(n_tt, t_begin + args.seg_tiles) - t_begin;  // >= 1 by construction

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(2 * NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int k = 0; k < NS; ++k) {
            mbar_init(&bar_full[k], 1);
            mbar_init(&bar_empty[k], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&bar_acc_full[k], 1);
            mbar_init(&bar_acc_empty[k], EPI_WARPS);
        }
        mbar_init(&bar_q, 1);
        mbar_init(&bar_done, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    auto give_up = [&]() {
        s_abort = 1;
        atomicExch(args.error, 1);
    };

    if (warp == EPI_WARPS) {
        // ---- loader ----
        if (lane == 0) {
            mbar_expect_tx(&bar_q, G::TILE);
            bulk_load(sQ, args.q + (size_t)blockIdx.x * G::TILE, G::TILE, &bar_q);
            int issued = 0;  // slabs
            const int total = nt * G::NSL;
            for (int k = 0; k < total; ++k) {
                const int sl = k % NS;
                if (k >= NS && !mbar_wait_bounded(&bar_empty[sl], (uint32_t)(((k / NS) - 1) & 1), &s_abort)) {
                    give_up();
                    break;
                }
                const int p = k / G::NSL, j = k - p * G::NSL;
                mbar_expect_tx(&bar_full[sl], G::SLAB);
                bulk_load(sRing + (size_t)sl * G::SLAB, args.t + (size_t)(t_begin + p) * G::TILE + (size_t)j * G::SLAB,
                          G::SLAB, &bar_full[sl]);
                ++issued;
            }
            // the copies in flight land in this CTA's shared memory: let the
            // last NS of them finish (bounded) before the CTA can exit
            mbar_wait_bounded(&bar_q, 0u, nullptr);
            for (int k = max(0, issued - NS); k < issued; ++k)
                mbar_wait_bounded(&bar_full[k % NS], (uint32_t)((k / NS) & 1), nullptr);
        }
    } else if (warp == EPI_WARPS + 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            constexpr uint32_t idesc =
                MODE == SIM_I8 ? umma_idesc_i8(true) : MODE == DIST_U8 ? umma_idesc_i8(false) : umma_idesc(0);
            bool ok = mbar_wait_bounded(&bar_q, 0u, &s_abort);
            int k = 0;  // slabs consumed
            for (int p = 0; ok && p < nt; ++p) {
                const int a = p & 1;
                if (p >= 2 && !mbar_wait_bounded(&bar_acc_empty[a], (uint32_t)(((p - 2) >> 1) & 1), &s_abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(a * NT);
                for (int j = 0; j < G::NSL; ++j, ++k) {
                    const int sl = k % NS;
                    if (!mbar_wait_bounded(&bar_full[sl], (uint32_t)((k / NS) & 1), &s_abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t a0 = smem_u32(sQ + (size_t)j * G::SLAB), b0 = smem_u32(sRing + (size_t)sl * G::SLAB);
                    // one MMA covers 32 bytes of K: two core matrices
#pragma unroll
                    for (int u = 0; u < G::SW / 2; ++u) {
                        const uint64_t da = umma_desc(a0 + u * 256, 128, G::SW * 128);
                        const uint64_t db = umma_desc(b0 + u * 256, 128, G::SW * 128);
                        const uint32_t acc = (j > 0 || u > 0) ? 1u : 0u;
                        if (MODE == SIM_I8 || MODE == DIST_U8)
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                                "l"(da), "l"(db), "r"(idesc), "r"(acc));
                        else if (MODE == SPLIT_FP8)
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                                "l"(da), "l"(db), "r"(idesc), "r"(acc));
                        else
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                                "l"(da), "l"(db), "r"(idesc), "r"(acc));
                    }
                    umma_commit(&bar_empty[sl]);  // the slab is free once these MMAs complete
                }
                if (!ok) break;
                umma_commit(&bar_acc_full[a]);
            }
            if (!ok) give_up();
            // every MMA issued has completed before the tensor memory is released
            umma_commit(&bar_done);
            mbar_wait_bounded(&bar_done, 0u, nullptr);
        }
    } else {
        // ---- reducers ----
        const int quad = warp & 3, half = warp >> 2;  // TMEM lane quadrant, column half of each tile
        const int rloc = quad * 32 + lane;            // this thread's query row in the block
        const int q0 = blockIdx.x * MT;
        const float sq = (MODE == SIM_I8 && q0 + rloc < args.n_q) ? args.scale_q[q0 + rloc] : 1.0f;
        float k1 = -INFINITY, k2 = -INFINITY, m1 = -INFINITY, m2 = -INFINITY;
        int i1 = 0x7fffffff, j1 = 0x7fffffff;
        Top3 tc;  // chunk-level state (CHUNKED)
        top3_init(tc);
        bool fail = false;
        for (int p = 0; p < nt; ++p) {
            const int a = p & 1;
            if (!mbar_wait_bounded(&bar_acc_full[a], (uint32_t)((p >> 1) & 1), &s_abort)) {
                fail = true;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int tcol0 = (t_begin + p) * NT;
            const int lim_tile = args.n_t - tcol0;
            uint32_t v0[32], v1[32];
            const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * NT + half * 64);
#define PYSIFT_TMEM_LD32(V, ADDR)                                                                                 \
    asm volatile(                                                                                                 \
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "                                                                 \
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"                                                 \
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                \
        : "=r"(V[0]), "=r"(V[1]), "=r"(V[2]), "=r"(V[3]), "=r"(V[4]), "=r"(V[5]), "=r"(V[6]), "=r"(V[7]),        \
          "=r"(V[8]), "=r"(V[9]), "=r"(V[10]), "=r"(V[11]), "=r"(V[12]), "=r"(V[13]), "=r"(V[14]), "=r"(V[15]), \
          "=r"(V[16]), "=r"(V[17]), "=r"(V[18]), "=r"(V[19]), "=r"(V[20]), "=r"(V[21]), "=r"(V[22]),           \
          "=r"(V[23]), "=r"(V[24]), "=r"(V[25]), "=r"(V[26]), "=r"(V[27]), "=r"(V[28]), "=r"(V[29]),           \
          "=r"(V[30]), "=r"(V[31])                                                                                \
        : "r"(ADDR))
            PYSIFT_TMEM_LD32(v0, taddr);
            PYSIFT_TMEM_LD32(v1, taddr + 32u);
#undef PYSIFT_TMEM_LD32
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            // the accumulator is read: hand it back to the MMA issuer
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_acc_empty[a]);
            const int c0 = tcol0 + half * 64;
            if constexpr (CHUNKED) {
                const float* nrm = MODE == SPLIT_FP8 ? args.norm_t + c0 : nullptr;
                const int* nri = MODE == DIST_U8 ? args.norm_ti + c0 : nullptr;
                top3_push(tc, chunk_max<MODE>(v0, lim_tile - half * 64, nrm, nri), c0);
                top3_push(tc, chunk_max<MODE>(v1, lim_tile - half * 64 - 32, nrm ? nrm + 32 : nullptr,
                                              nri ? nri + 32 : nullptr),
                          c0 + 32);
            } else {
                const int ca = c0 + lane, cb = c0 + 32 + lane;
                const int sa = __float_as_int(ca < args.n_t ? args.scale_t[ca] : 1.0f);
                const int sb = __float_as_int(cb < args.n_t ? args.scale_t[cb] : 1.0f);
                scan_chunk_i8(v0, c0, lim_tile - half * 64, sa, sq, k1, k2, i1, m1, m2, j1);
                scan_chunk_i8(v1, c0 + 32, lim_tile - half * 64 - 32, sb, sq, k1, k2, i1, m1, m2, j1);
            }
        }
        if (fail) give_up();
        // the two column halves of the row (named barrier over the reducers)
        const int row = q0 + rloc;
        if constexpr (CHUNKED) {
            if (half == 1) s_half[rloc] = tc;
            asm volatile("bar.sync 1, %0;" ::"n"(MATCH_THREADS) : "memory");
            if (half == 0 && !s_abort && row < args.n_q) {
                top3_merge(tc, s_half[rloc]);
                tc.pad[0] = tc.pad[1] = tc.pad[2] = 0;
                static_cast<Top3*>(args.part)[(size_t)row * gridDim.y + blockIdx.y] = tc;
            }
        } else {
            top2_merge(k1, k2, i1, m1, m2, j1);
            Top2* sh2 = reinterpret_cast<Top2*>(&s_half[rloc]);
            if (half == 1) {
                Top2 h;
                h.k1 = k1;
                h.k2 = k2;
                h.i1 = i1;
                h.pad = 0;
                *sh2 = h;
            }
            asm volatile("bar.sync 1, %0;" ::"n"(MATCH_THREADS) : "memory");
            if (half == 0 && !s_abort && row < args.n_q) {
                const Top2 h = *sh2;
                top2_merge(k1, k2, i1, h.k1, h.k2, h.i1);
                Top2 r;
                r.k1 = k1;
                r.k2 = k2;
                r.i1 = i1;
                r.pad = 0;
                static_cast<Top2*>(args.part)[(size_t)row * gridDim.y + blockIdx.y] = r;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * NT));
}

// SIM_I8: merge the column-level segments of one scan (in index order),
// ratio test on the similarities (pysift/core.py:2676-2680, float32).
__global__ void k_match_merge_i8(const Top2* __restrict__ part, int n, int nseg, float ratio_sq,
                                 int* __restrict__ best, int* __restrict__ pass, float* __restrict__ dist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float k1 = -INFINITY, k2 = -INFINITY;
    int i1 = 0x7fffffff;
    for (int s = 0; s < nseg; ++s) {
        const Top2 p = part[(size_t)i * nseg + s];
        k2 = fmaxf(fmaxf(k2, p.k2), fminf(p.k1, k1));
        i1 = p.k1 > k1 ? p.i1 : i1;
        k1 = fmaxf(k1, p.k1);
    }
    int ok = 0;
    float d = 0.0f;
    if (k2 > -INFINITY) {
        float db = 2.0f - 2.0f * k1;
        float ds = 2.0f - 2.0f * k2;
        db = db < 0.0f ? 0.0f : db;
        ds = ds < 0.0f ? 0.0f : ds;
        ok = (ds > 1e-10f) && (db < ratio_sq * ds);
        d = sqrtf(db);
    }
    best[i] = (k1 > -INFINITY) ? i1 : -1;
    pass[i] = ok;
    if (dist) dist[i] = d;
}

// Warp-wide top-2 of 64-bit keys (larger first): the best and the second
// (a second copy of the best counts), 0 = none.
__device__ __forceinline__ void warp_top2_u64(unsigned long long& kb, unsigned long long& ks) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(FULL_MASK, kb, o), os = __shfl_xor_sync(FULL_MASK, ks, o);
        ks = max(max(ks, os), min(kb, ob));
        kb = max(kb, ob);
    }
}

// Segments of one chunk-level scan, merged in segment order (every lane
// reads the same parts).
__device__ __forceinline__ Top3 shfl_xor_top3(const Top3& t, int o) {
    Top3 r;
    r.k1 = __shfl_xor_sync(FULL_MASK, t.k1, o);
    r.k2 = __shfl_xor_sync(FULL_MASK, t.k2, o);
    r.k3 = __shfl_xor_sync(FULL_MASK, t.k3, o);
    r.i1 = __shfl_xor_sync(FULL_MASK, t.i1, o);
    r.i2 = __shfl_xor_sync(FULL_MASK, t.i2, o);
    return r;
}

// The segments of one row merged by the whole warp: lane s loads parts s,
// s + 32, ... (all loads in flight at once), then a butterfly of top3_merge
// leaves the union in every lane.  The union's two first entries in
// (key desc, first column asc) order and its third key do not depend on the
// order of the merges.
__device__ __forceinline__ Top3 merge_parts(const Top3* __restrict__ part, int i, int nseg) {
    const int lane = threadIdx.x & 31;
    Top3 a;
    top3_init(a);
    for (int s_ = lane; s_ < nseg; s_ += 32) top3_merge(a, part[(size_t)i * nseg + s_]);
    for (int o = 16; o > 0; o >>= 1) top3_merge(a, shfl_xor_top3(a, o));
    return a;
}

// DIST_U8 / SPLIT_FP8: the best chunk of row i (the first chunk holding
// the row's largest key) recomputed exactly from the uint8 rows, one warp per
// row and one column per lane: the best column is the first in that chunk
// with the chunk's key, and the second key the larger of the chunk's second
// and the other chunks' largest (a.k2).  Keys 2 a.b - |b|^2 are exact
// integers on both sides, so the recomputed maximum equals a.k1; a mismatch
// (or a scan that gave up) leaves the row without a match.
__global__ void k_match_merge_u8(const Top3* __restrict__ part, int n, int nseg, float ratio_sq,
                                 const uint8_t* __restrict__ q, const uint8_t* __restrict__ t, int n_t, int D,
                                 const int* __restrict__ norm_q, const int* __restrict__ norm_t,
                                 const int* __restrict__ error, int* __restrict__ best, int* __restrict__ pass,
                                 float* __restrict__ dist) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n) return;
    const Top3 a = merge_parts(part, i, nseg);
    const bool bad = *error || !(a.k1 > -INFINITY) || a.i1 < 0 || a.i1 >= n_t;
    unsigned long long kb = 0, ks = 0;
    if (!bad) {
        const int c = a.i1 + lane;
        if (c < n_t) {
            const uint4* pq = reinterpret_cast<const uint4*>(q + (size_t)i * D);
            const uint4* pt = reinterpret_cast<const uint4*>(t + (size_t)c * D);
            unsigned acc = 0;
            for (int w = 0; w < D / 16; ++w) {
                const uint4 x = pq[w], y = pt[w];
                acc = __dp4a(x.x, y.x, acc);
                acc = __dp4a(x.y, y.y, acc);
                acc = __dp4a(x.z, y.z, acc);
                acc = __dp4a(x.w, y.w, acc);
            }
            const int key = 2 * (int)acc - norm_t[c];  // > -2^24
            // order-preserving bits of the key above the complemented column
            kb = ((unsigned long long)((unsigned)key ^ 0x80000000u) << 32) | (0xFFFFFFFFu - (unsigned)c);
        }
    }
    warp_top2_u64(kb, ks);
    if (lane != 0) return;
    auto key_of = [](unsigned long long k) { return (int)((unsigned)(k >> 32) ^ 0x80000000u); };
    int ok = 0, b = -1;
    float d = 0.0f;
    if (!bad && kb && (float)key_of(kb) == a.k1) {
        b = (int)(0xFFFFFFFFu - (unsigned)(kb & 0xFFFFFFFFu));
        float k2 = a.k2;  // the other chunks' largest key (exact)
        if (ks) k2 = fmaxf(k2, (float)key_of(ks));
        if (k2 > -INFINITY) {
            const double na = (double)norm_q[i];
            const double d1 = na - (double)a.k1, d2 = na - (double)k2;  // exact integers
            ok = (d2 > 0.0) && (d1 < (double)ratio_sq * d2);
            d = sqrtf((float)d1);
        }
    }
    best[i] = b;
    pass[i] = ok;
    if (dist) dist[i] = d;
}

// ---- SIM_F16: the canonical similarity fp16(exact a.b) ----

// The binary16 value nearest to x (ties to even) as a float, +0 for zero:
// x is scaled by a power of two to the integer grid of its binade (exact),
// rounded with rint (nearest, ties to even) and scaled back.
__device__ __forceinline__ float f16_round_f64(double x) {
    const double ax = fabs(x);
    if (!(ax < 65520.0)) return x < 0.0 ? -INFINITY : INFINITY;  // 65520: the tie that rounds up to 2^16
    int shift = 24;                                               // subnormal quantum 2^-24
    if (ax >= 6.103515625e-05) {                                  // 2^-14: normal, quantum 2^(E - 10)
        const int E = (int)((__double_as_longlong(ax) >> 52) & 0x7FF) - 1023;
        shift = 10 - E;
    }
    const double up = __longlong_as_double((long long)(1023 + shift) << 52);
    const double dn = __longlong_as_double((long long)(1023 - shift) << 52);
    return (float)(rint(x * up) * dn) + 0.0f;
}

// Exact dot product of two fp16 rows of D elements (16-byte aligned): each
// product is exact in fp32 (11-bit significands), and for rows of norm <= 1
// every float64 partial sum is exact (a multiple of 2^-48 below 2^5).
// Four partial sums (one per 16-byte word position mod 4) added at the end:
// exact in any order, so the result is the same as one running sum.
__device__ __forceinline__ double dot_f16_exact(const __half* a, const __half* b, int D) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const uint4* pa = reinterpret_cast<const uint4*>(a);
    const uint4* pb = reinterpret_cast<const uint4*>(b);
    for (int c = 0; c < D / 8; c += 4) {  // D / 8 is 8 or 16
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const uint4 x = pa[c + w], y = pb[c + w];
            const __half2* hx = reinterpret_cast<const __half2*>(&x);
            const __half2* hy = reinterpret_cast<const __half2*>(&y);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float2 fx = __half22float2(hx[q]), fy = __half22float2(hy[q]);
                acc[w] += (double)__fmul_rn(fx.x, fy.x);
                acc[w] += (double)__fmul_rn(fx.y, fy.y);
            }
        }
    }
    return (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

// Row L2 norms of the two fp16 sets (set 1's rows, then set 2's) and the
// largest of each set, rounded up with a relative margin of 2^-20, the
// largest as float bits (non-negative floats order as their bits, so the
// integer maximum is the float maximum and the result does not depend on the
// order of the updates).  One warp per row; the block's largest per set
// goes to one atomicMax each.
__global__ void k_f16_max_norms(const __half* __restrict__ a, int n1, const __half* __restrict__ b, int n2, int D,
                                unsigned* __restrict__ out, float* __restrict__ row_norm) {
    __shared__ unsigned s_max[2];
    if (threadIdx.x < 2) s_max[threadIdx.x] = 0u;
    __syncthreads();
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (w < n1 + n2) {
        const __half* row = w < n1 ? a + (size_t)w * D : b + (size_t)(w - n1) * D;
        double s = 0.0;
        for (int k = lane; k < D; k += 32) {
            const float f = __half2float(row[k]);
            s += (double)__fmul_rn(f, f);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL_MASK, s, o);
        if (lane == 0) {
            const float nrm = __double2float_ru(sqrt(s) * (1.0 + 0x1p-20));
            row_norm[w] = nrm;
            atomicMax(&s_max[w < n1 ? 0 : 1], __float_as_uint(nrm));
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 && s_max[threadIdx.x]) atomicMax(&out[threadIdx.x], s_max[threadIdx.x]);
}

__device__ __forceinline__ void finish_f16_row(int i, float f1, float f2, int c1, float ratio_sq, int* best, int* pass,
                                               float* dist) {
    // pysift/core.py:2676-2680 (float32); no second column: no pass
    int ok = 0;
    float d = 0.0f;
    if (f2 > -INFINITY) {
        float db = 2.0f - 2.0f * f1;
        float ds = 2.0f - 2.0f * f2;
        db = db < 0.0f ? 0.0f : db;
        ds = ds < 0.0f ? 0.0f : ds;
        ok = (ds > 1e-10f) && (db < ratio_sq * ds);
        d = sqrtf(db);
    }
    best[i] = c1;
    pass[i] = ok;
    if (dist) dist[i] = d;
}

// Order-preserving bits of a float above the complemented column index: the
// integer maximum is the largest value with the lowest index.
__device__ __forceinline__ unsigned long long sim_key(float f, int c) {
    const unsigned u = __float_as_uint(f);
    const unsigned ord = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((unsigned long long)ord << 32) | (0xFFFFFFFFu - (unsigned)c);
}
__device__ __forceinline__ float sim_key_value(unsigned long long k) {
    const unsigned o = (unsigned)(k >> 32);
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}
__device__ __forceinline__ int sim_key_column(unsigned long long k) {
    return (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFu));
}

// Merge the chunk-level segments of one SIM_F16 scan (in segment order) and
// settle the row from its two best chunks: every column of both is
// recomputed exactly (one warp per row, a column of each chunk per lane),
// giving the exact best F1 (lowest index on ties) and second F2 among them.
// Every column of the other chunks has an fp32 value <= k3 (the third chunk's
// largest), so its exact value is <= k3 + e and its fp16 similarity
// <= U = fp16(k3 + e); the row is settled when U <= F2 and U < F1 (a column
// tying F1 could have a lower index).  Unsettled rows are appended to
// `recheck` (their order there does not matter: each row's result is
// computed on its own).
__global__ void k_match_merge_f16(const Top3* __restrict__ part, int n, int nseg, float ratio_sq,
                                  const __half* __restrict__ q, const __half* __restrict__ t, int n_t, int D,
                                  const float* __restrict__ norm_q, const unsigned* __restrict__ maxnorm_t,
                                  const int* __restrict__ error,
                                  int* __restrict__ best, int* __restrict__ pass, float* __restrict__ dist,
                                  int* __restrict__ recheck, int* __restrict__ n_recheck) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n) return;
    const Top3 a = merge_parts(part, i, nseg);
    // a scan that gave up on its MMA barrier left its parts unwritten: no
    // result, and no candidate chunk is trusted
    const bool c2 = a.k2 > -INFINITY;
    if (*error || !(a.k1 > -INFINITY) || a.i1 < 0 || a.i1 >= n_t || (c2 && (a.i2 < 0 || a.i2 >= n_t))) {
        if (lane == 0) {
            best[i] = -1;
            pass[i] = 0;
            if (dist) dist[i] = 0.0f;
        }
        return;
    }
    const __half* qi = q + (size_t)i * D;
    unsigned long long kb = 0, ks = 0;
    const int ca = a.i1 + lane, cb = a.i2 + lane;
    if (ca < n_t) kb = sim_key(f16_round_f64(dot_f16_exact(qi, t + (size_t)ca * D, D)), ca);
    if (c2 && cb < n_t) {
        const unsigned long long k = sim_key(f16_round_f64(dot_f16_exact(qi, t + (size_t)cb * D, D)), cb);
        ks = min(kb, k);
        kb = max(kb, k);
    }
    warp_top2_u64(kb, ks);
    if (lane != 0) return;
    const float f1 = sim_key_value(kb);
    const float f2 = ks ? sim_key_value(ks) : -INFINITY;
    if (a.k3 > -INFINITY) {
        const double e = (double)D * 0x1p-21 * (double)norm_q[i] * (double)__uint_as_float(*maxnorm_t);
        const float u = f16_round_f64((double)a.k3 + e);
        if (!(u <= f2 && u < f1)) {
            recheck[atomicAdd(n_recheck, 1)] = i;
            return;
        }
    }
    finish_f16_row(i, f1, f2, sim_key_column(kb), ratio_sq, best, pass, dist);
}

// Rows the merge could not settle: the exact fp16 similarity against every
// column, top-2 by (similarity desc, index asc).  One CTA per row (grid
// stride over both directions' lists); keys pack the order-preserving bits
// of the similarity above the complemented column index, so the integer
// maximum is the best with the lowest index.
constexpr int RECHECK_T = 1024;

__global__ void __launch_bounds__(RECHECK_T) k_match_recheck_f16(const int* __restrict__ list0, const int* __restrict__ list1,
                                                           const int* __restrict__ counts, const __half* __restrict__ a,
                                                           int n1, const __half* __restrict__ b, int n2, int D,
                                                           float ratio_sq, int* __restrict__ fbest,
                                                           int* __restrict__ fpass, float* __restrict__ fdist,
                                                           int* __restrict__ bbest, int* __restrict__ bpass,
                                                           float* __restrict__ bdist) {
    __shared__ __align__(16) __half qrow[128];
    __shared__ unsigned long long s_b[RECHECK_T / 32], s_s[RECHECK_T / 32];
    const int c0 = counts[0], call = c0 + counts[1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int v = blockIdx.x; v < call; v += gridDim.x) {
        const bool fwd = v < c0;
        const int i = fwd ? list0[v] : list1[v - c0];
        const __half* t = fwd ? b : a;
        const int nt = fwd ? n2 : n1;
        if ((int)threadIdx.x < D) qrow[threadIdx.x] = (fwd ? a : b)[(size_t)i * D + threadIdx.x];
        __syncthreads();
        unsigned long long kb = 0, ks = 0;  // best and second keys; 0 = none
        for (int j = threadIdx.x; j < nt; j += blockDim.x) {
            const unsigned long long key = sim_key(f16_round_f64(dot_f16_exact(qrow, t + (size_t)j * D, D)), j);
            ks = max(ks, min(kb, key));
            kb = max(kb, key);
        }
        warp_top2_u64(kb, ks);
        if (lane == 0) {
            s_b[warp] = kb;
            s_s[warp] = ks;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                ks = max(max(ks, s_s[w]), min(kb, s_b[w]));
                kb = max(kb, s_b[w]);
            }
            const float f1 = sim_key_value(kb);
            const float f2 = ks ? sim_key_value(ks) : -INFINITY;
            const int c1 = sim_key_column(kb);
            if (fwd)
                finish_f16_row(i, f1, f2, c1, ratio_sq, fbest, fpass, fdist);
            else
                finish_f16_row(i, f1, f2, c1, ratio_sq, bbest, bpass, bdist);
        }
        __syncthreads();
    }
}

// Mutual matches in query order: fwd[i] = j passes, bwd[j] = i passes.
// One CTA; each thread owns a run of up to 32 consecutive rows (so the pairs
// of a thread are consecutive in the output), tests them with its loads
// issued eight rows at a time, and one block scan of the per-thread counts
// places them; more than 32 x blockDim rows take several rounds.
__global__ void __launch_bounds__(1024) k_match_mutual(const int* __restrict__ fbest, const int* __restrict__ fpass,
                                                       const float* __restrict__ fdist, const int* __restrict__ bbest,
                                                       const int* __restrict__ bpass, int n1, int2* __restrict__ pairs,
                                                       float* __restrict__ pdist, int* __restrict__ count) {
    __shared__ int sh[33];
    const int span = (int)blockDim.x * 32;
    int base = 0;
    for (int c0 = 0; c0 < n1; c0 += span) {
        const int per = min(32, ceil_div(min(span, n1 - c0), (int)blockDim.x));
        const int r0 = c0 + (int)threadIdx.x * per;
        unsigned mask = 0;
        for (int k0 = 0; k0 < per; k0 += 8) {
            int j[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = r0 + k0 + u;
                j[u] = (k0 + u < per && i < n1 && fpass[i]) ? fbest[i] : -1;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = r0 + k0 + u;
                if (j[u] >= 0 && bpass[j[u]] && bbest[j[u]] == i) mask |= 1u << (k0 + u);
            }
        }
        int tot;
        int pos = base + block_excl_scan(__popc(mask), &tot, sh);
        while (mask) {
            const int k = __ffs(mask) - 1;
            mask &= mask - 1;
            const int i = r0 + k;
            pairs[pos] = make_int2(i, fbest[i]);
            pdist[pos] = fdist[i];
            ++pos;
        }
        base += tot;
    }
    if (threadIdx.x == 0) *count = base;
}

// |row|^2 of uint8 rows as int32 and float32 (exact: below 2^24).  Rows
// n .. n_pad-1 get zero norms.
__global__ void k_row_norms_u8(const uint8_t* __restrict__ d, int n, int n_pad, int D, int* __restrict__ norms,
                               float* __restrict__ fnorms) {
    const int i = blockIdx.x * blockDim.y + threadIdx.y;
    if (i >= n_pad) return;
    int s = 0;
    for (int k = threadIdx.x; k < D; k += 32) {
        const int v = i < n ? d[(size_t)i * D + k] : 0;
        s += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL_MASK, s, o);
    if (threadIdx.x == 0) {
        norms[i] = s;
        fnorms[i] = (float)s;
    }
}

// Split-nibble e4m3 planes of uint8-valued rows, v = 16 h + l with h, l in
// 0..15 (e4m3 holds 0..15 and 16 * (0..15) exactly).  The query-side row is
// [16h | h | 16l | l], the train-side row [16h | 16l | h | l], each plane D
// bytes, so that the 4D-long dot product of the two is
// 256 h.h' + 16 h.l' + 16 l.h' + l.l' = v.v', the four nibble GEMMs in one.
// Both sides are written in the tiled layout of 4D-byte rows; rows
// n .. n_pad-1 are zero.
__global__ void k_split_nibbles_u8(const uint8_t* __restrict__ d, int n, int n_pad, int D,
                                   uint8_t* __restrict__ qside, uint8_t* __restrict__ tside) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n_pad * D) return;
    const int r = (int)(i / D), k = (int)(i - (size_t)r * D);
    const int v = r < n ? d[i] : 0;
    const float h = (float)(v >> 4), l = (float)(v & 15);
    const uint8_t e16h = __nv_cvt_float_to_fp8(16.0f * h, __NV_SATFINITE, __NV_E4M3);
    const uint8_t eh = __nv_cvt_float_to_fp8(h, __NV_SATFINITE, __NV_E4M3);
    const uint8_t e16l = __nv_cvt_float_to_fp8(16.0f * l, __NV_SATFINITE, __NV_E4M3);
    const uint8_t el = __nv_cvt_float_to_fp8(l, __NV_SATFINITE, __NV_E4M3);
    const int RB = 4 * D;
    auto at = [&](int byte) { return tiled_off(r, byte >> 4, RB) + (byte & 15); };
    qside[at(k)] = e16h;
    qside[at(D + k)] = eh;
    qside[at(2 * D + k)] = e16l;
    qside[at(3 * D + k)] = el;
    tside[at(k)] = e16h;
    tside[at(D + k)] = e16l;
    tside[at(2 * D + k)] = eh;
    tside[at(3 * D + k)] = el;
}

static int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return n > 0 ? n : 148;
}

// Segments of the train side.  Two CTAs fit on an SM (tensor memory), so a
// grid of n_qb x nseg CTAs runs in ceil(n_qb nseg / (2 SMs)) waves of
// ceil(n_tt / nseg) tiles each (+1 for a CTA's prologue): the segment count
// with the fewest tile-steps is taken (the smaller one on ties), so that a
// few CTAs past a full wave do not double the scan.
static void scan_split(int n_q, int n_t, int& nseg, int& seg_tiles) {
    const int n_qb = ceil_div(n_q, MT), n_tt = ceil_div(n_t, NT);
    const long long slots = 2LL * sm_count();
    long long best = -1;
    nseg = 1;
    for (int s_ = 1; s_ <= n_tt; ++s_) {
        const int st_ = ceil_div(n_tt, s_);
        if (ceil_div(n_tt, st_) != s_) continue;  // a segment count that leaves none empty
        const long long waves = (n_qb * (long long)s_ + slots - 1) / slots;
        const long long cost = waves * (st_ + 1);
        if (best < 0 || cost < best) {
            best = cost;
            nseg = s_;
        }
    }
    seg_tiles = ceil_div(n_tt, nseg);
    nseg = ceil_div(n_tt, seg_tiles);
}

template <int MODE, int RB>
static int launch_scan(const RowScanArgs& a, int nseg, cudaStream_t st) {
    // query tile + the slab ring: about 96 KB, so that no more than two CTAs
    // (2 x 256 tensor-memory columns) share an SM
    using G = TileGeom<RB>;
    const size_t smem_launch = std::max((size_t)G::TILE + (size_t)G::NS * G::SLAB, (size_t)80 * 1024);
    PYSIFT_CUDA_TRY(cudaFuncSetAttribute(k_match_rows<MODE, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_launch));
    dim3 grid(ceil_div(a.n_q, MT), nseg);
    k_match_rows<MODE, RB><<<grid, SCAN_THREADS, smem_launch, st>>>(a);
    PYSIFT_LAUNCH_CHECK("k_match_rows");
    return PYSIFT_OK;
}

// row bytes: 2 D for fp16 rows, 4 D for the split e4m3 planes, D for uint8 / int8
static int launch_scan_mode(int mode, const RowScanArgs& a, int D, int nseg, cudaStream_t st) {
    if (mode == SIM_I8) return D == 64 ? launch_scan<SIM_I8, 64>(a, nseg, st) : launch_scan<SIM_I8, 128>(a, nseg, st);
    if (mode == SIM_F16) return D == 64 ? launch_scan<SIM_F16, 128>(a, nseg, st) : launch_scan<SIM_F16, 256>(a, nseg, st);
    if (mode == DIST_U8) return D == 64 ? launch_scan<DIST_U8, 64>(a, nseg, st) : launch_scan<DIST_U8, 128>(a, nseg, st);
    return D == 64 ? launch_scan<SPLIT_FP8, 256>(a, nseg, st) : launch_scan<SPLIT_FP8, 512>(a, nseg, st);
}

struct MatchLayout {
    // off_ctl: int[8] = error flag, SIM_F16 recheck counts (forward, backward),
    // max row norms (set 1, set 2) as float bits
    size_t off_fpart, off_bpart, off_fbest, off_fpass, off_fdist, off_bbest, off_bpass, off_bdist, off_ctl;
    size_t off_rl0, off_rl1, off_nrm;
    size_t off_na, off_nb, off_fna, off_fnb;
    // the scan operands in the tiled layout (rows padded to whole tiles):
    // query side and train side of each set (the same buffer except for the
    // split e4m3 planes)
    size_t off_qa, off_ta, off_qb, off_tb;
    size_t total;
};

static int pad_rows(int n) { return ceil_div(n, MT) * MT; }

// exact: 0 = fp16 similarity (and int8 similarity, whose D-byte rows fit in
// its buffers), 1 = exact via unsigned 8-bit MMAs, 2 = exact via split e4m3
// (scan row bytes: 2 D, D, 4 D)
static MatchLayout match_layout(int n1, int n2, int D, int exact) {
    MatchLayout l;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t r = off;
        off = align_up(off + bytes, 256);
        return r;
    };
    // segments never exceed the tiles of the other side
    const size_t part_bytes = sizeof(Top3);
    l.off_fpart = take((size_t)n1 * ceil_div(n2, NT) * part_bytes);
    l.off_bpart = take((size_t)n2 * ceil_div(n1, MT) * part_bytes);
    l.off_fbest = take((size_t)n1 * 4);
    l.off_fpass = take((size_t)n1 * 4);
    l.off_fdist = take((size_t)n1 * 4);
    l.off_bbest = take((size_t)n2 * 4);
    l.off_bpass = take((size_t)n2 * 4);
    l.off_bdist = take((size_t)n2 * 4);
    l.off_ctl = take(8 * sizeof(int));
    l.off_rl0 = l.off_rl1 = l.off_nrm = 0;
    if (exact == 0) {
        l.off_rl0 = take((size_t)n1 * 4);
        l.off_rl1 = take((size_t)n2 * 4);
        l.off_nrm = take(((size_t)n1 + n2) * 4);
    }
    l.off_na = l.off_nb = l.off_fna = l.off_fnb = 0;
    if (exact == 1 || exact == 2) {  // |row|^2 as int32 and as float32, padded to whole tiles
        l.off_na = take((size_t)pad_rows(n1) * 4);
        l.off_nb = take((size_t)pad_rows(n2) * 4);
        l.off_fna = take((size_t)pad_rows(n1) * 4);
        l.off_fnb = take((size_t)pad_rows(n2) * 4);
    }
    const size_t rb = exact == 2 ? 4 * (size_t)D : exact == 1 ? (size_t)D : 2 * (size_t)D;
    l.off_qa = take((size_t)pad_rows(n1) * rb);
    l.off_qb = take((size_t)pad_rows(n2) * rb);
    l.off_ta = l.off_qa;
    l.off_tb = l.off_qb;
    if (exact == 2) {
        l.off_ta = take((size_t)pad_rows(n1) * rb);
        l.off_tb = take((size_t)pad_rows(n2) * rb);
    }
    l.total = off;
    return l;
}

template <typename T>
static T* wsp(void* ws, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(ws) + off);
}

// a / b: the query-side and train-side rows of each set (the same rows
// except for the split e4m3 planes, whose two sides differ)
// rows_a, rows_b: the row-major descriptor sets as the caller passed them
// (fp16, uint8 or int8 rows, 16-byte aligned); the scan operands are built
// from them in the workspace in the tiled layout.
static int run_match(int mode, const uint8_t* rows_a, int n1, const uint8_t* rows_b, int n2, int D, float ratio_sq,
                     const MatchLayout& l, void* ws, int* fbest_out, int* fpass_out, int* bbest_out, int* bpass_out,
                     int32_t* pairs, float* pdist, int32_t* count, cudaStream_t st, const float* sa = nullptr,
                     const float* sb = nullptr) {
    int* ctl = wsp<int>(ws, l.off_ctl);
    int* err = ctl;
    PYSIFT_CUDA_TRY(cudaMemsetAsync(ctl, 0, 8 * sizeof(int), st));
    const __half* ha = reinterpret_cast<const __half*>(rows_a);
    const __half* hb = reinterpret_cast<const __half*>(rows_b);
    unsigned* maxnorm = reinterpret_cast<unsigned*>(ctl + 3);
    uint8_t* qa = wsp<uint8_t>(ws, l.off_qa);
    uint8_t* ta = wsp<uint8_t>(ws, l.off_ta);
    uint8_t* qb = wsp<uint8_t>(ws, l.off_qb);
    uint8_t* tb = wsp<uint8_t>(ws, l.off_tb);
    const int p1 = pad_rows(n1), p2 = pad_rows(n2);
    const bool sim = mode == SIM_F16 || mode == SIM_I8;
    int* na = !sim ? wsp<int>(ws, l.off_na) : nullptr;
    int* nb = !sim ? wsp<int>(ws, l.off_nb) : nullptr;
    float* fna = !sim ? wsp<float>(ws, l.off_fna) : nullptr;
    float* fnb = !sim ? wsp<float>(ws, l.off_fnb) : nullptr;
    if (sim) {
        const int rb = mode == SIM_F16 ? 2 * D : D;
        k_tile_rows<<<(unsigned)ceil_div_ll((long long)p1 * (rb / 16), 256), 256, 0, st>>>(rows_a, n1, p1, rb, qa);
        PYSIFT_LAUNCH_CHECK("k_tile_rows");
        k_tile_rows<<<(unsigned)ceil_div_ll((long long)p2 * (rb / 16), 256), 256, 0, st>>>(rows_b, n2, p2, rb, qb);
        PYSIFT_LAUNCH_CHECK("k_tile_rows");
    } else {
        k_row_norms_u8<<<ceil_div(p1, 8), dim3(32, 8), 0, st>>>(rows_a, n1, p1, D, na, fna);
        PYSIFT_LAUNCH_CHECK("k_row_norms_u8");
        k_row_norms_u8<<<ceil_div(p2, 8), dim3(32, 8), 0, st>>>(rows_b, n2, p2, D, nb, fnb);
        PYSIFT_LAUNCH_CHECK("k_row_norms_u8");
        if (mode == DIST_U8) {
            k_tile_rows<<<(unsigned)ceil_div_ll((long long)p1 * (D / 16), 256), 256, 0, st>>>(rows_a, n1, p1, D, qa);
            PYSIFT_LAUNCH_CHECK("k_tile_rows");
            k_tile_rows<<<(unsigned)ceil_div_ll((long long)p2 * (D / 16), 256), 256, 0, st>>>(rows_b, n2, p2, D, qb);
            PYSIFT_LAUNCH_CHECK("k_tile_rows");
        }
        if (mode == SPLIT_FP8) {
            k_split_nibbles_u8<<<(unsigned)ceil_div_ll((long long)p1 * D, 256), 256, 0, st>>>(rows_a, n1, p1, D, qa, ta);
            PYSIFT_LAUNCH_CHECK("k_split_nibbles_u8");
            k_split_nibbles_u8<<<(unsigned)ceil_div_ll((long long)p2 * D, 256), 256, 0, st>>>(rows_b, n2, p2, D, qb, tb);
            PYSIFT_LAUNCH_CHECK("k_split_nibbles_u8");
        }
    }
    if (mode == SIM_F16) {
        k_f16_max_norms<<<ceil_div(n1 + n2, 8), 256, 0, st>>>(ha, n1, hb, n2, D, maxnorm, wsp<float>(ws, l.off_nrm));
        PYSIFT_LAUNCH_CHECK("k_f16_max_norms");
    }
    int* fbest = fbest_out ? fbest_out : wsp<int>(ws, l.off_fbest);
    int* fpass = fpass_out ? fpass_out : wsp<int>(ws, l.off_fpass);
    int* bbest = bbest_out ? bbest_out : wsp<int>(ws, l.off_bbest);
    int* bpass = bpass_out ? bpass_out : wsp<int>(ws, l.off_bpass);
    float* fdist = wsp<float>(ws, l.off_fdist);
    float* bdist = wsp<float>(ws, l.off_bdist);
    for (int dir = 0; dir < 2; ++dir) {
        RowScanArgs s;
        s.q = dir == 0 ? qa : qb;
        s.t = dir == 0 ? tb : ta;
        s.n_q = dir == 0 ? n1 : n2;
        s.n_t = dir == 0 ? n2 : n1;
        s.norm_t = dir == 0 ? fnb : fna;
        s.norm_ti = dir == 0 ? nb : na;
        s.scale_q = dir == 0 ? sa : sb;
        s.scale_t = dir == 0 ? sb : sa;
        s.part = wsp<void>(ws, dir == 0 ? l.off_fpart : l.off_bpart);
        s.error = err;
        int nseg;
        scan_split(s.n_q, s.n_t, nseg, s.seg_tiles);
        const int rc = launch_scan_mode(mode, s, D, nseg, st);
        if (rc) return rc;
        int* best = dir == 0 ? fbest : bbest;
        int* pass = dir == 0 ? fpass : bpass;
        float* dist = dir == 0 ? fdist : bdist;
        if (mode == SIM_F16) {
            k_match_merge_f16<<<ceil_div(s.n_q, 8), 256, 0, st>>>(
                static_cast<const Top3*>(s.part), s.n_q, nseg, ratio_sq, dir == 0 ? ha : hb, dir == 0 ? hb : ha,
                s.n_t, D, wsp<float>(ws, l.off_nrm) + (dir == 0 ? 0 : n1), maxnorm + (dir == 0 ? 1 : 0), err, best,
                pass, dist,
                wsp<int>(ws, dir == 0 ? l.off_rl0 : l.off_rl1), ctl + 1 + dir);
            PYSIFT_LAUNCH_CHECK("k_match_merge_f16");
        } else if (mode == SIM_I8) {
            k_match_merge_i8<<<ceil_div(s.n_q, 256), 256, 0, st>>>(static_cast<const Top2*>(s.part), s.n_q, nseg,
                                                                   ratio_sq, best, pass, dist);
            PYSIFT_LAUNCH_CHECK("k_match_merge_i8");
        } else {
            k_match_merge_u8<<<ceil_div(s.n_q, 8), 256, 0, st>>>(
                static_cast<const Top3*>(s.part), s.n_q, nseg, ratio_sq, dir == 0 ? rows_a : rows_b,
                dir == 0 ? rows_b : rows_a, s.n_t, D, dir == 0 ? na : nb, dir == 0 ? nb : na, err, best, pass, dist);
            PYSIFT_LAUNCH_CHECK("k_match_merge_u8");
        }
    }
    if (mode == SIM_F16) {
        k_match_recheck_f16<<<sm_count(), RECHECK_T, 0, st>>>(wsp<int>(ws, l.off_rl0), wsp<int>(ws, l.off_rl1), ctl + 1,
                                                             ha, n1, hb, n2, D, ratio_sq, fbest, fpass, fdist, bbest,
                                                             bpass, bdist);
        PYSIFT_LAUNCH_CHECK("k_match_recheck_f16");
    }
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
    PYSIFT_CHECK_ARG(exact_u8 >= 0 && exact_u8 <= 2, "exact_u8 must be 0, 1 or 2");
    *bytes = match_layout(n1, n2, D, exact_u8).total;
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
    MatchLayout l = match_layout(n1, n2, D, 0);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    const float ratio_sq = (float)((double)ratio * (double)ratio);
    const uint8_t* a = reinterpret_cast<const uint8_t*>(d1);
    const uint8_t* b = reinterpret_cast<const uint8_t*>(d2);
    return run_match(SIM_F16, a, n1, b, n2, D, ratio_sq, l, workspace, fwd_best, fwd_pass, bwd_best, bwd_pass, pairs,
                     pair_dist, pair_count, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_match_fp16_recheck_counts(const void* workspace, int32_t n1, int32_t n2, int32_t D, int32_t* counts,
                                     pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(workspace && counts, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n1 >= 1 && n2 >= 1 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    const MatchLayout l = match_layout(n1, n2, D, 0);
    PYSIFT_CUDA_TRY(cudaMemcpyAsync(counts, static_cast<const char*>(workspace) + l.off_ctl + sizeof(int),
                                    2 * sizeof(int), cudaMemcpyDeviceToDevice, reinterpret_cast<cudaStream_t>(stream)));
    return PYSIFT_OK;
}

int pysift_match_u8_exact(const uint8_t* d1, int32_t n1, const uint8_t* d2, int32_t n2, int32_t D, float ratio,
                          void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                          int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                          int32_t* pair_count, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(d1 && d2 && workspace && pairs && pair_dist && pair_count, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n1 >= 1 && n2 >= 1 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    PYSIFT_CHECK_ARG((reinterpret_cast<uintptr_t>(d1) & 15) == 0 && (reinterpret_cast<uintptr_t>(d2) & 15) == 0,
                     "descriptor arrays must be 16-byte aligned");
    MatchLayout l = match_layout(n1, n2, D, 1);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    const float ratio_sq = (float)((double)ratio * (double)ratio);
    return run_match(DIST_U8, d1, n1, d2, n2, D, ratio_sq, l, workspace, fwd_best, fwd_pass, bwd_best, bwd_pass,
                     pairs, pair_dist, pair_count, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_match_u8_split_fp8(const uint8_t* d1, int32_t n1, const uint8_t* d2, int32_t n2, int32_t D, float ratio,
                              void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                              int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                              int32_t* pair_count, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(d1 && d2 && workspace && pairs && pair_dist && pair_count, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n1 >= 1 && n2 >= 1 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    PYSIFT_CHECK_ARG((reinterpret_cast<uintptr_t>(d1) & 15) == 0 && (reinterpret_cast<uintptr_t>(d2) & 15) == 0,
                     "descriptor arrays must be 16-byte aligned");
    MatchLayout l = match_layout(n1, n2, D, 2);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    const float ratio_sq = (float)((double)ratio * (double)ratio);
    return run_match(SPLIT_FP8, d1, n1, d2, n2, D, ratio_sq, l, workspace, fwd_best, fwd_pass, bwd_best, bwd_pass,
                     pairs, pair_dist, pair_count, reinterpret_cast<cudaStream_t>(stream));
}

int pysift_match_i8(const int8_t* d1, const float* s1, int32_t n1, const int8_t* d2, const float* s2, int32_t n2,
                    int32_t D, float ratio, void* workspace, size_t workspace_bytes, int32_t* fwd_best,
                    int32_t* fwd_pass, int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                    int32_t* pair_count, pysift_stream_t stream) {
    PYSIFT_CHECK_ARG(d1 && d2 && s1 && s2 && workspace && pairs && pair_dist && pair_count, "NULL pointer argument");
    PYSIFT_CHECK_ARG(n1 >= 1 && n2 >= 1 && (D == 64 || D == 128), "bad sizes (D must be 64 or 128)");
    PYSIFT_CHECK_ARG((reinterpret_cast<uintptr_t>(d1) & 15) == 0 && (reinterpret_cast<uintptr_t>(d2) & 15) == 0,
                     "descriptor arrays must be 16-byte aligned");
    MatchLayout l = match_layout(n1, n2, D, 0);
    if (workspace_bytes < l.total) {
        set_error("workspace %zu bytes < required %zu", workspace_bytes, l.total);
        return PYSIFT_ERR_WORKSPACE;
    }
    const float ratio_sq = (float)((double)ratio * (double)ratio);
    const uint8_t* a = reinterpret_cast<const uint8_t*>(d1);
    const uint8_t* b = reinterpret_cast<const uint8_t*>(d2);
    return run_match(SIM_I8, a, n1, b, n2, D, ratio_sq, l, workspace, fwd_best, fwd_pass, bwd_best, bwd_pass, pairs,
                     pair_dist, pair_count, reinterpret_cast<cudaStream_t>(stream), s1, s2);
}

}  // extern "C"
