// Shared helpers for the pysift_b200 CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/pysift_b200.h"

namespace pysift {

constexpr unsigned FULL_MASK = 0xffffffffu;

// Thread-local error message behind pysift_last_error().
void set_error(const char* fmt, ...);

#define PYSIFT_CHECK_ARG(cond, ...)            \
    do {                                       \
        if (!(cond)) {                         \
            ::pysift::set_error(__VA_ARGS__);  \
            return PYSIFT_ERR_INVALID_ARG;     \
        }                                      \
    } while (0)

#define PYSIFT_CUDA_TRY(call)                                                              \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            ::pysift::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                                __FILE__, __LINE__);                                       \
            return PYSIFT_ERR_CUDA;                                                        \
        }                                                                                  \
    } while (0)

// Every kernel launch of the library is followed by exactly one
// PYSIFT_LAUNCH_CHECK, which also counts it (pysift_launch_count()).
void count_launch();

#define PYSIFT_LAUNCH_CHECK(name)                                                          \
    do {                                                                                   \
        ::pysift::count_launch();                                                          \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess) {                                                           \
            ::pysift::set_error("launch of %s failed: %s", name, cudaGetErrorString(e_));  \
            return PYSIFT_ERR_CUDA;                                                        \
        }                                                                                  \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

__device__ __forceinline__ float round_half(float v) { return __half2float(__float2half_rn(v)); }

// Exclusive scan of one int per thread across a block of blockDim.x
// threads (multiple of 32, <= 1024).  sh must hold 33 ints.  Returns the
// thread's exclusive prefix; *total receives the block total.
__device__ __forceinline__ int block_excl_scan(int v, int* total, int* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(FULL_MASK, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = (lane < nwarps) ? sh[lane] : 0;
        int s = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int y = __shfl_up_sync(FULL_MASK, s, d);
            if (lane >= d) s += y;
        }
        sh[lane] = s - w;
        if (lane == 31) sh[32] = s;
    }
    __syncthreads();
    int res = sh[warp] + x - v;
    *total = sh[32];
    __syncthreads();
    return res;
}

// Exclusive scan of one value per warp (lane 0's v) across the block; returns
// the warp's exclusive prefix, *total = block sum.  sh: 33 ints.
__device__ __forceinline__ int block_warp_excl_scan(int v, int* total, int* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int w = (lane < nwarps) ? sh[lane] : 0;
        int s = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(FULL_MASK, s, d);
            if (lane >= d) s += y;
        }
        sh[lane] = s - w;
        if (lane == 31) sh[32] = s;
    }
    __syncthreads();
    const int res = sh[warp];
    *total = sh[32];
    __syncthreads();
    return res;
}

// Ordered compaction of [0, n) by the whole block (blockDim.x a multiple of
// 32).  load(i) returns element i's payload (called for every i < n, before
// any store of the chunk, so the loads of a chunk are all in flight
// together); keep(payload) says whether it is kept; store(pos, payload)
// writes a kept element at pos = number of kept elements before it.  A warp
// covers 32*K consecutive elements per chunk (coalesced, K-major then lane);
// positions come from ballot popcounts and one scan of the warp counts per
// chunk.  Returns the number of kept elements.
template <int K, typename P, typename LoadF, typename KeepF, typename StoreF>
__device__ __forceinline__ int block_compact(int n, LoadF load, KeepF keep, StoreF store, int* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const int chunk = (int)blockDim.x * K;
    int base = 0;
    for (int c0 = 0; c0 < n; c0 += chunk) {
        const int wbase = c0 + warp * 32 * K;
        P pl[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = wbase + k * 32 + lane;
            if (i < n) pl[k] = load(i);
        }
        unsigned bal[K];
        int wcnt = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = wbase + k * 32 + lane;
            bal[k] = __ballot_sync(FULL_MASK, i < n && keep(pl[k]));
            wcnt += __popc(bal[k]);
        }
        int tot;
        int pos = base + block_warp_excl_scan(wcnt, &tot, sh);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if ((bal[k] >> lane) & 1u) store(pos + __popc(bal[k] & below), pl[k]);
            pos += __popc(bal[k]);
        }
        base += tot;
    }
    return base;
}

__device__ __forceinline__ int warp_excl_scan(int v, int* total) {
    const int lane = threadIdx.x & 31;
    int x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(FULL_MASK, x, d);
        if (lane >= d) x += y;
    }
    *total = __shfl_sync(FULL_MASK, x, 31);
    return x - v;
}

}  // namespace pysift
