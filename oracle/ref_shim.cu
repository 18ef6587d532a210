// Launchers of the reference's own CUDA kernels -- TEST INFRASTRUCTURE ONLY.
//
// The kernels themselves are compiled by oracle/build_ref.py from the source
// strings in the reference's pysift/core.py; this file declares them and
// launches each with the grid, block and shared-memory shape the reference
// uses (core.py:583-602 for the separable blur, 1409-1419 for the extrema,
// 1481-1488 for the refinement, 1577-1582 for the orientation and 1849-1855
// for the descriptor).  All pointers are device pointers; every function
// returns the launch's cudaError_t.
#include <cuda_runtime.h>

extern "C" __global__ void gauss_h(const float* in, float* out, const float* kern, int H, int W, int radius);
extern "C" __global__ void gauss_v(const float* in, float* out, const float* kern, int H, int W, int radius);
extern "C" __global__ void find_extrema_fused(const float* dog, int* coords, int* count, int S, int H, int W,
                                              float thresh, int max_cands, int border);
extern "C" __global__ void refine_keypoints(const float* dogs_flat, const int* dogs_meta, const int* all_cands, int N,
                                            int n_scales, int border_, float contrast_thresh_s, float edge_score,
                                            int* out_valid, int* out_oct, float* out_ri, float* out_ci, int* out_si,
                                            float* out_response);
extern "C" __global__ void orientation_hist(const float* gauss_3d, const float* kpts, float* out_angles, int N, int H,
                                            int W);
extern "C" __global__ void sift_descriptor_coop(const float* gauss_3d, const float* kpts, float* descs, int N,
                                                int n_slices, int H, int W);

extern "C" {

// _fast_gaussian: horizontal pass into tmp, vertical pass into out.
int ref_gaussian(const float* in, float* tmp, float* out, const float* kern, int H, int W, int radius,
                 cudaStream_t st) {
    const int tpb_h = 256;
    gauss_h<<<dim3((W + tpb_h - 1) / tpb_h, H), tpb_h, (tpb_h + 2 * radius) * 4, st>>>(in, tmp, kern, H, W, radius);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    gauss_v<<<dim3((W + 31) / 32, (H + 7) / 8), dim3(32, 8), (8 + 2 * radius) * 32 * 4, st>>>(tmp, out, kern, H, W,
                                                                                              radius);
    return (int)cudaGetLastError();
}

int ref_find_extrema(const float* dog, int* coords, int* count, int S, int H, int W, float thresh, int max_cands,
                     int border, cudaStream_t st) {
    const long long total = (long long)S * H * W;
    find_extrema_fused<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(dog, coords, count, S, H, W, thresh, max_cands,
                                                                       border);
    return (int)cudaGetLastError();
}

int ref_refine(const float* dogs_flat, const int* dogs_meta, const int* cands, int N, int n_scales, int border,
               float cts, float edge, int* valid, int* oct, float* ri, float* ci, int* si, float* resp,
               cudaStream_t st) {
    if (N <= 0) return 0;
    refine_keypoints<<<(N + 255) / 256, 256, 0, st>>>(dogs_flat, dogs_meta, cands, N, n_scales, border, cts, edge,
                                                       valid, oct, ri, ci, si, resp);
    return (int)cudaGetLastError();
}

int ref_orientation(const float* gauss_3d, const float* kpts, float* angles, int N, int H, int W, cudaStream_t st) {
    if (N <= 0) return 0;
    orientation_hist<<<(N + 3) / 4, 128, 0, st>>>(gauss_3d, kpts, angles, N, H, W);
    return (int)cudaGetLastError();
}

int ref_descriptor(const float* gauss_3d, const float* kpts, float* descs, int N, int n_slices, int H, int W,
                   cudaStream_t st) {
    if (N <= 0) return 0;
    sift_descriptor_coop<<<N, 128, 516 * 4, st>>>(gauss_3d, kpts, descs, N, n_slices, H, W);
    return (int)cudaGetLastError();
}

}  // extern "C"
