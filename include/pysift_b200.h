/*
 * pysift_b200.h -- C ABI of the B200 SIFT-and-stitching hot path.
 *
 * Every entry point takes device pointers, sizes and a cudaStream_t, returns
 * an int status (PYSIFT_OK or a negative PYSIFT_ERR_*), never synchronises
 * the device, and allocates no device memory: buffers (including the
 * workspace) are owned by the caller.  pysift_last_error() returns a
 * thread-local message for the last failing call on the calling thread.
 *
 * Reference interfaces replaced (paths in SivaIITM/PySIFT):
 *   PySIFT.detectAndCompute           pysift/core.py:2021-2172
 *   PySIFT._build_gaussian_pyramid    pysift/core.py:1234-1352
 *   _fast_gaussian / gauss_h / gauss_v pysift/core.py:475-608
 *   _adaptive_contrast_thresh         pysift/core.py:1129-1148
 */
#ifndef PYSIFT_B200_H
#define PYSIFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* pysift_stream_t; /* == cudaStream_t */

#define PYSIFT_OK 0
#define PYSIFT_ERR_INVALID_ARG (-1)
#define PYSIFT_ERR_WORKSPACE (-2)    /* workspace too small */
#define PYSIFT_ERR_CUDA (-3)         /* a launch or CUDA call failed */
#define PYSIFT_ERR_UNSUPPORTED (-4)  /* configuration outside the supported range */
#define PYSIFT_ERR_CAPACITY (-5)     /* an output buffer is too small */

#define PYSIFT_MAX_OCTAVES 8
#define PYSIFT_MAX_LEVELS 8          /* n_scales + 3 */
#define PYSIFT_MAX_RADIUS 48
#define PYSIFT_MAX_TAPS (2 * PYSIFT_MAX_RADIUS + 1)
#define PYSIFT_DESC_DIM 128

/* Detector configuration.  The host fills the tables the reference computes
 * on the host (Gaussian weights in numpy float32, the per-scale sigma and
 * patch-half-width tables, the keypoint size table); pysift_b200/core.py
 * does this exactly as pysift/core.py:563-577, 1555, 1798-1810, 1512-1521. */
typedef struct pysift_detect_config {
    int32_t n_octaves;            /* 1..8 (reference: 5 on >= 12 GB GPUs)          */
    int32_t n_scales;             /* S, 1..5                                        */
    float sigma0;                 /* 1.6                                            */
    double contrast_thresh;       /* base threshold before entropy scaling (0.04)   */
    float edge_score;             /* float32((edge+1)^2/edge)                       */
    int32_t double_image;         /* 2x cubic upsample when H*W < double_px_cap     */
    int64_t double_px_cap;        /* 16,000,000 (>= 12 GB tier) or 4,194,304        */
    int32_t fp16_pyramid;         /* store octaves >= 2 rounded to binary16         */
    int32_t dsp;                  /* DSP-SIFT pooling                               */
    int32_t n_dsp;                /* 3, 4 or 5                                      */
    float dsp_scales[8];
    int32_t rootsift;             /* RootSIFT post-normalisation                    */
    int32_t max_cands_per_octave; /* 25000                                          */
    int32_t keypoint_cap;         /* 8000                                           */
    int32_t starvation_min;       /* 100: retry at half threshold below this        */
    int32_t border;               /* 5                                              */
    /* Gaussian kernels: [0] base blur when doubled, [1] base blur when not
     * doubled, [2 + s] increment s -> s+1 for s = 0 .. n_scales+1.
     * radius 0 means "no blur" (sigma < 0.01). */
    int32_t blur_radius[2 + PYSIFT_MAX_LEVELS];
    float blur_weights[2 + PYSIFT_MAX_LEVELS][PYSIFT_MAX_TAPS];
    float ori_sigma[PYSIFT_MAX_LEVELS];           /* orientation sigma per scale index   */
    float desc_ph[PYSIFT_MAX_LEVELS];             /* descriptor patch half-width per si  */
    float kp_size[2][PYSIFT_MAX_OCTAVES][PYSIFT_MAX_LEVELS]; /* [doubled][o][si]     */
    /* 0: every oriented keypoint, rows in the reference's (x, y) order.
     * N > 0: when there are more than N, only the N with the largest
     * response are described and returned, ordered by response (descending,
     * ties in (x, y) order) -- the selection GPUPyStitch's feature extraction
     * makes after detection (pysift/core.py:2566-2571). */
    int32_t output_limit;
} pysift_detect_config;

/* Device-side counters written by pysift_detect_and_compute (int32 each). */
#define PYSIFT_STAT_N_KEYPOINTS 0       /* oriented keypoints written             */
#define PYSIFT_STAT_N_REFINED 1         /* refined keypoints before the cap       */
#define PYSIFT_STAT_N_KEPT 2            /* after the keypoint cap                 */
#define PYSIFT_STAT_RETRIED 3           /* 1 when the half-threshold retry ran    */
#define PYSIFT_STAT_CAPPED 4            /* 1 when the keypoint cap applied        */
#define PYSIFT_STAT_DOUBLED 5           /* 1 when the 2x upsample ran             */
#define PYSIFT_STAT_CAND_OVERFLOW 6     /* octaves whose candidates were truncated */
#define PYSIFT_STAT_CANDS 8             /* [8..15] extrema found per octave       */
#define PYSIFT_STAT_REFINED_OCT 16      /* [16..23] refined per octave            */
#define PYSIFT_STAT_THRESH_BITS 24      /* float bits of ct/S actually used       */
#define PYSIFT_STAT_COUNT 32

/* sizeof(pysift_detect_config), for bindings that mirror the struct. */
size_t pysift_detect_config_size(void);

/* Bytes of workspace pysift_detect_and_compute needs for an H x W image. */
int pysift_detect_workspace_size(const pysift_detect_config* cfg, int32_t H, int32_t W, size_t* bytes);

/* Largest number of keypoints the call can emit (4 orientations x cap). */
int32_t pysift_detect_max_keypoints(const pysift_detect_config* cfg);

/*
 * Full detectAndCompute on a device-resident uint8 grayscale image
 * (pysift/core.py:2021-2172).  Outputs, sorted by (x, y) like the reference:
 *   kpts[i] = {x, y, size, angle}   (float32, the reference's gpu_output rows)
 *   response[i] (float32), octave[i] (int32), desc[i][128] (float32;
 *   RootSIFT when cfg->rootsift, else the L2/clip/L2 vector).
 * stats (int32[PYSIFT_STAT_COUNT], device) receives the counters above;
 * stats[PYSIFT_STAT_N_KEYPOINTS] is the number of rows written.
 * max_out must be >= pysift_detect_max_keypoints(cfg).
 * stage_events: NULL, or PYSIFT_DETECT_STAGE_EVENTS cudaEvent_t handles that
 * are recorded on `stream` at the stage boundaries: 0 start, 1 base image
 * ready, 2 Gaussian pyramid ready, 3 extrema bitmask ready, 4 keypoints
 * refined and capped, 5 orientations ready, 6 end.
 */
#define PYSIFT_DETECT_STAGE_EVENTS 7
int pysift_detect_and_compute(const pysift_detect_config* cfg, const uint8_t* gray, int32_t H, int32_t W,
                              int64_t pitch_bytes, void* workspace, size_t workspace_bytes, float* kpts,
                              float* response, int32_t* octave, float* desc, int32_t max_out, int32_t* stats,
                              void* const* stage_events, pysift_stream_t stream);

/* Locate an intermediate buffer of a run inside its workspace (for tests
 * and tools).  what: 0 = Gaussian level (octave, level) as stored for the
 * consumers (binary16-rounded in fp16 mode), 1 = the upsampled/converted
 * base image before the first blur (octave, level ignored).  Returns the
 * byte offset, rows, cols and row pitch (in floats). */
int pysift_detect_workspace_view(const pysift_detect_config* cfg, int32_t H, int32_t W, int32_t what,
                                 int32_t octave, int32_t level, size_t* offset, int32_t* rows, int32_t* cols,
                                 int32_t* pitch_floats);

/* Separable Gaussian blur of one float32 image (_fast_gaussian,
 * pysift/core.py:552-608): horizontal then vertical FMA chain, reflect
 * boundary.  in/out pitches in floats; weights has 2*radius+1 entries
 * (host memory). */
int pysift_gauss_blur(const float* in, int32_t in_pitch, float* out, int32_t out_pitch, int32_t H, int32_t W,
                      const float* weights, int32_t radius, pysift_stream_t stream);

/* Testing hook: the blur's tile height (16, 32 or 40 rows) is normally
 * picked per launch from the level size and the device's occupancy;
 * rows = 16, 32 or 40 forces it for every later launch in the process,
 * rows = 0 restores the automatic choice.  Results do not depend on it. */
int pysift_set_blur_tile_rows(int32_t rows);

/* Tile heights measured by an autotuner (pysift_b200/autotune.py), used
 * when no height is forced: rows[r * 16 + c] for radius r = 0 .. 16 (row 0
 * unused) and level size class c = pysift_blur_size_class(H, W) (floor of
 * log2 of the level's pixel count, minus 10, clamped to 0 .. 15): 16, 32 or
 * 40, or 0 for the built-in rule.  n = 17 * 16 entries, or 0 to clear the
 * table.  Applies to later calls in the process; results do not depend on
 * it.  No counterpart in the reference (its blur launches have one shape,
 * pysift/core.py:583-602). */
int pysift_blur_size_class(int32_t H, int32_t W);
int pysift_set_blur_tile_table(const int32_t* rows, int32_t n);

/* 2x cubic B-spline zoom of a uint8 image scaled by 1/255
 * (cupyx.scipy.ndimage.zoom(order=3) at pysift/core.py:1270-1275).
 * coef: caller scratch of H*W doubles; out: 2H x 2W floats, pitch in floats. */
int pysift_zoom2x_u8(const uint8_t* gray, int32_t H, int32_t W, int64_t pitch_bytes, int32_t fp16_round,
                     double* coef, float* out, int32_t out_pitch, pysift_stream_t stream);

/* ---- brute-force ratio-test matching (tcgen05 tensor cores) ----
 * Replaces GPUPyStitch._match_symmetric / _match_one_direction and the
 * mutual intersection of _match_features (pysift/core.py:2574-2701,
 * 2930-2940).  Per direction: best index, ratio-test pass flag; the mutual
 * pairs (i, j) in query order with distance sqrt(d1^2).  Ties between equal
 * scores go to the lower index.  D must be 64 or 128.  Workspace mode
 * exact_u8: 0 = pysift_match_fp16, 1 = pysift_match_u8_exact,
 * 2 = pysift_match_u8_split_fp8. */
int pysift_match_workspace_size(int32_t n1, int32_t n2, int32_t D, int32_t exact_u8, size_t* bytes);

/* Reference semantics: fp16 operands (16-byte aligned rows), the similarity
 * s = the fp16 rounding (nearest, ties to even) of the exact dot product,
 * d^2 = max(0, 2 - 2 s), pass iff d2^2 > 1e-10 and d1^2 < ratio^2 d2^2
 * (float32). pairs: int32[n1][2].  The tensor-core scan keeps, per row, the
 * three 32-column chunks with the largest fp32 values; the columns of the two
 * best chunks are recomputed exactly and the rows they do not settle are
 * recomputed over every column, so the result is the one the exact
 * similarity matrix gives, for rows of L2 norm <= 1 (the stitch path's
 * normalised descriptors; the float64 sums are exact there). */
int pysift_match_fp16(const uint16_t* d1, int32_t n1, const uint16_t* d2, int32_t n2, int32_t D, float ratio,
                      void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                      int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist, int32_t* pair_count,
                      pysift_stream_t stream);

/* Rows of the last pysift_match_fp16 on this workspace that the candidate
 * check left to the exact recomputation over every column, forward and
 * backward: counts (device int32[2]) receives them, stream-ordered.  A
 * diagnostic; no counterpart in the reference. */
int pysift_match_fp16_recheck_counts(const void* workspace, int32_t n1, int32_t n2, int32_t D, int32_t* counts,
                                     pysift_stream_t stream);

/* Exact squared L2 of uint8 descriptors (16-byte aligned rows) via unsigned
 * 8-bit tensor-core products with 32-bit integer accumulation (exact for
 * D <= 128), pass iff d2^2 > 0 and d1^2 < ratio^2 d2^2. */
int pysift_match_u8_exact(const uint8_t* d1, int32_t n1, const uint8_t* d2, int32_t n2, int32_t D, float ratio,
                          void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                          int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                          int32_t* pair_count, pysift_stream_t stream);

/* The same exact matching through FP8: each uint8 value v = 16 h + l is split
 * into e4m3 planes (16h, h, 16l, l all exact in e4m3) and one kind::f8f6f4
 * tcgen05 GEMM over the 4D concatenated planes forms 256 h.h' + 16 h.l' +
 * 16 l.h' + l.l' = v.v' (the four nibble GEMMs in one accumulation).
 * Rows 16-byte aligned.  Workspace from
 * pysift_match_workspace_size(..., exact_u8 = 2, ...). */
int pysift_match_u8_split_fp8(const uint8_t* d1, int32_t n1, const uint8_t* d2, int32_t n2, int32_t D, float ratio,
                              void* workspace, size_t workspace_bytes, int32_t* fwd_best, int32_t* fwd_pass,
                              int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                              int32_t* pair_count, pysift_stream_t stream);

/* uint8 descriptors as OpenCV writes them: saturate(rint(512 v)) of each
 * float of n_rows x 128 descriptors (the L2 / clip / L2 vector, i.e. a
 * detection with rootsift = 0); device pointers. */
int pysift_desc_to_u8(const float* desc, int64_t n_rows, uint8_t* out, pysift_stream_t stream);

/* ---- stitch path (GPUPyStitch) ---- */

/* cv2.cvtColor(BGR2GRAY) for uint8 (pysift/core.py:2546). */
int pysift_bgr2gray(const uint8_t* bgr, int32_t H, int32_t W, int64_t pitch_bytes, uint8_t* gray, int32_t gray_pitch,
                    pysift_stream_t stream);

/* cv2.createCLAHE(clip_limit, (tiles_x, tiles_y)).apply (pysift/core.py:2563-2565);
 * lut: caller scratch of pysift_clahe_lut_bytes bytes. */
int pysift_clahe_lut_bytes(int32_t tiles_x, int32_t tiles_y, size_t* bytes);
int pysift_clahe(const uint8_t* src, int32_t H, int32_t W, int32_t pitch, double clip_limit, int32_t tiles_x,
                 int32_t tiles_y, uint8_t* lut, uint8_t* dst, int32_t dst_pitch, pysift_stream_t stream);

/* Indices of the k rows with the largest response, in the order of a
 * stable descending sort (pysift/core.py:2566-2571); k <= n.  rank: caller
 * scratch of n int32. */
int pysift_topk_by_response(const float* response, int32_t n, int32_t k, int32_t* rank, int32_t* out_idx,
                            pysift_stream_t stream);

/* pts[m] = (double) kpts[pairs[m][col]][0:2] for m < count (device count). */
int pysift_gather_points(const float* kpts, const int32_t* pairs, const int32_t* count, int32_t max_pairs, int32_t col,
                         double* pts, pysift_stream_t stream);

/* Matcher preparation (pysift/core.py:2877-2888, 2703-2743): row L2
 * normalisation (+1e-7), PCA statistics (float32 mean, float64 covariance,
 * both summed over fixed 128-row chunks) of the stacked normalised sets in a
 * caller workspace of pysift_pca_workspace_size bytes, projection (D in
 * {64, 128}, P in {32, 64, 128}) + normalisation to fp16. */
int pysift_l2_normalize_rows(const float* in, int32_t n, int32_t D, float* out, pysift_stream_t stream);
int pysift_pca_workspace_size(int32_t n, int32_t D, size_t* bytes);
int pysift_pca_stats(const float* x, int32_t n, int32_t D, void* workspace, size_t workspace_bytes, float* mean,
                     double* cov, pysift_stream_t stream);
/* PCA basis from a D x D float64 covariance (D even, <= 128), replacing the
 * reference's cp.linalg.eigh (pysift/core.py:2729-2736): proj (device,
 * float32 D x P, row-major) receives the eigenvectors of the P largest
 * eigenvalues in ascending eigenvalue order (as eigh's v[:, -P:]), found by
 * a round-robin parallel Jacobi in float64 on the device (sweeps until no
 * off-diagonal element exceeds 2^-60 trace; sweeps, if not NULL, a device
 * int32 receiving their count).  Workspace: pysift_pca_basis_workspace_size. */
int pysift_pca_basis_workspace_size(int32_t D, size_t* bytes);
int pysift_pca_basis(const double* cov, int32_t D, int32_t P, void* workspace, size_t workspace_bytes, float* proj,
                     int32_t* sweeps, pysift_stream_t stream);
int pysift_pca_project_f16(const float* x, int32_t n, int32_t D, const float* mean, const float* proj, int32_t P,
                           uint16_t* out, pysift_stream_t stream);
int pysift_to_f16(const float* in, int64_t n, uint16_t* out, pysift_stream_t stream);

/* int8 matching (GPUPyStitch(int8_matching=True), pysift/core.py:2894-2923):
 * pysift_pca_project_f32 is pysift_pca_project_f16 with the normalised rows
 * kept in float32; pysift_quantize_i8_rows quantises float32 rows per row,
 * scale = 127 / (max |x| + 1e-7) (as reciprocal * 127), q = trunc(clamp(x *
 * scale, -127, 127)); pysift_match_i8 matches int8 rows (16-byte aligned)
 * with a tcgen05 kind::i8 GEMM, similarity = int32 / (s1 * s2) in float32,
 * then the ratio test, mutual check and outputs of pysift_match_fp16
 * (workspace from pysift_match_workspace_size(..., exact_u8 = 0, ...)). */
int pysift_pca_project_f32(const float* x, int32_t n, int32_t D, const float* mean, const float* proj, int32_t P,
                           float* out, pysift_stream_t stream);
int pysift_quantize_i8_rows(const float* x, int32_t n, int32_t D, int8_t* q, float* scale, pysift_stream_t stream);
int pysift_match_i8(const int8_t* d1, const float* s1, int32_t n1, const int8_t* d2, const float* s2, int32_t n2,
                    int32_t D, float ratio, void* workspace, size_t workspace_bytes, int32_t* fwd_best,
                    int32_t* fwd_pass, int32_t* bwd_best, int32_t* bwd_pass, int32_t* pairs, float* pair_dist,
                    int32_t* pair_count, pysift_stream_t stream);

/* The raw 32-bit MT19937 stream of torch.Generator(device='cpu').manual_seed(seed):
 * torch.randint(0, N, (B, 4), generator=g) equals out[0:4B] % N (host function). */
void pysift_mt19937_u32(uint32_t seed, uint32_t* out, int64_t n);

/* Batched RANSAC with MAGSAC++ (or classic) scoring and two LO refits
 * (pysift/core.py:2272-2313, 3011-3097).  pts: n x 2 float64 on the device;
 * rand_u32: 4*n_hyp raw MT19937 draws; outputs H (9 float64, row-major),
 * inlier mask (n bytes) and info = {n_inliers, best hypothesis, LO stage}. */
int pysift_ransac_workspace_size(int32_t n, int32_t n_hyp, size_t* bytes);
int pysift_ransac(const double* pts1, const double* pts2, int32_t n, const uint32_t* rand_u32, int32_t n_hyp,
                  double inlier_thresh, double sigma_max, int32_t magsac, int32_t min_inliers, void* workspace,
                  size_t workspace_bytes, double* H_out, uint8_t* mask_out, int32_t* info, pysift_stream_t stream);
/* The same with the point count on the device (n_dev, e.g. the match count
 * pysift_match_* wrote), so that matching, point gathering and RANSAC run
 * without the host reading the count in between: pts hold up to n_cap
 * points, the workspace is sized for n_cap, and a count below 4 yields
 * info = {0, 0, 0} (the caller reports the shortage after reading info).
 * No counterpart in the reference (its RANSAC takes host arrays). */
int pysift_ransac_count(const double* pts1, const double* pts2, const int32_t* n_dev, int32_t n_cap,
                        const uint32_t* rand_u32, int32_t n_hyp, double inlier_thresh, double sigma_max,
                        int32_t magsac, int32_t min_inliers, void* workspace, size_t workspace_bytes, double* H_out,
                        uint8_t* mask_out, int32_t* info, pysift_stream_t stream);

/* Normalised DLT homography of all n correspondences (pysift/core.py:2959-2981). */
int pysift_dlt_homography(const double* pts1, const double* pts2, int32_t n, int32_t* idx_scratch, double* H_out,
                          pysift_stream_t stream);

/* Warp of image 1 (BGR uint8) onto a cw x ch canvas through hinv9
 * (float32 inverse homography) with grid_sample(bilinear, zeros,
 * align_corners=True) semantics and uint8 truncation
 * (pysift/core.py:3210-3239), placement of image 2 at (iox, ioy)
 * (pysift/core.py:3794-3800) and, where both cover the canvas, a linear
 * feather blend (weights 1 + distance to the image border).  Optional
 * outputs: warped image 1, both masks, per-row/column coverage extents;
 * out may be NULL when warped image 1 and its mask are requested. */
int pysift_warp_feather(const uint8_t* img1, int32_t hs, int32_t ws, int32_t pitch1, const uint8_t* img2, int32_t h2,
                        int32_t w2, int32_t pitch2, int32_t cw, int32_t ch, const float* hinv9, float ox, float oy,
                        int32_t iox, int32_t ioy, int32_t feather, uint8_t* out, uint8_t* warped, uint8_t* mask1,
                        uint8_t* mask2, int32_t* row_lo, int32_t* row_hi, int32_t* col_lo, int32_t* col_hi,
                        pysift_stream_t stream);

/* Differentiation (no counterpart in the reference, which has no autograd):
 * float forms of the descriptor and of the warp + feather blend with
 * hand-written adjoints, used by pysift_b200/grad.py.
 *
 * pysift_desc_f32_forward: float descriptors (L2 -> clip 0.2 -> L2, no
 * RootSIFT) of n keypoints on one Gaussian level (kp: n rows [centre row,
 * centre column, angle in degrees]; patch half-width ph, pysift/core.py:
 * 693-835), the raw 128-bin histograms in hist.  pysift_desc_f32_backward
 * adds dL/dlevel (glevel, same pitch as level) given dL/ddesc, recomputing
 * the samples from the level and hist.  pysift_blur_adjoint: gin (+)= B^T gout
 * for the separable blur B of pysift_gauss_blur with half-sample symmetric
 * reflection (radius below both sides; weights on the device; tmp: H x W
 * scratch).  pysift_warp_f32_forward/backward: the float warp of image 1 by
 * hinv onto a cw x ch canvas, image 2 at (iox, ioy), linear feather blend;
 * the backward adds dL/dimg1, dL/dimg2 and dL/dhinv (float64). */
int pysift_desc_f32_forward(const float* level, int32_t H, int32_t W, int32_t pitch, const float* kp, int32_t n,
                            int32_t ph, float* hist, float* desc, pysift_stream_t stream);
int pysift_desc_f32_backward(const float* level, int32_t H, int32_t W, int32_t pitch, const float* kp, int32_t n,
                             int32_t ph, const float* hist, const float* gdesc, float* glevel,
                             pysift_stream_t stream);
int pysift_blur_adjoint(const float* gout, int32_t gout_pitch, float* gin, int32_t gin_pitch, float* tmp,
                        int32_t tmp_pitch, int32_t H, int32_t W, const float* weights_dev, int32_t radius,
                        int32_t accumulate, pysift_stream_t stream);
int pysift_warp_f32_forward(const float* img1, int32_t hs, int32_t ws, int32_t C, const float* img2, int32_t h2,
                            int32_t w2, int32_t cw, int32_t ch, const double* hinv_host, double ox, double oy,
                            int32_t iox, int32_t ioy, float* out, pysift_stream_t stream);
int pysift_warp_f32_backward(const float* img1, int32_t hs, int32_t ws, int32_t C, const float* img2, int32_t h2,
                             int32_t w2, int32_t cw, int32_t ch, const double* hinv_host, double ox, double oy,
                             int32_t iox, int32_t ioy, const float* gout, float* gimg1, float* gimg2, double* ghinv,
                             pysift_stream_t stream);

/* Reference composition (pysift/core.py:3386-3553, 3686-3714, 3794-3814):
 * gain compensation, seam cost (colour difference + 0.05 |Sobel| of the
 * average gray), dynamic-programming seam along the longer overlap axis,
 * seam mask blurred with sigma 3 inside the overlap, Laplacian pyramid blend
 * of n_levels levels and the paste with uint8 truncation.  image1: cw x ch
 * x 3, uint8 (image1_f32 = 0: the warped image) or float32 (image1_f32 = 1:
 * the unclipped result of an earlier blend, as the second pass of a
 * three-image stitch takes it, pysift/core.py:3931-3947); canvas2: cw x ch x
 * 3 uint8; masks: cw x ch bytes (0 / 1); all on the device.  seam_k25: the 25
 * float32 taps of the sigma-3 seam-mask blur (host); gauss_w9: the 9 float64
 * taps of gaussian_filter(sigma = 1) (host).  color_match: 0 = the gain
 * (pysift/core.py:3697-3698), 1 = histogram matching (_hist_match,
 * pysift/core.py:3591-3625, color_match='hist').  Outputs (at least one of pano
 * and blended): pano (cw x ch x 3 uint8, zero where neither image covers),
 * blended (cw x ch x 3 float32, the blend before any clipping), both (union
 * mask) and seam_rmse (one double on the device: the RMS colour difference
 * over the overlap after gain, NaN when there is no overlap). */
int pysift_place_image(const uint8_t* img, int32_t h, int32_t w, int32_t pitch, int32_t cw, int32_t ch, int32_t iox,
                       int32_t ioy, uint8_t* canvas, uint8_t* mask, pysift_stream_t stream);
int pysift_blend_workspace_size(int32_t cw, int32_t ch, int32_t n_levels, size_t* bytes);
int pysift_blend_multiband(const void* image1, int32_t image1_f32, const uint8_t* mask1, const uint8_t* canvas2,
                           const uint8_t* mask2, int32_t cw, int32_t ch, int32_t n_levels, int32_t color_match,
                           const float* seam_k25,
                           const double* gauss_w9, void* workspace, size_t workspace_bytes, uint8_t* pano,
                           uint8_t* both, float* blended, double* seam_rmse, pysift_stream_t stream);
/* Per-row and per-column first / last set pixel of a cw x ch coverage mask
 * (INT32_MAX / -1 where a line is empty): the inputs of the inner-rectangle
 * crop (pysift/core.py:3627-3684). */
int pysift_mask_extents(const uint8_t* mask, int32_t cw, int32_t ch, int32_t* row_lo, int32_t* row_hi,
                        int32_t* col_lo, int32_t* col_hi, pysift_stream_t stream);
/* The inner-rectangle crop (pysift/core.py:3627-3684) from the four extents
 * arrays of pysift_mask_extents, computed on the HOST (all pointers are host
 * memory; no stream).  box[0..3] = x, y, width, height of the crop in the
 * canvas; box[4] = 0 when no pixel is covered (the whole canvas), 1 when the
 * coverage has no inner rectangle (its bounding box), 2 for the inner
 * rectangle. */
int pysift_autocrop_box(const int32_t* row_lo, const int32_t* row_hi, const int32_t* col_lo, const int32_t* col_hi,
                        int32_t cw, int32_t ch, int32_t* box);
/* height rows of width_bytes from src (row pitch src_pitch) to dst (row pitch
 * dst_pitch), asynchronously on the stream; either side may be device or
 * page-locked host memory (the copy direction follows the pointers).  Used to
 * read a crop of a device canvas into host memory in one copy. */
int pysift_copy2d(void* dst, size_t dst_pitch, const void* src, size_t src_pitch, size_t width_bytes, size_t height,
                  pysift_stream_t stream);

/* Allocation-free 2x zoom (no counterpart in the reference; it exists for
 * callers that cannot allocate device memory at the call site, such as a
 * plugin inside a host application that owns the device heap).  Same result
 * as pysift_zoom2x_u8, but the coefficient scratch is a fixed file-scope
 * device array of PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS doubles (8 MiB) that every
 * GPU loading the library holds until exit.  Inputs larger than that
 * (H*W > PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS) return PYSIFT_ERR_CAPACITY.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  The address is cached per device ordinal for
 * the process: it holds for the device's primary context (the one the CUDA
 * runtime uses) and only until that context is destroyed, so the entry point
 * is not for callers that make their own driver-API contexts current or call
 * cudaDeviceReset between calls.  All calls share the one array: calls that
 * overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  Allocates nothing. */
#define PYSIFT_ZOOM2X_NOALLOC_MAX_PIXELS (1 << 20)
int pysift_zoom2x_u8_noalloc(const uint8_t* gray, int32_t H, int32_t W, int64_t pitch_bytes, int32_t fp16_round,
                             float* out, int32_t out_pitch, pysift_stream_t stream);

/* Number of kernel launches the library has issued in this process
 * (all threads and devices).  A caller that captures library calls into a
 * CUDA graph and replays it adds the graph's kernel count per replay with
 * pysift_count_launches (and subtracts the captured launches, which did not
 * run), so that the count stays the number of kernels that ran. */
int64_t pysift_launch_count(void);
void pysift_count_launches(int64_t n);

/* memcpy of `bytes` host bytes split over up to n_threads host threads (the
 * caller and a persistent pool of at most 7 workers; below 1 MiB, or with
 * n_threads = 1, one plain memcpy).  Used for the staging copy of a host image
 * into page-locked memory ahead of its upload.  Synchronous; concurrent
 * callers are served one after another. */
int pysift_host_copy(void* dst, const void* src, size_t bytes, int32_t n_threads);

const char* pysift_last_error(void);
const char* pysift_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif
