/*
 * oracle/pfd_oracle.h -- CPU oracle of the plenoptic depth hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline legs of bench.py load this library, and only to check or time the
 * reference algorithm; the product library never links it.
 *
 * Pins.  The reference (fengyunxuan6/plenoptic-for-depth) ships no tests,
 * fixtures or golden vectors.  The PatchMatch restatement (patchmatch.c) is
 * pinned to the reference's own frame kernels, compiled from its sources in
 * oracle/ref and run beside the engine on the same hypotheses and the same
 * random streams (tests/test_gpu_refpin.py): the two differ only by the
 * reference's fast-math arithmetic, by as much as the reference's own IEEE
 * build differs from it.  The host-side stages (checks.c, fuse.c, vdrd.c,
 * select.cpp, mla.cpp, blur.c) restate reference code that needs the OpenCV
 * C++ SDK, Eigen, Boost, libpleno, yaml-cpp and libv, none of which is
 * installed, so it cannot run here: their parity with the reference is
 * unpinned, and they are pinned to OpenCV (cv2) on the OpenCV arithmetic they
 * call, to known answers and to an FP64 cross-check; refocus.c has no
 * reference counterpart.  The texture emulation is pinned to tex2D on a B200.
 *
 * Every function cites the reference lines it restates.  Arithmetic follows
 * oracle/canon.h.
 */
#ifndef PFD_ORACLE_H
#define PFD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One frame of micro-images (views), the layout AdaptMIPMFrame builds in
 * BuildViewIndexMap (AdaptMIPMFrame.cpp:145-222): views in problem-map order,
 * neighbour ids padded with -1, counts per view. */
typedef struct {
    int n_views;
    int mi_w, mi_h;              /* MLA_Mask_Width_Cuda / Height (AdaptMIPMFrame.cpp:139-140) */
    int max_nb;                  /* m_max_neighbors (16 in the reference; up to 32 here) */
    const float* gray;           /* [V][mi_h][mi_w], integer values 0..255 */
    const float* blur;           /* [V][mi_h][mi_w] or NULL (no blur channel: penalty 0) */
    const float* centers;        /* [V][2] lens centres, raw pixel coordinates */
    const int* nb_ids;           /* [V][max_nb] view ids, -1 padded */
    const int* nb_counts;        /* [V] */
} orc_frame;

/* PatchMatchParamsLF (LFDepthInfo.h:19-46) fields the Frame path reads. */
typedef struct {
    int max_iterations;
    int patch_size;
    int radius_increment;
    int top_k;
    float sigma_spatial;
    float sigma_color;
    float depth_min;
    float depth_max;
    float base;                  /* Base: lens pitch in pixels (AdaptMIPMFrame.cpp:138) */
    int shifted;                 /* 0: the reference's NCC moments; 1: moments of (texel - centre texel) */
    int acmm;                    /* 1: the ACMM matcher's rules (AdaptMIPMFrameACMM.cu), single pyramid level */
} orc_params;

/* Per-pixel state, the four ping-pong buffers of AdaptMIPMFrame
 * (AdaptMIPMFrame.cpp:311-318), each [V * mi_w * mi_h]. */
typedef struct {
    float* plane;                /* float4: nx, ny, nz, disparity */
    float* cost;
    float* disp;                 /* float4: d, d_real, baseline, baseline/d_real */
    uint32_t* sel;
} orc_state;

/* Cost of each hypothesis against each neighbour of its view:
 * ComputeMultiViewCostVector_Frame (AdaptMIPMFrame.cu:181-225).  costs is
 * [n][max_nb] (2.0 beyond the view's count), disps [n][max_nb][4]. */
int orc_cost_vectors(const orc_frame* f, const orc_params* p, const int* vids, const int* pxy,
                     const float* planes, int n, float* costs, float* disps);

/* NCC of one (pixel, plane, neighbour) in FP64 with exact (unquantised)
 * bilinear sampling: the precision oracle. */
double orc_ncc_fp64(const orc_frame* f, const orc_params* p, int vid, int k, int px, int py,
                    const float* plane);
/* orc_ncc_fp64 for n hypotheses and all max_nb neighbours (2.0 past a view's
 * count) into out [n][max_nb].  sampling 0: exact bilinear at sample points
 * computed in double; 1: the texture's own sampling (point rounded to 1/256
 * texel, 8-bit weights) at those points, in double; 2: the texture's sampling
 * at the FP32 path's own anchor and sample points (canonical float
 * arithmetic), everything after the sample in double, which leaves the
 * accumulation of the weights and moments as the only difference from FP32. */
void orc_ncc_fp64_batch(const orc_frame* f, const orc_params* p, const int* vids, const int* pxy,
                        const float* planes, int n, int sampling, int nthreads, double* out);

/* RandomInitializationForFrame (AdaptMIPMFrame.cu:474-518) over all pixels. */
int orc_pm_init(const orc_frame* f, const orc_params* p, uint64_t seed, orc_state* out, int nthreads);

/* Same, restricted to views [v0, v1) (the bounded CPU-baseline sample). */
int orc_pm_init_views(const orc_frame* f, const orc_params* p, uint64_t seed, orc_state* out, int v0, int v1,
                      int nthreads);

/* One CheckerboardUpdateFrame launch (AdaptMIPMFrame.cu:520-947): next <- update(prev). */
int orc_pm_sweep(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                 const orc_state* prev, orc_state* next, int nthreads);

/* Same, restricted to views [v0, v1): the bounded sample the CPU baseline times. */
/* orc_pm_sweep that also returns the in-bounds NCC taps the reference's algorithm
 * evaluates in it (the roofline's algorithmic unit), or -1. */
long long orc_pm_sweep_taps(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                            const orc_state* prev, orc_state* next, int nthreads);
/* orc_pm_sweep_taps on views [v0, v1) only. */
long long orc_pm_sweep_views_taps(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                                  const orc_state* prev, orc_state* next, int v0, int v1, int nthreads);
int orc_pm_sweep_views(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                       const orc_state* prev, orc_state* next, int v0, int v1, int nthreads);

/* RunPatchMatchCUDAForFrame_Impl (AdaptMIPMFrame.cu:949-995): init, then
 * max_iterations x (phase 0, phase 1).  Result in out.  With p->acmm,
 * RunPatchMatchCUDAForFrameACMM_Impl (AdaptMIPMFrameACMM.cu:931-990) for one
 * pyramid level: the same, then orc_acmm_post_refine. */
int orc_patchmatch(const orc_frame* f, const orc_params* p, uint64_t seed, orc_state* out, int nthreads);
/* PostRefineMetadataFrame (AdaptMIPMFrameACMM.cu:903-929) over every pixel of st. */
int orc_acmm_post_refine(const orc_frame* f, const orc_params* p, orc_state* st, int nthreads);

/* ---- consistency pass (oracle/checks.c) ---- */

/* MIDisparityFilterConfig (CheckModule/MIDisparityFilter.h:24-57); the values
 * MIStereoMatch::FilterAndStatic uses are in MIStereoMatch.cpp:759-778. */
typedef struct {
    int   max_triplet;
    float min_valid_disp;
    int   use_selected_views_only;
    int   clear_selected_views_when_invalid;
    int   enable_cost_filter;
    float max_cost;
    int   enable_cycle_geo_filter;
    float max_geo_err_px;
    int   enable_cycle_photo_filter;
    float max_photo_err_u;
    int   min_good_neighbors;
    int   enable_spike_filter;
    float spike_abs_diff;
    int   spike_min_neighbors;
} orc_filter_cfg;

/* PixelRejectReason (MIDisparityFilter.h:102-109) */
enum { ORC_PR_KEEP = 0, ORC_PR_COST = 80, ORC_PR_NOSUPPORT = 140, ORC_PR_CYCLE = 200, ORC_PR_SPIKE = 255 };
/* MIDisparityFilterStats counters (MIDisparityFilter.h:59-77) */
enum { ORC_FS_TOTAL = 0, ORC_FS_VALID_IN, ORC_FS_KEPT, ORC_FS_REMOVED, ORC_FS_COST, ORC_FS_NOSUPPORT,
       ORC_FS_CYCLE, ORC_FS_SPIKE, ORC_FS_COUNT };

/* MIDisparityFilterCPU::FilterGlobal (MIDisparityFilter.cpp:962-986): filters
 * the views in order, invalidating rejected pixels of st in place; reason
 * [V*mi_w*mi_h] receives the reject reasons, stats[ORC_FS_COUNT] the counters. */
int orc_filter_global(const orc_frame* f, const orc_filter_cfg* cfg, float baseline_unit, orc_state* st,
                      uint8_t* reason, long long* stats);

/* ComputeTileReprojectionErrorMap (MIDisparityFilter.cpp:695-842) for all
 * views: per-pixel median cycle error, -1 where undefined. */
int orc_reprojection_error(const orc_frame* f, const orc_filter_cfg* cfg, float baseline_unit, const orc_state* st,
                           float* err);

/* MICycleClampConfig (MICycleCheck.h:54-78) and MICycleMaskParams (:44-50);
 * doubles of the reference become floats here because every use casts them
 * to float first. */
typedef struct orc_cycle_cfg {
    int   max_triplet;
    int   clamp_photo;
    float photo_u;
    int   clamp_geo;
    float geo_u_px;
    int   pixel_gate_enabled;
    int   gate_min_good_neighbors;
    float gate_geo_px;
    float gate_photo_u;
    int   gate_use_clamped;
    float sobel_thresh;
    float var_thresh;
    int   use_and;
} orc_cycle_cfg;

/* MICycleCheckStats (MICycleCheck.h:24-42) plus the texture-masked figures that
 * CheckGlobal logs (MICycleCheck.cpp:805-880). */
typedef struct orc_cycle_stats {
    double  mean_geo_err_px, median_geo_err_px, p90_geo_err_px, mean_photo_err;
    long long num_samples;
    double  rmse_geo_err_px, rmse_photo_err;
    double  completeness, completeness_geo, completeness_photo;
    long long completeness_masked_pixels, completeness_good_pixels, completeness_good_pixels_geo,
              completeness_good_pixels_photo;
    long long masked_count, all_count;
    double  masked_geo_mean, masked_photo_mean, masked_geo_rmse, masked_photo_rmse, coverage;
    double  masked_geo_median_approx, masked_geo_p90_approx, masked_geo_min, masked_geo_max;
} orc_cycle_stats;

/* BuildTextureMaskAndViz (MICycleCheck.cpp:186-213) on one W x H float image:
 * Sobel magnitude, 7x7 variance (reflect-101 borders) and the 0/255 mask. */
int orc_texture_mask(const float* gray, int W, int H, const orc_cycle_cfg* cfg, float* grad, float* var,
                     uint8_t* mask);

/* MICycleCheckerCPU::CheckGlobal (MICycleCheck.cpp:727-893) with CheckTile
 * (:282-725): read-only.  geo_err / pho_err / texmask ([V*mi_w*mi_h], each
 * nullable) receive the per-tile maps. */
int orc_cycle_check(const orc_frame* f, const orc_cycle_cfg* cfg, float baseline_unit, const orc_state* st,
                    orc_cycle_stats* out, float* geo_err, float* pho_err, uint8_t* texmask);

/* cv::meanStdDev of the 3x3 window with top-left (x0, y0) (test hook). */
void orc_mean_std_3x3(const float* img, int W, int x0, int y0, float* mean, float* stdv);

/* Focal-stack render (no multi-slice render exists in the reference; it is
 * defined from the reference's own back-projection, LFRefocus::BackProject2MI,
 * FocalStack/LFRefocus.cpp:2119-2125, with the micro-image centre
 * ((m-1)/2 + 1) of FuseVirtualDepth_BackProject, :1635-1636).  Output pixel
 * (ox, oy) of slice s sits at raw coordinates X = (ox + 0.5) * (W / out_w) - 0.5
 * (Y likewise); every view i, in index order, whose back-projection
 * u = (X - c_i) / vd_s + (m-1)/2 + 1 lies in [0, m-1]^2 contributes the
 * bilinear sample of its gray micro-image at u:
 *   top = fma(ax, T01 - T00, T00), bot = fma(ax, T11 - T10, T10),
 *   val = fma(ay, bot - top, top)        (T01 = the texel right of T00)
 * and the output is the mean of the contributions (0 when there are none).
 * out: [n_slices][out_h][out_w]. */
int orc_refocus(const orc_frame* f, int raw_w, int raw_h, const float* slice_vd, int n_slices, int out_w, int out_h,
                float* out);
/* Number of (slice, output pixel, view) contributions, the render's work unit. */
long long orc_refocus_samples(const orc_frame* f, int raw_w, int raw_h, const float* slice_vd, int n_slices,
                              int out_w, int out_h);

/* Virtual-depth fusion and all-in-focus splat, LFRefocus::FuseVirtualDepth_BackProject
 * (FocalStack/LFRefocus.cpp:1553-1794).  The thresholds are the reference's
 * literals; mla_base = LightFieldParams::baseline * g_bl0 / (g_bl0 + g_B)
 * (ComputeVirtualDepth, :2087-2098). */
typedef struct {
    float mla_base;
    float min_ref_disp;          /* 1.0: reference pixels with a smaller disparity are skipped (:1641) */
    float max_reproj_px;         /* 1.0 (:1734) */
    float max_rel_vd;            /* 0.05 (:1734) */
    int   min_consistent;        /* 2 (:1752) */
} orc_fuse_params;
/* plane [V*ppv][4] (normal, disparity: ph_cuda.xyz and d_cuda), bgr [V][mi_h][mi_w][3]
 * (m_Image_rgb) or NULL for the gray images in all three channels; lists [V][max_list]
 * the views' m_NeighsSortVecForMatch as view ids (-1: a key with no result);
 * is_ref [V]: 1 for the micro-images fused as references (not garbage).
 * Outputs (raw_h x raw_w, zeroed first): vd_map float, conf u8, aif u8 x 3 (BGR);
 * points (may be NULL) [n][9] point, normal, colour in the reference's push order.
 * Returns the number of points, or -1. */
long long orc_fuse_virtual_depth(const orc_frame* f, const float* plane, const uint8_t* bgr, const int* lists,
                                 const int* list_counts, int max_list, const uint8_t* is_ref,
                                 const orc_fuse_params* p, int raw_w, int raw_h, float* vd_map, uint8_t* conf,
                                 uint8_t* aif, float* points);

/* Micro-lens centres from a white image (DepthSolver::ComputeMLACentersFromWhiteImage,
 * DepthSolver.cpp:710-870; Otsu :486-546).  bgr: 3-channel 8-bit image, row stride
 * step bytes.  orc_mla_otsu: the reference's threshold (histogram of the first W
 * bytes of each row).  orc_mla_contours: centroid and area of every external
 * contour of the thresholded gray image, in OpenCV's order.  orc_mla_centers: the
 * map entries in key order (row, column). */
int orc_mla_otsu(const uint8_t* bgr, int W, int H, int step);
int orc_mla_contours(const uint8_t* bgr, int W, int H, int step, int threshold, float* cx, float* cy, double* area,
                     int max_out);
int orc_mla_centers(const uint8_t* bgr, int W, int H, int step, float baseline, int mla_u_size, int mla_v_size,
                    int* out_col, int* out_row, float* out_cx, float* out_cy, float* out_area, int* out_abandon,
                    int max_out, int* threshold_out);

/* Matching-neighbour lists, SelectNeighbors::CollectMIANeighImagesForMatch
 * (MINeighbor/SelectNeighbors.cpp:113-193) with MISimilarityMeasure::MeasureSimilarity
 * and MLA_Problem's RANSAC outlier test (oracle/select.cpp). */
int orc_similarity(const uint8_t* src_bin, const uint8_t* nb_bin, int W, int H, float dx, float dy);
int orc_select_neighbors(int n_views, const float* centers, const int* tilekeys, int u_size, int v_size, float pitch,
                         const uint8_t* images, int mi_w, int mi_h, int max_out, int* nb_ids, int* nb_counts,
                         float* nb_sim);

/* Virtual-to-real depth (FocalStack/LFRefocus.cpp:2515-2593,
 * FocalStack/VirtualToRealDepthFunc.cpp:3390-3450), FP64. */
float orc_vd_to_rd(float v_depth, const double c[3]);
float orc_vd_to_rd_segment(float v_depth, const double* segs /* [nseg][5]: min, max, c0, c1, c2 */, int nseg);
void  orc_vd_to_rd_map(const float* vd, long n, const double c[3], double* rd);
int   orc_behavioral_fit(const float* real_depth, const float* vd, long n, double c[3]);

/* Scalar hooks for unit tests of the canonical arithmetic. */
float orc_expf(float x);
float orc_uniform(uint64_t seed, uint32_t sweep, uint32_t pixel, uint32_t n);
float orc_tex_fetch(const float* img, int w, int h, float sx, float sy);
void  orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Count of NCC taps with both reference and source sample inside the window,
 * for the hypotheses given (the algorithmic unit of the roofline). */
long long orc_count_taps(const orc_frame* f, const orc_params* p, const int* vids, const int* pxy,
                         const float* planes, int n);

/* Blur channel (oracle/blur.c).  orc_laplacian: cv::Laplacian(gray, CV_32F),
 * ksize 1, into score [H][W].  orc_blur_tiles: every view's window (origin
 * [V][2]) of the saturated score into tiles [V][mi_h][mi_w], and in counts [V]
 * (may be NULL) the window's pixels with score > 10.  Returns 0, or -1 for a
 * window outside the frame. */
void orc_laplacian(const uint8_t* gray, int W, int H, int pitch, float* score);
int orc_blur_tiles(const uint8_t* gray, int W, int H, int pitch, const int* origin, int V, int mi_w, int mi_h,
                   uint8_t* tiles, uint32_t* counts);

/* Richness channel (oracle/blur.c).  orc_glcm_contrast: the GLCM contrast map
 * of QuantizeRichnessByGLCM before normalisation, into score [H][W].
 * orc_normalize_minmax: cv::normalize(NORM_MINMAX) of a float map in place.
 * orc_richness_tiles: every view's window of the normalised map (score_tiles),
 * of its threshold at 10 in 8 bits (binary) and the count of 255s (counts);
 * each may be NULL.  Returns 0, or -1 for a window outside the frame. */
void orc_glcm_contrast(const uint8_t* gray, int W, int H, int pitch, float* score);
void orc_normalize_minmax(float* map, size_t n, double lo, double hi);
int orc_richness_tiles(const uint8_t* gray, int W, int H, int pitch, const int* origin, int V, int mi_w, int mi_h,
                       float* score_tiles, uint8_t* binary, uint32_t* counts);

#ifdef __cplusplus
}
#endif
#endif
