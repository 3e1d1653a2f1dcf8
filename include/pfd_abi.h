/*
 * pfd_abi.h -- C ABI of the B200 plenoptic depth engine (libpfd.so).
 *
 * The engine replaces the GPU half of the reference's micro-image matching
 * path.  In fengyunxuan6/plenoptic-for-depth that path is
 *   MIStereoMatch::StereoMatchingForMIA_FrameCrossViews (MIStereo/MIStereoMatch.cpp:626-696)
 *     -> AdaptMIPMFrame::Initialize / RunPatchMatchCUDAForFrame /
 *        WriteBackResults / ReleaseMemory          (MIStereo/AdaptMIPMFrame.h:23-27)
 *     -> RandomInitializationForFrame, CheckerboardUpdateFrame
 *                                                  (MIStereo/AdaptMIPMFrame.cu:474-995)
 * The C++ classes that keep the reference's signatures (AdaptMIPMFrame,
 * MIStereoMatch; include/pfd/) sit on top of these functions.
 *
 * Conventions
 *  - Every function returns a pfd_status: 0 on success, a negative PFD_E* code
 *    otherwise; pfd_last_error() describes the last failure of a context.
 *    Nothing here exits the process or resets the device (the reference's
 *    CudaSafeCall exits, Common/CommonCUDA.cpp:77-86, and DepthSolver resets
 *    the device every frame, DepthSolver.cpp:371).
 *  - The caller owns every host buffer; the library owns the device state of
 *    each frame until pfd_frame_free or pfd_destroy.
 *  - One context per host thread.  Work is ordered on the context's stream;
 *    functions that return host data synchronise that stream.
 *  - Micro-image ("view") order is the caller's: the reference uses the
 *    problem-map order, tile keys ascending by (row, column)
 *    (Common/QuadTree.h:137-148, AdaptMIPMFrame.cpp:152-180).
 */
#ifndef PFD_ABI_H
#define PFD_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfd_ctx pfd_ctx;
typedef int pfd_status;

#define PFD_OK           0
#define PFD_EINVAL      -1   /* bad argument, size or parameter */
#define PFD_ENOMEM      -2   /* device allocation failed or the context's HBM budget is exhausted */
#define PFD_ECUDA       -3   /* a CUDA runtime call failed */
#define PFD_ENOFRAME    -4   /* unknown frame id */
#define PFD_ETIMEDOUT   -5   /* a bounded device wait gave up */
#define PFD_ENODEV      -6   /* no such CUDA device */
#define PFD_ESTATE      -7   /* call out of order (e.g. a sweep before initialisation) */

/* Longest neighbour list of a view: selected-view masks are 32 bits. */
#define PFD_MAX_NEIGHBORS 32

/* Matching parameters: the fields of PatchMatchParamsLF (MVStereo/LFDepthInfo.h:19-46)
 * that the frame path reads, as AdaptMIPMFrame::InitGPUParamsFromCPUParams sets
 * them (AdaptMIPMFrame.cpp:126-143). */
typedef struct {
    int   max_iterations;    /* red-black iterations (3 in the reference) */
    int   patch_size;        /* odd NCC patch side */
    int   radius_increment;  /* tap stride inside the patch (1) */
    int   top_k;             /* views averaged by the initial cost (5) */
    float sigma_spatial;     /* bilateral spatial sigma (> 0) */
    float sigma_color;       /* bilateral colour sigma (> 0) */
    float depth_min;         /* disparity search range: 0 ... */
    float depth_max;         /* ... baseline / 2 */
    float base;              /* lens pitch in pixels (LightFieldParams::baseline) */
} pfd_pm_params;

/* ---- context ------------------------------------------------------------ */

/* Opens a context on CUDA device `device` (-1: the calling thread's current
 * device, the one cudaSetDevice chose) with its own stream.  hbm_budget_bytes
 * caps the device memory the context's frames may hold (0 = no cap). */
pfd_status pfd_create(pfd_ctx** out, int device, size_t hbm_budget_bytes);
/* Frees every frame and the context.  Safe on NULL. */
void pfd_destroy(pfd_ctx* ctx);
/* Text of the context's last failure ("" if none).  Valid until the next call. */
const char* pfd_last_error(pfd_ctx* ctx);
/* The context's cudaStream_t, for callers that time or order work around it. */
void* pfd_stream(pfd_ctx* ctx);
/* Waits for the context's stream; reports any device-side error flag. */
pfd_status pfd_sync(pfd_ctx* ctx);
/* Device memory currently held by the context: its frames and the sweep's
 * cudaMalloc'd cost-vector scratch. */
size_t pfd_bytes_in_use(pfd_ctx* ctx);

/* ---- frames ---------------------------------------------------------------
 * Replaces AdaptMIPMFrame::Initialize (AdaptMIPMFrame.cpp:329-335):
 * BuildViewIndexMap (:145-222) becomes the caller's arrays, InitializeGPU's
 * texture objects and state buffers (:278-327) become the frame's device state.
 *
 *   raw        8-bit grayscale frame, W x H, row pitch raw_pitch bytes
 *              (BGR2GRAY of the reference's raw is exact for gray input)
 *   centers    [n_views][2] lens centres in raw pixels (MLA_Info::GetCenter)
 *   tilekeys   [n_views][2] (column, row) tile keys; used by the consistency pass
 *   mi_w, mi_h matching window, floor(pitch * 0.7071) (Common/Common.cpp:34-38);
 *              view v's window starts at trunc(center - (mi - 1) / 2)
 *              (DepthSolver.cpp:1894-1895), and must lie inside the frame
 *   nb_ids     [n_views][max_nb] neighbour view ids in matching order, -1 padded
 *              (m_NeighsSortVecForMatch, AdaptMIPMFrame.cpp:207-218)
 *   nb_counts  [n_views], each <= max_nb <= 32
 *   blur       optional [n_views][mi_h][mi_w] 8-bit blur channel
 *              (MLA_Problem::m_Image_Blureness); NULL = no blur penalty
 */
pfd_status pfd_frame_create(pfd_ctx* ctx, int* frame_id, int W, int H,
                            const float* centers, const int* tilekeys, int n_views,
                            int mi_w, int mi_h, const int* nb_ids, const int* nb_counts,
                            int max_nb, const uint8_t* blur);
/* Copies a raw frame from host memory and slices the micro-images
 * (Slice_RawMLAImage, DepthSolver.cpp:1951-1997). */
pfd_status pfd_frame_set_raw(pfd_ctx* ctx, int frame_id, const uint8_t* raw, int raw_pitch);
/* Same, from a raw frame already in this device's memory. */
pfd_status pfd_frame_set_raw_device(pfd_ctx* ctx, int frame_id, const uint8_t* raw_dev, int raw_pitch);
/* Fills the micro-images directly, for callers that hold them already sliced:
 * MLA_Problem::m_Image_gray of every view, the images
 * AdaptMIPMFrame::BuildViewIndexMap (AdaptMIPMFrame.cpp:126-215) collects and
 * CreateGrayImageObject (:217-245) binds to textures.  images [n_views][mi_h][mi_w],
 * views in frame order.  The frame then has no raw image (pfd_refocus needs one).
 * Returns when the host buffer may be reused. */
pfd_status pfd_frame_set_micro_images(pfd_ctx* ctx, int frame_id, const uint8_t* images);
/* The blur channel computed on the device from the frame's raw image:
 * ImageQualityEstimate::QuantizeBlurByLaplacian (Util/ImageQualityEstimate.cpp:
 * 211-230) then DepthSolver::SliceAndIndicatlizeForMI (DepthSolver.cpp:
 * 2709-2754).  Every view's blur tile becomes the raw frame's Laplacian (ksize
 * 1, borders reflected without repeating the edge) over its window, saturated
 * to 8 bits (MLA_Problem::m_Image_Blureness); it replaces any blur channel given
 * to pfd_frame_create, and the frame's costs carry the blur penalty from then
 * on.  blur_out [n_views][mi_h][mi_w] (may be NULL) receives the channel;
 * blureness [n_views] (may be NULL) MLA_Problem::m_BlurenessValue, the window's
 * pixels whose Laplacian exceeds 10 (ComputeBlurenessValue,
 * MVStereo/LFDepthInfo.cpp:65-83).  With either output the call waits for the
 * device.  Needs a raw frame (pfd_frame_set_raw); the PatchMatch state must be
 * initialised again afterwards. */
pfd_status pfd_frame_compute_blur(pfd_ctx* ctx, int frame_id, uint8_t* blur_out, uint32_t* blureness);
/* The richness channel computed on the device from the frame's raw image:
 * ImageQualityEstimate::QuantizeRichnessByGLCM (Util/ImageQualityEstimate.cpp:
 * 310-340, calculate_matrix :659-682) then DepthSolver::SliceAndIndicatlizeForMI
 * (DepthSolver.cpp:2709-2754).  The frame's map holds, at every pixel with
 * 4 <= row < H - 4 and 4 <= col < W - 4, the contrast of the 3-bit GLCM of
 * diagonal neighbours in the 8x8 window at (col - 4, row - 4), 0 elsewhere,
 * normalised by cv::normalize(0, 255, NORM_MINMAX) over the frame.  Outputs,
 * each [n_views] windows in frame order and each may be NULL:
 *   score_out  [n_views][mi_h][mi_w] the normalised map's window
 *              (DepthSolver::GetRichnessScoreMI, :2307-2326);
 *   binary_out [n_views][mi_h][mi_w] 255 where it exceeds 10, else 0
 *              (MLA_Problem::m_Image_Richness);
 *   richness   [n_views] the window's 255s (MLA_Problem::m_RichnessValue,
 *              ComputeRichnessValue, MVStereo/LFDepthInfo.cpp:86-104).
 * The matcher does not read the channel (SelectNeighbors weighs richness by 0),
 * so the frame keeps no copy and its PatchMatch state is untouched.  Waits for
 * the device.  Needs a raw frame (pfd_frame_set_raw). */
pfd_status pfd_frame_compute_richness(pfd_ctx* ctx, int frame_id, float* score_out, uint8_t* binary_out,
                                      uint32_t* richness);
/* pfd_frame_create + pfd_frame_set_raw. */
pfd_status pfd_frame_upload(pfd_ctx* ctx, int* frame_id, const uint8_t* raw, int W, int H, int raw_pitch,
                            const float* centers, const int* tilekeys, int n_views,
                            int mi_w, int mi_h, const int* nb_ids, const int* nb_counts,
                            int max_nb, const uint8_t* blur);
/* Releases a frame's device memory (AdaptMIPMFrame::ReleaseMemory, AdaptMIPMFrame.cpp:53-124). */
pfd_status pfd_frame_free(pfd_ctx* ctx, int frame_id);

/* ---- PatchMatch ------------------------------------------------------------
 * Replaces AdaptMIPMFrame::RunPatchMatchCUDAForFrame (AdaptMIPMFrame.cpp:343-357,
 * AdaptMIPMFrame.cu:949-995): random initialisation, then max_iterations x
 * (red half-sweep, black half-sweep), enqueued without host synchronisation.
 * seed keys the Philox streams (the reference seeds cuRAND from clock64()). */
pfd_status pfd_patchmatch(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed);
/* pfd_patchmatch of n frames of the context at once (no counterpart in the
 * reference, which matches one frame at a time): every frame is initialised,
 * then each half-sweep is ONE persistent launch over all the frames that still
 * have iterations left (one launch per group of frames that share a blur
 * channel and whose own shared-memory plans allow the same CTAs per SM, so no
 * frame runs at a larger frame's occupancy), in which a CTA that finds one frame's micro-images all taken
 * moves straight on to the next frame, so small frames and the tails of large
 * ones do not leave the GPU idle between launches.  params[b] and seeds[b] are
 * frame b's own (sizes, neighbour counts, patch sizes and iteration counts may
 * all differ); every frame's result is bit for bit what pfd_patchmatch gives it
 * alone.  A frame whose micro-images fill the sweep's grid four times over or
 * more runs as pfd_patchmatch (measured slower inside a shared launch); the
 * others share launches.  Tap counting (pfd_set_tap_counting) runs the frames
 * one by one. */
pfd_status pfd_patchmatch_batch(pfd_ctx* ctx, const int* frame_ids, int n, const pfd_pm_params* params,
                                const uint64_t* seeds);
/* CUDA graphs for the context's later pfd_patchmatch calls and enqueue-only
 * pfd_filter calls (reason and stats NULL); no counterpart in the reference,
 * which launches and synchronises kernel by kernel.  Per frame, the first call
 * with a given key (the call's arguments and the context's matcher, moment
 * mode, sweep shape and sweep fetch) runs as usual, which sizes the scratch and tunes the
 * launch shape; the second is captured into a graph; later calls replay it.
 * A graph reads and writes the frame's buffers in place, so new raw data and
 * new neighbour lists are picked up; a new key, new neighbour lists (for the
 * filter) or moved sweep scratch make the next call run uncaptured again.
 * Results are the same bit for bit with graphs on or off. */
pfd_status pfd_set_graphs(pfd_ctx* ctx, int on);
/* The steps of pfd_patchmatch, separately: RandomInitializationForFrame
 * (AdaptMIPMFrame.cu:474-518) and one CheckerboardUpdateFrame launch (:520-947). */
pfd_status pfd_pm_init(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed);
pfd_status pfd_pm_sweep(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed,
                        int iter, int phase);
/* pfd_pm_sweep without any device allocation; no counterpart in the reference.
 * For callers that cannot allocate device memory once frames are streaming: an
 * application whose memory pool claimed all free HBM at start-up, or a
 * real-time loop that forbids cudaMalloc/cudaFree because they can synchronise
 * the whole device.  The cost-vector scratch is a fixed 8 MiB array in the
 * library's device image (held by every GPU that loads the library, until
 * exit) instead of a cudaMalloc'd buffer; inputs and outputs are the frame's
 * state exactly as for pfd_pm_sweep, and the results are the same bit for bit.
 * Limit: the array must hold one CTA's scratch (seven warps, each the cost
 * vectors of one pixel) for every SM: every max_nb up to 32 fits on a 148-SM
 * B200; a device with more SMs than the array holds CTAs gets PFD_EINVAL.
 * Every call looks up the array's device address (cudaGetSymbolAddress, a
 * host-side lookup), so the address stays right after a cudaDeviceReset; the
 * first call on a device may also load the library's device code there, so
 * make that call before any stream capture.  All calls on a device share the one
 * array (nothing in it has to start at zero): calls whose kernels overlap on
 * the GPU, from other streams or other contexts, race and corrupt each other. */
pfd_status pfd_pm_sweep_noalloc(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, uint64_t seed,
                                int iter, int phase);

/* How the NCC moments are accumulated by the context's later pfd_pm_init,
 * pfd_pm_sweep(_noalloc), pfd_patchmatch and pfd_ncc_costs calls.
 * PFD_NCC_REFERENCE (the default): the reference's FP32 sums of w r, w r^2,
 * w s, w s^2 and w r s (ComputeBilateralNCC_Frame, AdaptMIPMFrame.cu:110-174)
 * in the oracle's IEEE canonical arithmetic, bit for bit with the oracle (the
 * reference's fast-math build differs in the last bits); their variances E[r^2] - E[r]^2 lose digits to cancellation on
 * patches of low contrast.  PFD_NCC_SHIFTED: the same FP32 sums of the texels
 * and samples minus the patch's centre texel (exact subtractions: both are
 * multiples of 1/256 below 2^16); the NCC is unchanged in exact arithmetic
 * and its FP32 error against an FP64 evaluation is far smaller.  Not in the
 * reference: results differ from its bits. */
#define PFD_NCC_REFERENCE 0
#define PFD_NCC_SHIFTED   1
pfd_status pfd_set_ncc_moments(pfd_ctx* ctx, int mode);

/* The PatchMatch rules of the context's later pfd_pm_init, pfd_pm_sweep(_noalloc),
 * pfd_patchmatch and pfd_ncc_costs calls.
 * PFD_MATCHER_FRAME (the default): AdaptMIPMFrame (MIStereo/AdaptMIPMFrame.cu).
 * PFD_MATCHER_ACMM: one pyramid level of AdaptMIPMFrameACMM
 * (MIStereo/AdaptMIPMFrameACMM.cu), the matcher MIStereoMatch::
 * StereoMatchingForMIA_FrameCrossViews_ACMM runs (MIStereoMatch.cpp:698-740):
 * the same initialisation and half-sweeps with a blur penalty gain of 0.8
 * instead of 2 (:99), and each updated pixel stores the mean of the top_k
 * lowest costs of its final plane over every view, those views as its
 * selected-view mask and the lowest-cost view's disp (RecomputeSupportCostDisp_
 * Frame, :259-280, called at :890); pfd_patchmatch then ends with
 * pfd_acmm_post_refine.  The matcher builds its two-level pyramid only for
 * windows of 24 pixels and more (AdaptMIPMFrameACMM.cpp:312-321); the coarse
 * level and the warm start are not provided here: this is the matcher at one
 * level, which is all of it for windows below 24 pixels (pitch < 34 px).
 * The caller passes the level's parameters (the reference uses patch 5,
 * 5 iterations and top_k 6 at one level, :155-180). */
#define PFD_MATCHER_FRAME 0
#define PFD_MATCHER_ACMM  1
pfd_status pfd_set_matcher(pfd_ctx* ctx, int matcher);
/* Launch shape of the context's later half-sweeps (pfd_pm_sweep, pfd_patchmatch,
 * pfd_patchmatch_batch; no counterpart in the reference, whose sweep is one
 * thread per pixel in 16x16 blocks).  A shape is a number of warps per CTA and
 * the CTAs per SM its registers are sized for; every shape computes the same
 * state bit for bit.  Shape 0 (7 warps, 4 CTAs) is the default.
 * PFD_SHAPE_AUTOTUNE: the engine's autotuner picks the shape per key (window,
 * neighbour count, patch size and tap stride, blur channel, moment mode,
 * matcher) and device: the first half-sweep of a new key runs once in every
 * shape that fits the key's shared-memory plan, timed on the context's stream
 * (the stored cost vectors are neither read nor written by these trials, so
 * each writes the half-sweep's result), and the fastest is kept for the rest
 * of the process.  pfd_patchmatch_batch uses the shape of each launch's
 * largest frame.  Tap counting and pfd_pm_sweep_noalloc always run shape 0. */
#define PFD_SWEEP_SHAPES 4
#define PFD_SHAPE_AUTOTUNE -1
pfd_status pfd_set_sweep_shape(pfd_ctx* ctx, int shape);
/* Warps per CTA and CTAs per SM of shape 0 .. PFD_SWEEP_SHAPES - 1. */
pfd_status pfd_sweep_shape_info(int shape, int* warps_per_cta, int* ctas_per_sm);
/* The shape the autotuner chose for the key of (frame, params), or -1 when the
 * key has not been tuned in this process. */
pfd_status pfd_tuned_sweep_shape(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params, int* shape);
/* Where the context's later half-sweeps read neighbour samples.
 * PFD_FETCH_SHARED (the default): from the micro-image and its neighbours
 * staged in shared memory, blended as the texture unit does.
 * PFD_FETCH_TEXTURE: from the frame's micro-images held as layered float
 * textures with the reference's filter settings (linear filter, unnormalised
 * coordinates; AdaptMIPMFrame.cpp:224-249 makes one texture per micro-image),
 * one tex2DLayered fetch per tap as the reference's tex2D.  The textures (4
 * bytes per micro-image pixel and channel) are created at the frame's first
 * sweep under this mode (pfd_pm_sweep_noalloc creates none: it fetches from
 * textures only where they exist) and refilled, one launch, before the first
 * sweep after new tiles.  Both modes give the same state bit for bit; the
 * texture fetches measure slower on B200.  Tap counting always stages in
 * shared memory. */
#define PFD_FETCH_TEXTURE 0
#define PFD_FETCH_SHARED  1
pfd_status pfd_set_sweep_fetch(pfd_ctx* ctx, int mode);

/* PostRefineMetadataFrame (AdaptMIPMFrameACMM.cu:903-929): every pixel keeps
 * its plane and gets the cost, selected views and disp of it as the ACMM
 * write-back computes them, under the context's matcher and moment mode. */
pfd_status pfd_acmm_post_refine(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params);

/* Per-hypothesis cost vectors: ComputeMultiViewCostVector_Frame
 * (AdaptMIPMFrame.cu:181-225) for n (view, pixel, plane) hypotheses.
 * vids[n], pxy[n][2] (x, y inside the window), planes[n][4] (nx, ny, nz, d);
 * costs[n][max_nb] receives the costs (2.0 past the view's neighbour count). */
pfd_status pfd_ncc_costs(pfd_ctx* ctx, int frame_id, const pfd_pm_params* params,
                         const int* vids, const int* pxy, const float* planes, int n, float* costs);

/* Copies the frame's current per-pixel state to host buffers, each
 * [n_views * mi_w * mi_h] in view-major, row-major order; any may be NULL.
 * Replaces the device-to-host copies of AdaptMIPMFrame.cpp:352-356 that
 * WriteBackResults (:359-384) scatters into DisparityAndNormal::{ph_cuda,
 * c_cuda, disp_v_cuda, selected_views}. */
pfd_status pfd_download(pfd_ctx* ctx, int frame_id, float* plane /*[.][4]*/, float* cost,
                        float* disp /*[.][4]*/, uint32_t* sel);
/* pfd_download enqueued on the context's stream without waiting: the host
 * buffers (pinned, for the copies to be asynchronous) hold the state once the
 * stream has reached this point (pfd_sync, or an event or host function
 * enqueued on pfd_stream after it).  Device errors show at the next pfd_sync. */
pfd_status pfd_download_async(pfd_ctx* ctx, int frame_id, float* plane, float* cost, float* disp, uint32_t* sel);
/* The inverse of pfd_download: makes host arrays in the same layout the frame's
 * current state, for a consistency pass over results that live on the host
 * (the DisparityAndNormal arrays MIDisparityFilterCPU::FilterGlobal and
 * MICycleCheckerCPU::CheckGlobal read, MIDisparityFilter.cpp:962-986,
 * MICycleCheck.cpp:780-893).  All four are required.  Returns when the host
 * buffers may be reused. */
pfd_status pfd_state_upload(pfd_ctx* ctx, int frame_id, const float* plane /*[.][4]*/, const float* cost,
                            const float* disp /*[.][4]*/, const uint32_t* sel);

/* ---- consistency pass -------------------------------------------------------
 * MIDisparityFilterConfig (CheckModule/MIDisparityFilter.h:24-57).  The values
 * MIStereoMatch::FilterAndStatic passes (MIStereoMatch.cpp:759-778):
 * max_triplet 4, min_valid_disp 0, selected views only, clear views when
 * invalid, cost filter 1.8, geo 0.5 px, photo 0.5, 2 good neighbours, spike
 * filter 1.0 with 3 neighbours. */
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
} pfd_filter_cfg;

/* Reject reasons written to the reason map (MIDisparityFilter.h:102-109). */
#define PFD_PR_KEEP       0
#define PFD_PR_COST       80
#define PFD_PR_NOSUPPORT  140
#define PFD_PR_CYCLE      200
#define PFD_PR_SPIKE      255

/* MIDisparityFilterCPU::FilterGlobal (MIDisparityFilter.cpp:962-986): filters
 * the frame's current PatchMatch state in place, view by view in key order,
 * with the reference's in-place dependency between views kept exactly.
 * baseline_unit is LightFieldParams::baseline.  reason (host, [V*mi_w*mi_h],
 * may be NULL) receives the reject reasons; stats (may be NULL) the counters
 * total, valid_in, kept, removed, by_cost, by_no_support, by_cycle, by_spike. */
pfd_status pfd_filter(pfd_ctx* ctx, int frame_id, const pfd_filter_cfg* cfg, float baseline_unit,
                      uint8_t* reason, long long* stats);
/* ComputeTileReprojectionErrorMap (MIDisparityFilter.cpp:695-842) over the
 * frame: per-pixel median cycle reprojection error (-1 where fewer than
 * min_good_neighbors views support it).  err: host [V*mi_w*mi_h], or NULL to
 * keep the map on the device only. */
pfd_status pfd_reprojection_error(pfd_ctx* ctx, int frame_id, const pfd_filter_cfg* cfg, float baseline_unit,
                                  float* err);

/* MICycleClampConfig (CheckModule/MICycleCheck.h:54-78) and the texture-mask
 * parameters MICycleMaskParams (:44-50).  The reference's doubles are floats
 * here (every use casts them to float); bools are ints. */
typedef struct pfd_cycle_cfg {
    int   max_triplet;              /* selected views checked per pixel (CheckGlobal argument, 4) */
    int   clamp_photo;              /* 1 */
    float photo_u;                  /* 3.0 */
    int   clamp_geo;                /* 1 in MIStereoMatch.cpp:571 */
    float geo_u_px;                 /* 2.0 */
    int   pixel_gate_enabled;       /* 0 */
    int   gate_min_good_neighbors;  /* 2 */
    float gate_geo_px;              /* 0.5 */
    float gate_photo_u;             /* 0.5 */
    int   gate_use_clamped;         /* 0 */
    float sobel_thresh;             /* 8.0 (fixed in CheckTile, MICycleCheck.cpp:317-322) */
    float var_thresh;               /* 60.0 */
    int   use_and;                  /* 1 */
} pfd_cycle_cfg;

/* MICycleCheckStats (MICycleCheck.h:24-42) followed by the texture-masked
 * figures CheckGlobal logs (MICycleCheck.cpp:834-880). */
typedef struct pfd_cycle_stats {
    double    mean_geo_err_px, median_geo_err_px, p90_geo_err_px, mean_photo_err;
    long long num_samples;
    double    rmse_geo_err_px, rmse_photo_err;
    double    completeness, completeness_geo, completeness_photo;
    long long completeness_masked_pixels, completeness_good_pixels, completeness_good_pixels_geo,
              completeness_good_pixels_photo;
    long long masked_count, all_count;
    double    masked_geo_mean, masked_photo_mean, masked_geo_rmse, masked_photo_rmse, coverage;
    double    masked_geo_median_approx, masked_geo_p90_approx, masked_geo_min, masked_geo_max;
} pfd_cycle_stats;

/* MICycleCheckerCPU::CheckGlobal (MICycleCheck.cpp:727-893, tiles by CheckTile
 * :282-725) on the frame's current state; read-only.  stats receives the
 * global figures, folded over the views in key order as the reference does.
 * geo_err / pho_err (host float [V*mi_w*mi_h]) receive the per-pixel maximum
 * geometric and photometric errors, texmask (host u8) the 0/255 texture mask;
 * each may be NULL. */
pfd_status pfd_cycle_check(pfd_ctx* ctx, int frame_id, const pfd_cycle_cfg* cfg, float baseline_unit,
                           pfd_cycle_stats* stats, float* geo_err, float* pho_err, uint8_t* texmask);
/* With stats and all three maps NULL, pfd_cycle_check only enqueues the check
 * (no synchronisation), and this folds its statistics later, e.g. after the
 * filter and the render are enqueued behind it, so the device does not wait
 * for the host fold.  Valid until the frame's next cycle check. */
pfd_status pfd_cycle_check_stats(pfd_ctx* ctx, int frame_id, pfd_cycle_stats* stats);

/* ---- focal stack ----------------------------------------------------------
 * Renders n_slices refocused images of out_w x out_h from the frame's gray
 * micro-images.  The reference has no multi-slice render; this one is built
 * on its back-projection LFRefocus::BackProject2MI (FocalStack/LFRefocus.cpp:
 * 2119-2125): output pixel (ox, oy) of slice s sits at raw coordinates
 * X = (ox + 0.5) * (W / out_w) - 0.5 (Y likewise), micro-image i sees it at
 * u = (X - c_i) / slice_vd[s] + ((m-1)/2 + 1) (the micro-image centre of
 * FuseVirtualDepth_BackProject, :1635-1636), and every micro-image with u in
 * [0, m-1]^2 contributes its bilinear sample; the pixel is their mean (0 when
 * none), summed in view order.  The stack stays on the device; out (host,
 * float [n_slices][out_h][out_w]) receives a copy unless it is NULL. */
pfd_status pfd_refocus(pfd_ctx* ctx, int frame_id, const float* slice_vd, int n_slices, int out_w, int out_h,
                       float* out);

/* ---- matching-neighbour selection -----------------------------------------
 * SelectNeighbors::CollectMIANeighImagesForMatch (MINeighbor/SelectNeighbors.cpp:
 * 113-193) for every micro-image: up to five rings of lenses found by the
 * reference's walk over the key grid, each candidate scored by
 * MISimilarityMeasure::MeasureSimilarity (Util/MISimilarityMeasure.cpp:173-284,
 * computed on the device for every candidate), candidates rejected by the RANSAC
 * line fitted at the third ring (MVStereo/LFDepthInfo.cpp:136-211), the search
 * stopped at a ring with two or more outliers, and the survivors sorted by the
 * normalised baseline score (SelectNeighbors.cpp:770-832, LFDepthInfo.cpp:214-241):
 * m_NeighsSortVecForMatch.
 *   centers [n][2], tilekeys [n][2] (column, row) inside mla_u_size x mla_v_size
 *   images  [n][mi_h][mi_w] gray micro-images (MLA_Problem::m_Image_gray)
 *   nb_ids  [n][max_nb] view ids best first (-1 padded), nb_counts [n] (<= max_nb <= 128) */
pfd_status pfd_select_neighbors(pfd_ctx* ctx, const float* centers, const int* tilekeys, int n_views, int mla_u_size,
                                int mla_v_size, float pitch, const uint8_t* images, int mi_w, int mi_h, int max_nb,
                                int* nb_ids, int* nb_counts);
/* The same selection for a frame's own micro-images (the gray tiles cut on
 * the device from its raw image, or uploaded), which then becomes the frame's
 * matching lists: the first max_nb (the frame's) of each view's
 * m_NeighsSortVecForMatch, as AdaptMIPMFrame::BuildViewIndexMap keeps the
 * first entries of that list (AdaptMIPMFrame.cpp:207-218).  The frame's
 * PatchMatch state belongs to its old lists and must be initialised again.
 * nb_ids [n_views][max_list] and nb_counts [n_views] (both NULL, or both
 * given with max_list <= 128) receive the full lists.  Waits for the device. */
pfd_status pfd_frame_select_neighbors(pfd_ctx* ctx, int frame_id, int mla_u_size, int mla_v_size, float pitch,
                                      int max_list, int* nb_ids, int* nb_counts);

/* ---- micro-lens centres -------------------------------------------------
 * DepthSolver::ComputeMLACentersFromWhiteImage (DepthSolver.cpp:710-870) on the
 * device: the reference's Otsu threshold (:486-546, which histograms the first W
 * bytes of every row of the 3-channel image), BGR2GRAY and the binary threshold,
 * the external contours of the 8-connected bright blobs with their polygon
 * moments and areas (as findContours(RETR_EXTERNAL) + moments + contourArea
 * give them), then the reference's position filter, rows by running mean y,
 * columns by x and the small-area flag (area < 0.8 x the mean over all contours).
 * One entry per MLA_Info map key, in key order (row, then column). */
typedef struct {
    int   col, row;          /* the key (QuadTreeTileKey tile x, tile y) */
    float cx, cy;            /* MLA_Info::GetCenter */
    float area;              /* MLA_Info::GetArea (contour area) */
    int   abandon;           /* MLA_Info::IsAbandonByArea */
} pfd_mla_lens;
/* white_bgr: host 3-channel 8-bit image, W x H, rows step bytes apart (a gray
 * image repeated in three channels for a one-channel white image).  baseline,
 * mla_u_size, mla_v_size: LightFieldParams (lens pitch, lenses per row and per
 * column).  n_out receives the entry count; out (room for max_out entries) the
 * entries, or with out NULL only the count.  threshold (may be NULL) receives
 * the Otsu threshold. */
pfd_status pfd_mla_centers(pfd_ctx* ctx, const uint8_t* white_bgr, int W, int H, int step, float baseline,
                           int mla_u_size, int mla_v_size, pfd_mla_lens* out, int max_out, int* n_out,
                           int* threshold);

/* Least-squares hexagonal lattice through detected centres (FP64, normal
 * equations summed on the device): centre(col, row) = origin + (col + (row & 1)
 * / 2) u + row (sqrt(3) / 2) u_perp, u = pitch (cos angle, sin angle).  No
 * counterpart in the reference, which keeps the detected centres as they are;
 * it measures them.  fit: origin x, origin y, pitch, angle (radians), RMS
 * residual (pixels), lenses used.  skip_abandoned: leave out flagged lenses. */
pfd_status pfd_mla_lattice_fit(pfd_ctx* ctx, const pfd_mla_lens* lenses, int n, int skip_abandoned, double fit[6]);

/* ---- virtual-depth fusion ------------------------------------------------
 * LFRefocus::FuseVirtualDepth_BackProject (FocalStack/LFRefocus.cpp:1553-1794):
 * every reference micro-image pixel with disparity >= min_ref_disp becomes a
 * virtual point (ComputeVirtual3D, :2100-2117, at virtual depth mla_base / d,
 * ComputeVirtualDepth :2087-2098); it is back-projected into each micro-image of
 * its list (BackProject2MI, :2119-2125), and a list entry is consistent when
 * that pixel, unmasked and with a disparity > 0, projects back within
 * max_reproj_px at a virtual depth within max_rel_vd.  With min_consistent or
 * more consistent entries the point, normal and colour are averaged, written
 * to the raw-resolution maps at the rounded point position, and the entries'
 * pixels are masked for everything after: micro-images in frame order, pixels
 * row by row, exactly as the reference, whose result depends on that order.
 * The reference's literals are min_ref_disp 1, max_reproj_px 1, max_rel_vd
 * 0.05, min_consistent 2; mla_base = LightFieldParams::baseline * g_bl0 /
 * (g_bl0 + g_B). */
typedef struct {
    float mla_base;
    float min_ref_disp;
    float max_reproj_px;
    float max_rel_vd;
    int   min_consistent;
} pfd_fuse_params;
/* Reads the frame's current state (normal: plane.xyz, disparity: plane.w).
 *   lists        [n_views][max_list] each view's m_NeighsSortVecForMatch as view
 *                ids, -1 for a key with no result (skipped); max_list <= 128
 *   list_counts  [n_views]
 *   is_ref       [n_views] 1 for the micro-images fused as references (not garbage)
 *   bgr          [n_views][mi_h][mi_w][3] colour micro-images (MLA_Problem::
 *                m_Image_rgb), or NULL to use the gray ones in all channels
 * Outputs (host, any may be NULL), W x H of the frame's raw size:
 *   vd_map float (m_VirtualDepthMap), conf u8 (VD_Confidence), aif u8 x 3 BGR
 *   (m_AIF_Color); points [n][9] (point, normal, colour) in the reference's order,
 *   sized by a first call with points NULL and n_points set. */
pfd_status pfd_fuse_virtual_depth(pfd_ctx* ctx, int frame_id, const pfd_fuse_params* params, const int* lists,
                                  const int* list_counts, int max_list, const uint8_t* is_ref, const uint8_t* bgr,
                                  float* vd_map, uint8_t* conf, uint8_t* aif, float* points, long long* n_points);

/* ---- virtual depth to real depth (FP64) -----------------------------------
 * The behavioural model z = (v c1 + c2) / (1 - v c0) of FocalStack/
 * VirtualToRealDepthFunc.cpp and LFRefocus.cpp, in double precision on the
 * device.  vd and the outputs are host arrays of n values. */
/* VirtualToRealDepthFunc::convertVirtualToRealDepth (VirtualToRealDepthFunc.cpp:
 * 3421-3450): double results; NaN, infinite and negative values become 0. */
pfd_status pfd_vd_to_rd_map(pfd_ctx* ctx, const float* vd, size_t n, const double c[3], double* rd);
/* The same on device arrays (enqueued on the context's stream, no synchronisation). */
pfd_status pfd_vd_to_rd_map_device(pfd_ctx* ctx, const float* vd_dev, size_t n, const double c[3], double* rd_dev);
/* LFRefocus::ConvertVdToRd (LFRefocus.cpp:2515-2534) per value: |1 - v c0| < 1e-12,
 * non-finite or negative results give 0; float results. */
pfd_status pfd_vd_to_rd_points(pfd_ctx* ctx, const float* vd, size_t n, const double c[3], float* rd);
/* One depth interval of the segmented model (behaviorModelParamsSegment.xml). */
typedef struct pfd_vd_segment {
    double depth_min, depth_max, c0, c1, c2;
} pfd_vd_segment;
/* LFRefocus::ConvertVdToRdSegment (LFRefocus.cpp:2536-2593): the first segment
 * with depth_min <= v < depth_max applies, 0 when none does; at most 64
 * segments.  The reference re-reads the XML file for every pixel; here the
 * caller passes the segments once. */
pfd_status pfd_vd_to_rd_segments(pfd_ctx* ctx, const float* vd, size_t n, const pfd_vd_segment* segs, int nseg,
                                 float* rd);
/* VirtualToRealDepthFunc::BehavioralModel (VirtualToRealDepthFunc.cpp:3390-3418):
 * least-squares c of [a_L v, v, 1] c = a_L over n >= 3 pairs (a_L = real_depth).
 * The normal-equation sums are formed in FP64 on the device and the 3x3 system
 * is solved on the host (the reference uses cv::solve with SVD; results agree
 * to the system's conditioning). */
pfd_status pfd_fit_behavioral_model(pfd_ctx* ctx, const float* real_depth, const float* vd, size_t n, double c[3]);

/* ---- measurement --------------------------------------------------------
 * No counterpart in the reference (it has no timers or counters on this path,
 * see its Util/Logger only).  Tap counting switches the PatchMatch kernels to
 * a variant that also counts in-bounds NCC taps (reference and source sample
 * both inside their windows): the algorithmic unit of the roofline.  Timed
 * runs leave it off. */
pfd_status pfd_set_tap_counting(pfd_ctx* ctx, int enable);
/* Reads and clears the tap counter (synchronises the stream). */
pfd_status pfd_read_tap_count(pfd_ctx* ctx, unsigned long long* taps);
/* Number of kernels this context has launched so far (every engine kernel). */
pfd_status pfd_launch_count(pfd_ctx* ctx, unsigned long long* n);

#ifdef __cplusplus
}
#endif
#endif /* PFD_ABI_H */
