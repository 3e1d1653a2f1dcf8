// check_kernels.h -- device side of the consistency pass (check_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_device.cuh"

namespace pfd {

// Reject reasons and counters of MIDisparityFilterCPU (CheckModule/MIDisparityFilter.h:59-109).
constexpr uint8_t kPrKeep = 0, kPrCost = 80, kPrNoSupport = 140, kPrCycle = 200, kPrSpike = 255;
enum { kFsTotal = 0, kFsValidIn, kFsKept, kFsRemoved, kFsCost, kFsNoSupport, kFsCycle, kFsSpike };

// MIDisparityFilterConfig (MIDisparityFilter.h:24-57), same layout as pfd_filter_cfg.
struct FilterCfg {
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
};

struct CheckFrame {
    int V, W, H, K, tile_stride;
    const uint8_t* gray;       // [V][tile_stride]
    const float2* centers;
    const int* nb_ids;
    const int* nb_counts;
    float baseline_unit;       // LightFieldParams::baseline (lens pitch)
};

// MICycleClampConfig + MICycleMaskParams (CheckModule/MICycleCheck.h:44-78), same
// layout as pfd_cycle_cfg; the reference's doubles are cast to float at every use.
struct CycleCfg {
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
};

// Per-micro-image results of CheckTile (MICycleCheck.cpp:541-600): the sums
// the host folds, in key order, into MICycleCheckStats.  Each double sum runs
// over the tile's samples in pixel order, as the reference's std::vector does.
struct CycleTileRec {
    double sum_geo, sq_geo, sum_photo, sq_photo;              // all samples
    double sum_geo_m, sq_geo_m, sum_photo_m, sq_photo_m;      // samples under the texture mask
    int n, n_masked;
    int comp_total, comp_good, comp_good_geo, comp_good_photo;
    float min_geo_m, max_geo_m;                                // over finite masked samples >= 0
};
constexpr int kCycleHistBins = 128;                           // 0.5 px bins of masked geometric error

int cycle_smem_bytes(const CheckFrame& F);
cudaError_t launch_cycle(const CheckFrame& F, const CycleCfg& cfg, const StateDev& st, float* geo_err, float* pho_err,
                         uint8_t* texmask, CycleTileRec* recs, unsigned int* hist, cudaStream_t s);

int filter_smem_bytes(const CheckFrame& F);
// One wavefront step: the views step_views[0..n_step) filtered in parallel.
cudaError_t launch_filter_step(const CheckFrame& F, const FilterCfg& cfg, const StateDev& st, const int* step_views,
                               int n_step, uint8_t* reason, unsigned long long* stats, cudaStream_t s);
cudaError_t launch_reproj(const CheckFrame& F, const FilterCfg& cfg, const StateDev& st, float* err, cudaStream_t s);

}  // namespace pfd
