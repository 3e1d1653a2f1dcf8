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

int filter_smem_bytes(const CheckFrame& F);
// One wavefront step: the views step_views[0..n_step) filtered in parallel.
cudaError_t launch_filter_step(const CheckFrame& F, const FilterCfg& cfg, const StateDev& st, const int* step_views,
                               int n_step, uint8_t* reason, unsigned long long* stats, cudaStream_t s);
cudaError_t launch_reproj(const CheckFrame& F, const FilterCfg& cfg, const StateDev& st, float* err, cudaStream_t s);

}  // namespace pfd
