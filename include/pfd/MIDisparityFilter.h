/*
 * MIDisparityFilter.h -- cycle-consistency and spike filter of the matched
 * disparities (CheckModule/MIDisparityFilter.h), run on the B200 engine.
 *
 * Same public interface as the reference:
 *   MIDisparityFilterConfig                     :24-57 (same fields and defaults)
 *   MIDisparityFilterStats                      :59-78
 *   MIDisparityFilterCPU(int mi_w, int mi_h, float baseline_unit)   :83
 *   void FilterGlobal(frameName, MLA_info_map, problems_map, dis_normals,
 *                     cfg, out_stats, save_root = "") const         :85-92
 * FilterGlobal filters every micro-image that has a DisparityAndNormal, a
 * gray image and an MLA_Info, in problem-map order and in place (a view sees
 * its neighbours after the views before it were filtered), writes the
 * reference's InvalidatePixel values into dis_normals and fills out_stats,
 * including the whole-frame reprojection-error figures when cfg.dump_disp_error_map
 * is set and save_root is not empty (MIDisparityFilter.cpp:844-950).  The
 * debug images the reference writes under save_root are not produced.
 * Neighbour k of a view is entry k of its m_NeighsSortVecForMatch (or of
 * m_Res_Image_KeyVec when that is empty), as in BuildTileInputsFromMaps
 * (:362-421); only the first 32 can be named by the selected-view masks.
 *
 * The work runs on the calling thread's current CUDA device; no call exits
 * the process.  LastError() is empty after a successful call.
 */
#ifndef PFD_MIDISPARITYFILTER_H
#define PFD_MIDISPARITYFILTER_H

#include <cstdint>
#include <string>

#include "lf_types.h"

namespace LFMVS {

struct MIDisparityFilterConfig {
    int   max_triplet = 4;
    float min_valid_disp = 0.0f;
    bool  use_selected_views_only = true;
    bool  clear_selected_views_when_invalid = true;
    bool  enable_cost_filter = true;
    float max_cost = 1.8f;
    bool  enable_cycle_geo_filter = true;
    float max_geo_err_px = 0.5f;
    bool  enable_cycle_photo_filter = true;
    float max_photo_err_u = 0.5f;
    int   min_good_neighbors = 2;
    bool  enable_spike_filter = true;
    float spike_abs_diff = 1.0f;
    int   spike_min_neighbors = 3;
    bool  dump_debug_mask = true;
    bool  dump_disp_error_map = true;
    float disp_error_thresh_px = 0.5f;
    float disp_error_vis_max_px = 2.0f;
};

struct MIDisparityFilterStats {
    int64_t total_pixels = 0;
    int64_t initially_valid_pixels = 0;
    int64_t kept_pixels = 0;
    int64_t removed_pixels = 0;
    int64_t removed_by_cost = 0;
    int64_t removed_by_no_support = 0;
    int64_t removed_by_cycle = 0;
    int64_t removed_by_spike = 0;
    int64_t num_disp_error_samples = 0;
    int64_t num_disp_error_le_thresh = 0;
    double  mean_disp_error_px = 0.0;
    double  rmse_disp_error_px = 0.0;
    double  p90_disp_error_px = 0.0;
};

class MIDisparityFilterCPU {
public:
    MIDisparityFilterCPU(int mi_w, int mi_h, float baseline_unit);

    void FilterGlobal(const std::string& frameName, const QuadTreeTileInfoMap& MLA_info_map,
                      const QuadTreeProblemMap& problems_map, QuadTreeDisNormalMap& dis_normals,
                      const MIDisparityFilterConfig& cfg, MIDisparityFilterStats& out_stats,
                      const std::string& save_root = "") const;

    /* Not in the reference: why the last FilterGlobal did nothing ("" = it ran). */
    const std::string& LastError() const { return m_last_error; }

private:
    static float QuantileFromSorted(const std::vector<float>& sorted_vals, float q);

    const int   W_;
    const int   H_;
    const float baseline_unit_;
    mutable std::string m_last_error;
};

}  // namespace LFMVS

#endif
