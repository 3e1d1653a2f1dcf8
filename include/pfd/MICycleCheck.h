/*
 * MICycleCheck.h -- read-only cycle-consistency check of the matched
 * disparities with global statistics (CheckModule/MICycleCheck.h), run on the
 * B200 engine.
 *
 * Same public interface as the reference:
 *   MICycleCheckStats, MICycleMaskParams, MICycleClampConfig    :24-78
 *   MICycleCheckerCPU(int mi_w, int mi_h, float baseline_unit)  :83
 *   void CheckGlobal(frameName, MLA_info_map, problems_map, dis_normals,
 *                    out_stats, max_triplet = 4, dump_heatmap = true,
 *                    save_root = "CycleCheck", dump_hist = true, hist_bins = 60,
 *                    hist_geo_max_x = 2.0, vis_geo_max_px = 2.0,
 *                    vis_photo_max = 3.0, ccfg = MICycleClampConfig()) const  :85-100
 * CheckGlobal checks every micro-image that has a DisparityAndNormal, a gray
 * image and an MLA_Info, in problem-map order, and folds the statistics in
 * that order as MICycleCheck.cpp:727-893 does.  The heat maps, histograms and
 * logs the reference writes are not produced (the dump and visualisation
 * arguments are accepted and ignored), nor is VisualizeRandomMatchesGlobal.
 * skip_on_geo / skip_on_photo are accepted and, as in the reference's
 * CheckTile, have no effect.  The texture mask uses the reference's fixed
 * Sobel 8 / variance 60 thresholds (MICycleCheck.cpp:317-322).
 *
 * The work runs on the calling thread's current CUDA device; no call exits
 * the process.  LastError() is empty after a successful call.
 */
#ifndef PFD_MICYCLECHECK_H
#define PFD_MICYCLECHECK_H

#include <cstdint>
#include <string>

#include "lf_types.h"

namespace LFMVS {

struct MICycleCheckStats {
    double  mean_geo_err_px = 0.0;
    double  median_geo_err_px = 0.0;
    double  p90_geo_err_px = 0.0;
    double  mean_photo_err = 0.0;
    int     num_samples = 0;
    double  rmse_geo_err_px = 0.0;
    double  rmse_photo_err = 0.0;
    double  completeness = 0.0;
    double  completeness_geo = 0.0;
    double  completeness_photo = 0.0;
    int64_t completeness_masked_pixels = 0;
    int64_t completeness_good_pixels = 0;
    int64_t completeness_good_pixels_geo = 0;
    int64_t completeness_good_pixels_photo = 0;
};

struct MICycleMaskParams {
    double sobel_thresh = 8.0;
    double var_thresh = 60.0;
    bool   use_and = true;
    int    grad_hist_bins = 50;
    double grad_hist_max = 50.0;
};

struct MICycleClampConfig {
    bool   clamp_photo = true;
    double photo_u = 3.0;
    bool   clamp_geo = false;
    double geo_u_px = 2.0;
    bool   skip_on_geo = false;
    double skip_geo_u_px = 8.0;
    bool   skip_on_photo = false;
    double skip_photo_u = 10.0;
    bool   pixel_gate_enabled = false;
    int    gate_min_good_neighbors = 3;
    double gate_geo_px = 2.0;
    double gate_photo_u = 3.0;
    bool   gate_use_clamped = false;
};

class MICycleCheckerCPU {
public:
    MICycleCheckerCPU(int mi_w, int mi_h, float baseline_unit);

    void CheckGlobal(const std::string& frameName, const QuadTreeTileInfoMap& MLA_info_map,
                     QuadTreeProblemMap& problems_map, QuadTreeDisNormalMap& dis_normals,
                     MICycleCheckStats& out_stats, int max_triplet = 4, bool dump_heatmap = true,
                     const std::string& save_root = "CycleCheck", bool dump_hist = true, int hist_bins = 60,
                     double hist_geo_max_x = 2.0, double vis_geo_max_px = 2.0, double vis_photo_max = 3.0,
                     const MICycleClampConfig& ccfg = MICycleClampConfig()) const;

    /* Not in the reference: the texture-masked figures CheckGlobal logs
     * (MICycleCheck.cpp:834-880) from the last call, and why it did nothing
     * ("" = it ran). */
    struct MaskedFigures {
        int64_t masked_count = 0, all_count = 0;
        double  geo_mean = 0, photo_mean = 0, geo_rmse = 0, photo_rmse = 0, coverage = 0;
        double  geo_median_approx = 0, geo_p90_approx = 0, geo_min = 0, geo_max = 0;
    };
    const MaskedFigures& LastMaskedFigures() const { return m_masked; }
    const std::string& LastError() const { return m_last_error; }

private:
    const int   W_, H_;
    const float m_baseline_unit;
    mutable MaskedFigures m_masked;
    mutable std::string m_last_error;
};

}  // namespace LFMVS

#endif
