// MICycleCheck.cpp -- MICycleCheckerCPU::CheckGlobal (CheckModule/MICycleCheck.cpp:
// 727-893) over the engine's C ABI.  Read-only: the maps are not changed.
#include "../../include/pfd/MICycleCheck.h"

#include <cstdio>

#include "../../include/pfd_abi.h"
#include "frame_views.h"

namespace LFMVS {

MICycleCheckerCPU::MICycleCheckerCPU(int mi_w, int mi_h, float baseline_unit)
    : W_(mi_w), H_(mi_h), m_baseline_unit(baseline_unit)
{
}

void MICycleCheckerCPU::CheckGlobal(const std::string& frameName, const QuadTreeTileInfoMap& MLA_info_map,
                                    QuadTreeProblemMap& problems_map, QuadTreeDisNormalMap& dis_normals,
                                    MICycleCheckStats& out_stats, int max_triplet, bool /*dump_heatmap*/,
                                    const std::string& /*save_root*/, bool /*dump_hist*/, int /*hist_bins*/,
                                    double /*hist_geo_max_x*/, double /*vis_geo_max_px*/,
                                    double /*vis_photo_max*/, const MICycleClampConfig& ccfg) const
{
    out_stats = MICycleCheckStats{};
    m_masked = MaskedFigures{};
    m_last_error.clear();
    auto fail = [&](const std::string& why) {
        m_last_error = why;
        std::fprintf(stderr, "[MICycleCheck] frame=%s: %s\n", frameName.c_str(), why.c_str());
    };

    pfd_host::CheckViews views;
    std::string err;
    if (!pfd_host::build_check_views(MLA_info_map, problems_map, dis_normals, W_, H_, &views, &err)) return fail(err);
    const int V = (int)views.keys.size();
    if (V == 0) return;
    const size_t ppv = (size_t)W_ * H_, n = (size_t)V * ppv;

    // The checker reads ph.w as the disparity, with no fallback to d
    // (MICycleCheck.cpp:337, :365).
    std::vector<float4> plane(n), disp(n);
    std::vector<float> cost(n);
    std::vector<uint32_t> sel(n);
    for (int v = 0; v < V; ++v) {
        const DisparityAndNormal& dn = *views.dns[v];
        for (size_t i = 0; i < ppv; ++i) {
            plane[v * ppv + i] = dn.ph_cuda[i];
            cost[v * ppv + i] = dn.c_cuda[i];
            disp[v * ppv + i] = dn.disp_v_cuda[i];
            sel[v * ppv + i] = dn.selected_views[i];
        }
    }

    // The reference's doubles are used as floats by every comparison in
    // CheckTile; the texture mask thresholds are fixed there (:317-322).
    pfd_cycle_cfg c;
    c.max_triplet = max_triplet;
    c.clamp_photo = ccfg.clamp_photo;
    c.photo_u = (float)ccfg.photo_u;
    c.clamp_geo = ccfg.clamp_geo;
    c.geo_u_px = (float)ccfg.geo_u_px;
    c.pixel_gate_enabled = ccfg.pixel_gate_enabled;
    c.gate_min_good_neighbors = ccfg.gate_min_good_neighbors;
    c.gate_geo_px = (float)ccfg.gate_geo_px;
    c.gate_photo_u = (float)ccfg.gate_photo_u;
    c.gate_use_clamped = ccfg.gate_use_clamped;
    const MICycleMaskParams mcfg;
    c.sobel_thresh = (float)mcfg.sobel_thresh;
    c.var_thresh = (float)mcfg.var_thresh;
    c.use_and = mcfg.use_and;

    pfd_host::ScopedContext ctx;
    if (ctx.open() != PFD_OK) return fail("cannot open an engine context on the current device");
    int fid = 0;
    if (pfd_host::create_check_frame(ctx.ctx, views, W_, H_, &fid, &err) != PFD_OK) return fail(err);
    pfd_cycle_stats st;
    pfd_status s = pfd_state_upload(ctx.ctx, fid, &plane[0].x, cost.data(), &disp[0].x, sel.data());
    if (s == PFD_OK) s = pfd_cycle_check(ctx.ctx, fid, &c, m_baseline_unit, &st, nullptr, nullptr, nullptr);
    if (s != PFD_OK) return fail(pfd_last_error(ctx.ctx));

    out_stats.mean_geo_err_px = st.mean_geo_err_px;
    out_stats.median_geo_err_px = st.median_geo_err_px;
    out_stats.p90_geo_err_px = st.p90_geo_err_px;
    out_stats.mean_photo_err = st.mean_photo_err;
    out_stats.num_samples = (int)st.num_samples;
    out_stats.rmse_geo_err_px = st.rmse_geo_err_px;
    out_stats.rmse_photo_err = st.rmse_photo_err;
    out_stats.completeness = st.completeness;
    out_stats.completeness_geo = st.completeness_geo;
    out_stats.completeness_photo = st.completeness_photo;
    out_stats.completeness_masked_pixels = st.completeness_masked_pixels;
    out_stats.completeness_good_pixels = st.completeness_good_pixels;
    out_stats.completeness_good_pixels_geo = st.completeness_good_pixels_geo;
    out_stats.completeness_good_pixels_photo = st.completeness_good_pixels_photo;
    m_masked.masked_count = st.masked_count;
    m_masked.all_count = st.all_count;
    m_masked.geo_mean = st.masked_geo_mean;
    m_masked.photo_mean = st.masked_photo_mean;
    m_masked.geo_rmse = st.masked_geo_rmse;
    m_masked.photo_rmse = st.masked_photo_rmse;
    m_masked.coverage = st.coverage;
    m_masked.geo_median_approx = st.masked_geo_median_approx;
    m_masked.geo_p90_approx = st.masked_geo_p90_approx;
    m_masked.geo_min = st.masked_geo_min;
    m_masked.geo_max = st.masked_geo_max;
}

}  // namespace LFMVS
