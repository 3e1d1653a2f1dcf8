// MIDisparityFilter.cpp -- MIDisparityFilterCPU::FilterGlobal
// (CheckModule/MIDisparityFilter.cpp:962-1009) over the engine's C ABI.
//
// The micro-images, lens centres and results of the maps become one engine
// frame (frame_views.h), pfd_filter runs the per-view filter on the device
// with the reference's in-place view order, and the pixels it rejects get the
// values of InvalidatePixel (:158-174) in the caller's DisparityAndNormal
// arrays.  Every other pixel is left untouched, as in the reference.
#include "../../include/pfd/MIDisparityFilter.h"

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "../../include/pfd_abi.h"
#include "frame_views.h"

namespace LFMVS {

MIDisparityFilterCPU::MIDisparityFilterCPU(int mi_w, int mi_h, float baseline_unit)
    : W_(mi_w), H_(mi_h), baseline_unit_(baseline_unit)
{
}

// MIDisparityFilter.cpp:36-51
float MIDisparityFilterCPU::QuantileFromSorted(const std::vector<float>& sorted_vals, float q)
{
    if (sorted_vals.empty()) return 0.0f;
    if (sorted_vals.size() == 1) return sorted_vals[0];
    const float qq = std::max(0.0f, std::min(1.0f, q));
    const float pos = qq * static_cast<float>(sorted_vals.size() - 1);
    const int lo = static_cast<int>(std::floor(pos));
    const int hi = static_cast<int>(std::ceil(pos));
    const float t = pos - static_cast<float>(lo);
    if (lo == hi) return sorted_vals[lo];
    return sorted_vals[lo] * (1.0f - t) + sorted_vals[hi] * t;
}

void MIDisparityFilterCPU::FilterGlobal(const std::string& frameName, const QuadTreeTileInfoMap& MLA_info_map,
                                        const QuadTreeProblemMap& problems_map, QuadTreeDisNormalMap& dis_normals,
                                        const MIDisparityFilterConfig& cfg, MIDisparityFilterStats& out_stats,
                                        const std::string& save_root) const
{
    out_stats = MIDisparityFilterStats{};
    m_last_error.clear();
    auto fail = [&](const std::string& why) {
        m_last_error = why;
        std::fprintf(stderr, "[MIDisparityFilter] frame=%s: %s\n", frameName.c_str(), why.c_str());
    };

    pfd_host::CheckViews views;
    std::string err;
    if (!pfd_host::build_check_views(MLA_info_map, problems_map, dis_normals, W_, H_, &views, &err)) return fail(err);
    const int V = (int)views.keys.size();
    if (V == 0) return;
    const size_t ppv = (size_t)W_ * H_, n = (size_t)V * ppv;

    // State as the filter reads it: the disparity is ph.w, or d when ph.w is
    // not finite (read_disp and BilinearDisparity, :441-447, :96-105).
    std::vector<float4> plane(n), disp(n);
    std::vector<float> cost(n);
    std::vector<uint32_t> sel(n);
    for (int v = 0; v < V; ++v) {
        const DisparityAndNormal& dn = *views.dns[v];
        for (size_t i = 0; i < ppv; ++i) {
            float4 p = dn.ph_cuda[i];
            if (!std::isfinite(p.w)) p.w = dn.d_cuda[i];
            plane[v * ppv + i] = p;
            cost[v * ppv + i] = dn.c_cuda[i];
            disp[v * ppv + i] = dn.disp_v_cuda[i];
            sel[v * ppv + i] = dn.selected_views[i];
        }
    }

    pfd_filter_cfg c;
    c.max_triplet = cfg.max_triplet;
    c.min_valid_disp = cfg.min_valid_disp;
    c.use_selected_views_only = cfg.use_selected_views_only;
    c.clear_selected_views_when_invalid = cfg.clear_selected_views_when_invalid;
    c.enable_cost_filter = cfg.enable_cost_filter;
    c.max_cost = cfg.max_cost;
    c.enable_cycle_geo_filter = cfg.enable_cycle_geo_filter;
    c.max_geo_err_px = cfg.max_geo_err_px;
    c.enable_cycle_photo_filter = cfg.enable_cycle_photo_filter;
    c.max_photo_err_u = cfg.max_photo_err_u;
    c.min_good_neighbors = cfg.min_good_neighbors;
    c.enable_spike_filter = cfg.enable_spike_filter;
    c.spike_abs_diff = cfg.spike_abs_diff;
    c.spike_min_neighbors = cfg.spike_min_neighbors;

    pfd_host::ScopedContext ctx;
    if (ctx.open() != PFD_OK) return fail("cannot open an engine context on the current device");
    int fid = 0;
    if (pfd_host::create_check_frame(ctx.ctx, views, W_, H_, &fid, &err) != PFD_OK) return fail(err);
    std::vector<uint8_t> reason(n);
    long long st[8] = { 0 };
    pfd_status s = pfd_state_upload(ctx.ctx, fid, &plane[0].x, cost.data(), &disp[0].x, sel.data());
    if (s == PFD_OK) s = pfd_filter(ctx.ctx, fid, &c, baseline_unit_, reason.data(), st);
    const bool want_err = cfg.dump_disp_error_map && !save_root.empty();
    std::vector<float> err_map;
    if (s == PFD_OK && want_err) {
        err_map.resize(n);
        s = pfd_reprojection_error(ctx.ctx, fid, &c, baseline_unit_, err_map.data());
    }
    if (s != PFD_OK) return fail(pfd_last_error(ctx.ctx));

    // InvalidatePixel on the rejected pixels
    for (int v = 0; v < V; ++v) {
        DisparityAndNormal& dn = *views.dns[v];
        for (size_t i = 0; i < ppv; ++i) {
            if (reason[v * ppv + i] == PFD_PR_KEEP) continue;
            dn.d_cuda[i] = -1.0f;
            dn.ph_cuda[i].x = 0.0f;
            dn.ph_cuda[i].y = 0.0f;
            dn.ph_cuda[i].z = 0.0f;
            dn.ph_cuda[i].w = -1.0f;
            dn.c_cuda[i] = 2.0f;
            dn.disp_v_cuda[i].x = -1.0f;
            dn.disp_v_cuda[i].y = -1.0f;
            dn.disp_v_cuda[i].z = 0.0f;
            dn.disp_v_cuda[i].w = 0.0f;
            if (cfg.clear_selected_views_when_invalid) dn.selected_views[i] = 0u;
        }
    }
    out_stats.total_pixels = st[0];
    out_stats.initially_valid_pixels = st[1];
    out_stats.kept_pixels = st[2];
    out_stats.removed_pixels = st[3];
    out_stats.removed_by_cost = st[4];
    out_stats.removed_by_no_support = st[5];
    out_stats.removed_by_cycle = st[6];
    out_stats.removed_by_spike = st[7];

    // DumpWholeFrameReprojectionError (:844-950): the figures over the kept
    // errors <= disp_error_vis_max_px, views in map order, rows then columns.
    if (want_err) {
        std::vector<float> vals;
        for (size_t i = 0; i < n; ++i) {
            const float e = err_map[i];
            if (!std::isfinite(e) || e < 0.0f || e > cfg.disp_error_vis_max_px) continue;
            vals.push_back(e);
        }
        if (!vals.empty()) {
            int num_le = 0;
            double sum = 0.0, sqsum = 0.0;
            for (float e : vals) {
                sum += e;
                sqsum += static_cast<double>(e) * e;
                if (e <= cfg.disp_error_thresh_px) ++num_le;
            }
            std::sort(vals.begin(), vals.end());
            out_stats.num_disp_error_samples = (int64_t)vals.size();
            out_stats.num_disp_error_le_thresh = num_le;
            out_stats.mean_disp_error_px = sum / static_cast<double>(vals.size());
            out_stats.rmse_disp_error_px = std::sqrt(sqsum / static_cast<double>(vals.size()));
            out_stats.p90_disp_error_px = QuantileFromSorted(vals, 0.9f);
        }
    }
}

}  // namespace LFMVS
