// shim_probe.cpp -- test driver of the reference-interface classes
// (include/pfd/AdaptMIPMFrame.h, MIDisparityFilter.h, MICycleCheck.h).
//
// Builds the reference's maps (MLA_Info, MLA_Problem, DisparityAndNormal keyed
// by QuadTreeTileKey) from flat arrays, runs the classes exactly as
// MIStereoMatch::StereoMatchingForMIA_FrameCrossViews and FilterAndStatic use
// them, and returns the results as flat arrays, so the Python tests can compare
// them with the engine's C ABI called directly.
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/pfd/AdaptMIPMFrame.h"
#include "../../include/pfd/AdaptMIPMFrameACMM.h"
#include "../../include/pfd/MICycleCheck.h"
#include "../../include/pfd/MIDisparityFilter.h"
#include "../../include/pfd_abi.h"
#include "../../plenoptic-for-depth_b200/host/frame_views.h"

using namespace LFMVS;

namespace {

enum : uint8_t { kGarbage = 1, kNeedMatch = 2, kHasInfo = 4, kHasDN = 8, kHasGray = 16 };

// n problems: keys [n][2] (column, row), centers [n][2], flags [n],
// gray [n][mi][mi]; neighbour lists as (column, row) keys, problem i's in
// nb_keys[nb_off[i] .. nb_off[i+1]), which may name keys outside the map.
// dn_init [n][mi*mi][13]: ph (4), d, c, disp_v (4), selected (as float bits)
// and two unused, the initial DisparityAndNormal contents.
struct Scene {
    LightFieldParams lfp;
    std::vector<QuadTreeTileKeyPtr> keys;
    QuadTreeTileInfoMap info;
    QuadTreeProblemMap problems;
    QuadTreeDisNormalMap dns;
};

float4 f4(float x, float y, float z, float w)
{
    float4 r;
    r.x = x; r.y = y; r.z = z; r.w = w;
    return r;
}

QuadTreeTileKeyPtr make_key(int col, int row) { return std::make_shared<QuadTreeTileKey>(0, col, row); }

void build(Scene& s, int n, int mi, float pitch, const int* keys, const float* centers, const uint8_t* flags,
           const uint8_t* gray, const int* nb_off, const int* nb_keys, const float* dn_init)
{
    s.lfp.mi_width_for_match = mi;
    s.lfp.mi_height_for_match = mi;
    s.lfp.baseline = pitch;
    const size_t ppv = (size_t)mi * mi;
    for (int i = 0; i < n; ++i) {
        // separate key objects for the maps and for the neighbour lists, as the
        // reference's maps compare pointees, never pointers
        s.keys.push_back(make_key(keys[2 * i], keys[2 * i + 1]));
        const QuadTreeTileKeyPtr& k = s.keys.back();
        if (flags[i] & kHasInfo) {
            auto inf = std::make_shared<MLA_Info>();
            inf->SetCenter(Point2f(centers[2 * i], centers[2 * i + 1]));
            inf->SetCol(keys[2 * i]);
            inf->SetRow(keys[2 * i + 1]);
            s.info[k] = inf;
        }
        MLA_Problem& p = s.problems[k];
        p.m_ptrKey = k;
        p.m_bGarbage = (flags[i] & kGarbage) != 0;
        p.m_bNeedMatch = (flags[i] & kNeedMatch) != 0;
        if (flags[i] & kHasGray) {
            p.m_Image_gray = GrayImage(mi, mi);
            std::memcpy(p.m_Image_gray.data.data(), gray + i * ppv, ppv);
        }
        for (int j = nb_off[i]; j < nb_off[i + 1]; ++j)
            p.m_NeighsSortVecForMatch.push_back(make_key(nb_keys[2 * j], nb_keys[2 * j + 1]));
        if (flags[i] & kHasDN) {
            auto dn = std::make_shared<DisparityAndNormal>(s.lfp);
            dn->m_ptrKey = k;
            for (size_t q = 0; q < ppv; ++q) {
                const float* r = dn_init + (i * ppv + q) * 13;
                dn->ph_cuda[q] = f4(r[0], r[1], r[2], r[3]);
                dn->d_cuda[q] = r[4];
                dn->c_cuda[q] = r[5];
                dn->disp_v_cuda[q] = f4(r[6], r[7], r[8], r[9]);
                std::memcpy(&dn->selected_views[q], &r[10], 4);
            }
            s.dns[k] = dn;
        }
    }
}

void dump_dns(const Scene& s, int mi, float* out)
{
    const size_t ppv = (size_t)mi * mi;
    for (size_t i = 0; i < s.keys.size(); ++i) {
        auto it = s.dns.find(s.keys[i]);
        if (it == s.dns.end()) continue;
        const DisparityAndNormal& dn = *it->second;
        for (size_t q = 0; q < ppv; ++q) {
            float* r = out + (i * ppv + q) * 13;
            r[0] = dn.ph_cuda[q].x; r[1] = dn.ph_cuda[q].y; r[2] = dn.ph_cuda[q].z; r[3] = dn.ph_cuda[q].w;
            r[4] = dn.d_cuda[q];
            r[5] = dn.c_cuda[q];
            r[6] = dn.disp_v_cuda[q].x; r[7] = dn.disp_v_cuda[q].y;
            r[8] = dn.disp_v_cuda[q].z; r[9] = dn.disp_v_cuda[q].w;
            std::memcpy(&r[10], &dn.selected_views[q], 4);
            r[11] = (float)dn.m_StereoStage;
            r[12] = 0.0f;
        }
    }
}

// Exposes the view bookkeeping of AdaptMIPMFrame, which needs no device.
struct LayoutProbe : AdaptMIPMFrame {
    using AdaptMIPMFrame::AdaptMIPMFrame;
    bool layout(QuadTreeTileInfoMap& info, QuadTreeProblemMap& problems) { return BuildViewIndexMap(info, problems); }
};

int index_of(const Scene& s, const QuadTreeTileKeyPtr& k)
{
    for (size_t i = 0; i < s.keys.size(); ++i)
        if (*s.keys[i] == *k) return (int)i;
    return -1;
}

}  // namespace

extern "C" {

// AdaptMIPMFrame::BuildViewIndexMap on the scene: view_of[n] receives each
// problem's view id (-1 when not a view), nb [n][16] / nb_count [n] each
// view's neighbour list as problem indices.  Returns the view count, or -1.
int shim_match_layout(int n, int mi, float pitch, const int* keys, const float* centers, const uint8_t* flags,
                      const uint8_t* gray, const int* nb_off, const int* nb_keys, int* view_of, int* nb, int* nb_count)
{
    Scene s;
    std::vector<float> dn0((size_t)n * mi * mi * 13, 0.0f);
    build(s, n, mi, pitch, keys, centers, flags, gray, nb_off, nb_keys, dn0.data());
    LayoutProbe f(s.lfp);
    if (!f.layout(s.info, s.problems)) return -1;
    const QuadTreeTileKeyPtrVec& vk = f.ViewKeys();
    std::vector<int> prob_of(vk.size());
    for (int i = 0; i < n; ++i) view_of[i] = -1;
    for (size_t v = 0; v < vk.size(); ++v) {
        prob_of[v] = index_of(s, vk[v]);
        view_of[prob_of[v]] = (int)v;
    }
    for (size_t v = 0; v < vk.size(); ++v) {
        const int p = prob_of[v];
        nb_count[p] = f.NeighborCounts()[v];
        for (int k = 0; k < 16; ++k) {
            const int id = f.NeighborIds()[v * f.MaxNeighbors() + k];
            nb[p * 16 + k] = id < 0 ? -1 : prob_of[id];
        }
    }
    return f.GetValidViewCount();
}

// The consistency pass's views (frame_views.h): view_of [n], nb [n][32] as
// problem indices (-1: skipped neighbour), nb_count [n].  Returns the view count.
int shim_check_layout(int n, int mi, float pitch, const int* keys, const float* centers, const uint8_t* flags,
                      const uint8_t* gray, const int* nb_off, const int* nb_keys, int* view_of, int* nb, int* nb_count)
{
    Scene s;
    std::vector<float> dn0((size_t)n * mi * mi * 13, 0.0f);
    build(s, n, mi, pitch, keys, centers, flags, gray, nb_off, nb_keys, dn0.data());
    pfd_host::CheckViews v;
    std::string err;
    if (!pfd_host::build_check_views(s.info, s.problems, s.dns, mi, mi, &v, &err)) return -1;
    std::vector<int> prob_of(v.keys.size());
    for (int i = 0; i < n; ++i) view_of[i] = -1;
    for (size_t i = 0; i < v.keys.size(); ++i) {
        prob_of[i] = index_of(s, v.keys[i]);
        view_of[prob_of[i]] = (int)i;
    }
    for (size_t i = 0; i < v.keys.size(); ++i) {
        const int p = prob_of[i];
        nb_count[p] = v.nb_counts[i];
        for (int k = 0; k < 32; ++k) {
            const int id = k < v.max_nb ? v.nb_ids[i * v.max_nb + k] : -1;
            nb[p * 32 + k] = id < 0 ? -1 : prob_of[id];
        }
    }
    return (int)v.keys.size();
}

// MIStereoMatch::StereoMatchingForMIA_FrameCrossViews_ACMM through the class:
// AdaptMIPMFrameACMM Initialize / RunPatchMatchCUDAForFrameACMM /
// WriteBackResults / ReleaseMemory with the reference's own parameters and the
// given seed.  dn_match [n][mi*mi][13] as in shim_run; levels receives
// GetNumLevels().  Returns 0, or -1 with msg (256 bytes) filled.
int shim_run_acmm(int n, int mi, float pitch, const int* keys, const float* centers, const uint8_t* flags,
                  const uint8_t* gray, const int* nb_off, const int* nb_keys, const float* dn_init,
                  unsigned long long seed, float* dn_match, int* levels, char* msg)
{
    Scene s;
    build(s, n, mi, pitch, keys, centers, flags, gray, nb_off, nb_keys, dn_init);
    AdaptMIPMFrameACMM acmm(s.lfp);
    acmm.SetRandomSeed(seed);
    const bool ok = acmm.Initialize(s.info, s.problems);
    *levels = acmm.GetNumLevels();
    if (!ok) {
        std::snprintf(msg, 256, "%s", acmm.LastError().c_str());
        return -1;
    }
    acmm.RunPatchMatchCUDAForFrameACMM();
    if (!acmm.LastError().empty()) {
        std::snprintf(msg, 256, "%s", acmm.LastError().c_str());
        return -1;
    }
    acmm.WriteBackResults(s.dns);
    acmm.ReleaseMemory();
    dump_dns(s, mi, dn_match);
    return 0;
}

// The matching path end to end through the classes:
//   AdaptMIPMFrame Initialize / RunPatchMatchCUDAForFrame / WriteBackResults
//   (params: patch, iterations, top_k, sigma_s, sigma_c overriding the
//   reference's fixed ones; seed), then MICycleCheckerCPU::CheckGlobal on the
//   matched maps, then MIDisparityFilterCPU::FilterGlobal with save_root "x".
// dn_match / dn_filter [n][mi*mi][13] receive the DisparityAndNormal contents
// after matching and after filtering; fstats [13] the filter statistics
// (doubles), cstats [14] and cmasked [11] the cycle statistics.
// Returns 0, or -1 with msg (256 bytes) filled.
int shim_run(int n, int mi, float pitch, const int* keys, const float* centers, const uint8_t* flags,
             const uint8_t* gray, const int* nb_off, const int* nb_keys, const float* dn_init, int patch, int iters,
             int top_k, float sigma_s, float sigma_c, unsigned long long seed, const pfd_filter_cfg* fc,
             const pfd_cycle_cfg* cc, float* dn_match, float* dn_filter, double* fstats, double* cstats,
             double* cmasked, char* msg)
{
    Scene s;
    build(s, n, mi, pitch, keys, centers, flags, gray, nb_off, nb_keys, dn_init);
    auto fail = [&](const std::string& m) {
        std::strncpy(msg, m.c_str(), 255);
        msg[255] = 0;
        return -1;
    };
    {
        AdaptMIPMFrame frame(s.lfp);
        frame.SetRandomSeed(seed);
        if (!frame.Initialize(s.info, s.problems)) return fail("Initialize: " + frame.LastError());
        PatchMatchParamsLF& P = frame.GetParams();
        P.patch_size = patch;
        P.max_iterations = iters;
        P.top_k = top_k;
        P.sigma_spatial = sigma_s;
        P.sigma_color = sigma_c;
        frame.RunPatchMatchCUDAForFrame();
        if (!frame.LastError().empty()) return fail("RunPatchMatchCUDAForFrame: " + frame.LastError());
        frame.WriteBackResults(s.dns);
        frame.ReleaseMemory();
    }
    dump_dns(s, mi, dn_match);

    MICycleCheckerCPU checker(mi, mi, pitch);
    MICycleClampConfig ccfg;
    ccfg.clamp_photo = cc->clamp_photo;
    ccfg.photo_u = cc->photo_u;
    ccfg.clamp_geo = cc->clamp_geo;
    ccfg.geo_u_px = cc->geo_u_px;
    ccfg.pixel_gate_enabled = cc->pixel_gate_enabled;
    ccfg.gate_min_good_neighbors = cc->gate_min_good_neighbors;
    ccfg.gate_geo_px = cc->gate_geo_px;
    ccfg.gate_photo_u = cc->gate_photo_u;
    ccfg.gate_use_clamped = cc->gate_use_clamped;
    MICycleCheckStats cs;
    checker.CheckGlobal("probe", s.info, s.problems, s.dns, cs, cc->max_triplet, false, "x", true, 60, 2.0, 2.0, 3.0,
                        ccfg);
    if (!checker.LastError().empty()) return fail("CheckGlobal: " + checker.LastError());
    const double c[14] = { cs.mean_geo_err_px, cs.median_geo_err_px, cs.p90_geo_err_px, cs.mean_photo_err,
                           (double)cs.num_samples, cs.rmse_geo_err_px, cs.rmse_photo_err, cs.completeness,
                           cs.completeness_geo, cs.completeness_photo, (double)cs.completeness_masked_pixels,
                           (double)cs.completeness_good_pixels, (double)cs.completeness_good_pixels_geo,
                           (double)cs.completeness_good_pixels_photo };
    std::memcpy(cstats, c, sizeof(c));
    const auto& m = checker.LastMaskedFigures();
    const double mm[11] = { (double)m.masked_count, (double)m.all_count, m.geo_mean, m.photo_mean, m.geo_rmse,
                            m.photo_rmse, m.coverage, m.geo_median_approx, m.geo_p90_approx, m.geo_min, m.geo_max };
    std::memcpy(cmasked, mm, sizeof(mm));

    MIDisparityFilterCPU filter(mi, mi, pitch);
    MIDisparityFilterConfig cfg;
    cfg.max_triplet = fc->max_triplet;
    cfg.min_valid_disp = fc->min_valid_disp;
    cfg.use_selected_views_only = fc->use_selected_views_only;
    cfg.clear_selected_views_when_invalid = fc->clear_selected_views_when_invalid;
    cfg.enable_cost_filter = fc->enable_cost_filter;
    cfg.max_cost = fc->max_cost;
    cfg.enable_cycle_geo_filter = fc->enable_cycle_geo_filter;
    cfg.max_geo_err_px = fc->max_geo_err_px;
    cfg.enable_cycle_photo_filter = fc->enable_cycle_photo_filter;
    cfg.max_photo_err_u = fc->max_photo_err_u;
    cfg.min_good_neighbors = fc->min_good_neighbors;
    cfg.enable_spike_filter = fc->enable_spike_filter;
    cfg.spike_abs_diff = fc->spike_abs_diff;
    cfg.spike_min_neighbors = fc->spike_min_neighbors;
    MIDisparityFilterStats fs;
    filter.FilterGlobal("probe", s.info, s.problems, s.dns, cfg, fs, "x");
    if (!filter.LastError().empty()) return fail("FilterGlobal: " + filter.LastError());
    const double f[13] = { (double)fs.total_pixels, (double)fs.initially_valid_pixels, (double)fs.kept_pixels,
                           (double)fs.removed_pixels, (double)fs.removed_by_cost, (double)fs.removed_by_no_support,
                           (double)fs.removed_by_cycle, (double)fs.removed_by_spike,
                           (double)fs.num_disp_error_samples, (double)fs.num_disp_error_le_thresh,
                           fs.mean_disp_error_px, fs.rmse_disp_error_px, fs.p90_disp_error_px };
    std::memcpy(fstats, f, sizeof(f));
    dump_dns(s, mi, dn_filter);
    return 0;
}

}  // extern "C"
