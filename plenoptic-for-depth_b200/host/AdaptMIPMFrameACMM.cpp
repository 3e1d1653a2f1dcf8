// AdaptMIPMFrameACMM.cpp -- the reference's ACMM whole-frame matcher class
// (MIStereo/AdaptMIPMFrameACMM.cpp) over the engine's C ABI.
//
// View bookkeeping, device frame, download and write-back are AdaptMIPMFrame's
// (the reference's two classes have the same code for them); what differs is
// the level count, the level's parameters and the matcher the engine runs.
#include "../../include/pfd/AdaptMIPMFrameACMM.h"

#include <algorithm>

#include "../../include/pfd_abi.h"

namespace LFMVS {

namespace {

// BuildBlurAlignedPyramids (AdaptMIPMFrameACMM.cpp:312-321): levels while the
// window halves from at least 24 pixels to at least 12, at most two.
int pyramid_levels(int w, int h)
{
    int max_levels = 1;
    int cur_w = w, cur_h = h;
    while (max_levels < MAX_ACMM_LEVELS && cur_w >= 24 && cur_h >= 24) {
        cur_w /= 2;
        cur_h /= 2;
        if (cur_w < 12 || cur_h < 12) break;
        ++max_levels;
    }
    return std::max(1, std::min(2, max_levels));
}

}  // namespace

void AdaptMIPMFrameACMM::InitGPUParamsFromCPUParams(int level_id)
{
    AdaptMIPMFrame::InitGPUParamsFromCPUParams();
    // AdaptMIPMFrameACMM.cpp:155-180 at scale 1 (the only level built here)
    if (m_num_levels <= 1) {
        params.max_iterations = 5;
        params.patch_size = 5;
    } else if (level_id == 0) {
        params.max_iterations = 3;
        params.patch_size = 7;
    } else {
        params.max_iterations = 6;
        params.patch_size = 5;
    }
    params.patch_Bound_size = params.patch_size;
    params.top_k = (level_id == 0) ? 6 : 5;
}

bool AdaptMIPMFrameACMM::Initialize(QuadTreeTileInfoMap& MLA_info_map, QuadTreeProblemMap& problem_map)
{
    ReleaseMemory();
    m_bReleased = false;
    m_last_error.clear();
    m_num_levels = pyramid_levels(m_ParamsCUDA.mi_width_for_match, m_ParamsCUDA.mia_height_for_match);
    if (m_num_levels > 1)
        return Fail("windows of 24 pixels and more take the two-level pyramid, which is not built here");
    if (!BuildViewIndexMap(MLA_info_map, problem_map)) return false;
    InitGPUParamsFromCPUParams(0);
    return InitializeGPU();
}

void AdaptMIPMFrameACMM::RunPatchMatchCUDAForFrameACMM()
{
    m_has_results = false;
    if (!m_ctx || !m_frame_id) {
        Fail("RunPatchMatchCUDAForFrameACMM before a successful Initialize");
        return;
    }
    pfd_pm_params p;
    p.max_iterations = params.max_iterations;
    p.patch_size = params.patch_size;
    p.radius_increment = params.radius_increment;
    p.top_k = params.top_k;
    p.sigma_spatial = params.sigma_spatial;
    p.sigma_color = params.sigma_color;
    p.depth_min = params.depth_min;
    p.depth_max = params.depth_max;
    p.base = params.Base;
    pfd_status st = pfd_set_matcher(m_ctx, PFD_MATCHER_ACMM);
    if (st == PFD_OK) st = pfd_patchmatch(m_ctx, m_frame_id, &p, m_seed);
    if (st == PFD_OK)
        st = pfd_download(m_ctx, m_frame_id, &plane_final_host[0].x, cost_final_host.data(), &disp_final_host[0].x,
                          selected_final_host.data());
    if (st != PFD_OK) {
        Fail(pfd_last_error(m_ctx));
        return;
    }
    m_has_results = true;
}

}  // namespace LFMVS
