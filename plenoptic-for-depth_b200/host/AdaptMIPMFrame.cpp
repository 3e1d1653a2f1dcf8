// AdaptMIPMFrame.cpp -- the reference's whole-frame matcher class
// (MIStereo/AdaptMIPMFrame.cpp) over the engine's C ABI.
//
// The view bookkeeping keeps the reference's rules step for step, because the
// selected-view bit k of a result names neighbour k of this list:
//   * views: problem-map order, skipping garbage problems, problems that need
//     no matching and keys without an MLA_Info (AdaptMIPMFrame.cpp:152-166);
//   * neighbours: the first m_max_neighbors (16) keys of m_NeighsSortVecForMatch
//     that are views, in list order (:207-218);
//   * parameters: InitGPUParamsFromCPUParams (:126-143).
// The texture objects, ping-pong buffers and cuRAND states of InitializeGPU
// (:278-327) are the engine frame; the reference's limit of MAX_IMAGES views
// (4096, the size of its texture-object table, Common/Common.h:32) does not
// apply, since views are not texture objects here.
#include "../../include/pfd/AdaptMIPMFrame.h"

#include <cstdio>
#include <cstring>

#include "../../include/pfd_abi.h"
#include "frame_views.h"

namespace LFMVS {

AdaptMIPMFrame::AdaptMIPMFrame(LightFieldParams& paramsIn) : m_ParamsCUDA(paramsIn) {}

AdaptMIPMFrame::~AdaptMIPMFrame() { ReleaseMemory(); }

bool AdaptMIPMFrame::Fail(const std::string& what)
{
    m_last_error = what;
    std::fprintf(stderr, "[AdaptMIPMFrame] %s\n", what.c_str());
    return false;
}

void AdaptMIPMFrame::ReleaseMemory()
{
    if (m_bReleased) return;
    m_bReleased = true;
    m_view_keys.clear();
    m_key_to_viewid.clear();
    m_images.clear();
    m_blur.clear();
    m_centers.clear();
    m_tilekeys.clear();
    m_neighbor_ids.clear();
    m_neighbor_counts.clear();
    plane_final_host.clear();
    cost_final_host.clear();
    disp_final_host.clear();
    selected_final_host.clear();
    m_has_results = false;
    if (m_ctx) {
        if (m_frame_id) pfd_frame_free(m_ctx, m_frame_id);
        pfd_destroy(m_ctx);
    }
    m_ctx = nullptr;
    m_frame_id = 0;
}

void AdaptMIPMFrame::InitGPUParamsFromCPUParams()
{
    params.max_iterations = 3;
    params.patch_size = 5;
    params.patch_Bound_size = 5;
    params.propagation_Graph_size = 5;
    params.num_images = m_max_neighbors + 1;
    params.top_k = 5;
    params.depth_min = 0.0f;
    params.depth_max = m_ParamsCUDA.baseline * 0.5f;
    params.disparity_min = 0.0f;
    params.disparity_max = m_ParamsCUDA.baseline * 0.5f;
    params.Base = m_ParamsCUDA.baseline;
    params.MLA_Mask_Width_Cuda = m_ParamsCUDA.mi_width_for_match;
    params.MLA_Mask_Height_Cuda = m_ParamsCUDA.mia_height_for_match;
    params.base_height_ratio = 0.2f;
    params.base_height_sigma = 0.05f;
}

bool AdaptMIPMFrame::BuildViewIndexMap(QuadTreeTileInfoMap& MLA_info_map, QuadTreeProblemMap& problem_map)
{
    const int mi_w = m_ParamsCUDA.mi_width_for_match, mi_h = m_ParamsCUDA.mia_height_for_match;
    const size_t ppv = (size_t)mi_w * mi_h;
    m_view_keys.clear();
    m_key_to_viewid.clear();
    m_images.clear();
    m_blur.clear();
    m_centers.clear();
    m_tilekeys.clear();
    bool any_blur = false;
    std::vector<const decltype(MLA_Problem::m_Image_Blureness)*> blur_of;
    for (auto itrP = problem_map.begin(); itrP != problem_map.end(); ++itrP) {
        MLA_Problem& problem = itrP->second;
        if (problem.m_bGarbage || !problem.m_bNeedMatch) continue;
        auto itrInfo = MLA_info_map.find(itrP->first);
        if (itrInfo == MLA_info_map.end() || !itrInfo->second) continue;
        const auto& g = problem.m_Image_gray;
        if (g.rows != mi_h || g.cols != mi_w)
            return Fail("micro-image (" + std::to_string(itrP->first->GetTileX()) + ", " +
                        std::to_string(itrP->first->GetTileY()) + ") is not " + std::to_string(mi_w) + "x" +
                        std::to_string(mi_h));
        const auto& b = problem.m_Image_Blureness;
        if (!b.empty() && (b.rows != mi_h || b.cols != mi_w))
            return Fail("blur image of (" + std::to_string(itrP->first->GetTileX()) + ", " +
                        std::to_string(itrP->first->GetTileY()) + ") has the wrong size");
        any_blur = any_blur || !b.empty();
        const int vid = (int)m_view_keys.size();
        m_view_keys.push_back(itrP->first);
        m_key_to_viewid[itrP->first] = vid;
        for (int y = 0; y < mi_h; ++y) m_images.insert(m_images.end(), g.ptr(y), g.ptr(y) + mi_w);
        blur_of.push_back(&b);
        m_centers.push_back(itrInfo->second->GetCenter().x);
        m_centers.push_back(itrInfo->second->GetCenter().y);
        m_tilekeys.push_back(itrP->first->GetTileX());
        m_tilekeys.push_back(itrP->first->GetTileY());
    }
    m_num_views = (int)m_view_keys.size();
    if (m_num_views <= 0) return Fail("no valid micro-images for current frame");
    // The reference reads the blur channel through a texture for every view
    // and creates none for an empty image; here a view without a blur image
    // reads zeros, and a frame where no view has one gets no blur penalty.
    if (any_blur) {
        m_blur.assign((size_t)m_num_views * ppv, 0);
        for (int v = 0; v < m_num_views; ++v)
            if (!blur_of[v]->empty())
                for (int y = 0; y < mi_h; ++y)
                    std::memcpy(&m_blur[(size_t)v * ppv + (size_t)y * mi_w], blur_of[v]->ptr(y), mi_w);
    }
    m_neighbor_ids.assign((size_t)m_num_views * m_max_neighbors, -1);
    m_neighbor_counts.assign(m_num_views, 0);
    for (int vid = 0; vid < m_num_views; ++vid) {
        const MLA_Problem& problem = problem_map[m_view_keys[vid]];
        int count = 0;
        for (size_t i = 0; i < problem.m_NeighsSortVecForMatch.size() && count < m_max_neighbors; ++i) {
            const QuadTreeTileKeyPtr& nk = problem.m_NeighsSortVecForMatch[i];
            if (!nk) continue;
            auto itr = m_key_to_viewid.find(nk);
            if (itr == m_key_to_viewid.end()) continue;
            m_neighbor_ids[(size_t)vid * m_max_neighbors + count] = itr->second;
            ++count;
        }
        m_neighbor_counts[vid] = count;
    }
    return true;
}

bool AdaptMIPMFrame::InitializeGPU()
{
    const int mi_w = m_ParamsCUDA.mi_width_for_match, mi_h = m_ParamsCUDA.mia_height_for_match;
    m_pixels_per_view = mi_w * mi_h;
    std::string err;
    int W = 0, H = 0;
    if (!pfd_host::frame_extent(m_centers, mi_w, mi_h, &W, &H, &err)) return Fail(err);
    if (pfd_create(&m_ctx, -1, 0) != PFD_OK) return Fail("cannot open an engine context on the current device");
    pfd_status st = pfd_frame_create(m_ctx, &m_frame_id, W, H, m_centers.data(), m_tilekeys.data(), m_num_views, mi_w,
                                     mi_h, m_neighbor_ids.data(), m_neighbor_counts.data(), m_max_neighbors,
                                     m_blur.empty() ? nullptr : m_blur.data());
    if (st == PFD_OK) st = pfd_frame_set_micro_images(m_ctx, m_frame_id, m_images.data());
    if (st != PFD_OK) return Fail(pfd_last_error(m_ctx));
    const size_t frame_pixels = (size_t)m_pixels_per_view * m_num_views;
    plane_final_host.resize(frame_pixels);
    cost_final_host.resize(frame_pixels);
    disp_final_host.resize(frame_pixels);
    selected_final_host.resize(frame_pixels);
    return true;
}

bool AdaptMIPMFrame::Initialize(QuadTreeTileInfoMap& MLA_info_map, QuadTreeProblemMap& problem_map)
{
    ReleaseMemory();
    m_bReleased = false;
    m_last_error.clear();
    if (!BuildViewIndexMap(MLA_info_map, problem_map)) return false;
    InitGPUParamsFromCPUParams();
    return InitializeGPU();
}

void AdaptMIPMFrame::RunPatchMatchCUDAForFrame()
{
    m_has_results = false;
    if (!m_ctx || !m_frame_id) {
        Fail("RunPatchMatchCUDAForFrame before a successful Initialize");
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
    pfd_status st = pfd_set_matcher(m_ctx, PFD_MATCHER_FRAME);
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

void AdaptMIPMFrame::WriteBackResults(QuadTreeDisNormalMap& disNormals_map)
{
    if (!m_has_results) return;
    const int pixels = m_pixels_per_view;
    for (int vid = 0; vid < m_num_views; ++vid) {
        auto itr = disNormals_map.find(m_view_keys[vid]);
        if (itr == disNormals_map.end() || !itr->second) continue;
        DisparityAndNormal& dn = *itr->second;
        const size_t offset = (size_t)vid * pixels;
        for (int idx = 0; idx < pixels; ++idx) {
            dn.ph_cuda[idx] = plane_final_host[offset + idx];
            dn.d_cuda[idx] = plane_final_host[offset + idx].w;
            dn.c_cuda[idx] = cost_final_host[offset + idx];
            dn.disp_v_cuda[idx] = disp_final_host[offset + idx];
            dn.selected_views[idx] = selected_final_host[offset + idx];
        }
        dn.m_StereoStage = eSS_ACMH_Finished;
    }
}

}  // namespace LFMVS
