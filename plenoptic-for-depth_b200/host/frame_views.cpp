// frame_views.cpp -- see frame_views.h.
#include "frame_views.h"

#include <algorithm>
#include <cstring>

namespace pfd_host {

using namespace LFMVS;

bool frame_extent(const std::vector<float>& centers, int mi_w, int mi_h, int* W, int* H, std::string* err)
{
    int w = mi_w, h = mi_h;
    for (size_t v = 0; v < centers.size() / 2; ++v) {
        // the same float expression pfd_frame_create evaluates
        const float ox = (float)((double)centers[2 * v] - (mi_w - 1) * 0.5);
        const float oy = (float)((double)centers[2 * v + 1] - (mi_h - 1) * 0.5);
        if (!(ox >= 0.0f) || !(oy >= 0.0f)) {
            *err = "view " + std::to_string(v) + ": matching window starts outside the raw frame";
            return false;
        }
        w = std::max(w, (int)ox + mi_w);
        h = std::max(h, (int)oy + mi_h);
    }
    *W = w;
    *H = h;
    return true;
}

bool build_check_views(const QuadTreeTileInfoMap& info, const QuadTreeProblemMap& problems,
                       const QuadTreeDisNormalMap& dns, int mi_w, int mi_h, CheckViews* out, std::string* err)
{
    CheckViews& v = *out;
    v = CheckViews{};
    std::map<QuadTreeTileKeyPtr, int, QuadTreeTileKeyMapCmpLess> id_of;
    for (auto it = problems.begin(); it != problems.end(); ++it) {
        auto d = dns.find(it->first);
        if (d == dns.end() || !d->second) continue;
        const MLA_Problem& pr = it->second;
        if (pr.m_Image_gray.empty()) continue;
        auto m = info.find(it->first);
        if (m == info.end() || !m->second) continue;
        if (pr.m_Image_gray.rows != mi_h || pr.m_Image_gray.cols != mi_w) {
            *err = "micro-image " + std::to_string(it->first->GetTileX()) + "," + std::to_string(it->first->GetTileY()) +
                   " is not " + std::to_string(mi_w) + "x" + std::to_string(mi_h);
            return false;
        }
        id_of[it->first] = (int)v.keys.size();
        v.keys.push_back(it->first);
        v.dns.push_back(d->second);
        v.centers.push_back(m->second->GetCenter().x);
        v.centers.push_back(m->second->GetCenter().y);
        v.tilekeys.push_back(it->first->GetTileX());
        v.tilekeys.push_back(it->first->GetTileY());
        for (int y = 0; y < mi_h; ++y)
            v.gray.insert(v.gray.end(), pr.m_Image_gray.ptr(y), pr.m_Image_gray.ptr(y) + mi_w);
    }
    const int V = (int)v.keys.size();
    std::vector<std::vector<int>> lists(V);
    for (int i = 0; i < V; ++i) {
        const MLA_Problem& pr = problems.find(v.keys[i])->second;
        QuadTreeTileKeyPtrVec nk = pr.m_NeighsSortVecForMatch;
        if (nk.empty())
            for (const Res_image_Key& r : pr.m_Res_Image_KeyVec) nk.push_back(r.m_ptrKey);
        for (size_t k = 0; k < nk.size() && k < (size_t)PFD_MAX_NEIGHBORS; ++k) {
            auto f = nk[k] ? id_of.find(nk[k]) : id_of.end();
            // a view listed as its own neighbour has a zero baseline, which every
            // check skips (MIDisparityFilter.cpp:519-521)
            lists[i].push_back(f == id_of.end() || f->second == i ? -1 : f->second);
        }
        v.max_nb = std::max(v.max_nb, (int)lists[i].size());
    }
    v.nb_ids.assign((size_t)V * v.max_nb, -1);
    v.nb_counts.assign(V, 0);
    for (int i = 0; i < V; ++i) {
        std::copy(lists[i].begin(), lists[i].end(), v.nb_ids.begin() + (size_t)i * v.max_nb);
        v.nb_counts[i] = (int)lists[i].size();
    }
    return true;
}

pfd_status create_check_frame(pfd_ctx* ctx, const CheckViews& v, int mi_w, int mi_h, int* frame_id,
                              std::string* err)
{
    int W = 0, H = 0;
    if (!frame_extent(v.centers, mi_w, mi_h, &W, &H, err)) return PFD_EINVAL;
    pfd_status st = pfd_frame_create(ctx, frame_id, W, H, v.centers.data(), v.tilekeys.data(), (int)v.keys.size(),
                                     mi_w, mi_h, v.nb_ids.data(), v.nb_counts.data(), v.max_nb, nullptr);
    if (st == PFD_OK) st = pfd_frame_set_micro_images(ctx, *frame_id, v.gray.data());
    if (st != PFD_OK) *err = pfd_last_error(ctx);
    return st;
}

}  // namespace pfd_host
