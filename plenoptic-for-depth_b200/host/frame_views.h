// frame_views.h -- the engine frame a set of reference maps describes: which
// micro-images become views, in which order, with which neighbour lists.
// Shared by the classes of include/pfd/.
#ifndef PFD_HOST_FRAME_VIEWS_H
#define PFD_HOST_FRAME_VIEWS_H

#include <string>
#include <vector>

#include "../../include/pfd_abi.h"
#include "../../include/pfd/lf_types.h"

namespace pfd_host {

// A pfd context on the calling thread's current device, destroyed with the object.
struct ScopedContext {
    pfd_ctx* ctx = nullptr;
    pfd_status open() { return pfd_create(&ctx, -1, 0); }
    ~ScopedContext() { pfd_destroy(ctx); }
};

// Raw-frame extent that holds every view's matching window, whose origin is
// trunc(center - (mi - 1) / 2) (DepthSolver.cpp:1894-1895); false when an
// origin is negative.
bool frame_extent(const std::vector<float>& centers, int mi_w, int mi_h, int* W, int* H, std::string* err);

// Views of the consistency pass (MIDisparityFilter.cpp:962-986,
// MICycleCheck.cpp:757-776): every problem-map entry with a DisparityAndNormal,
// a non-empty gray image and an MLA_Info, in map order.  Neighbour k of a view
// is entry k of m_NeighsSortVecForMatch (else of m_Res_Image_KeyVec), mapped
// to its view id, or -1 when that key is not a view itself (the reference
// skips such a neighbour for every check); lists are cut at 32 entries, the
// width of the selected-view masks.  No qualifying problem gives no views and
// true, as the reference then checks nothing.
struct CheckViews {
    std::vector<LFMVS::QuadTreeTileKeyPtr> keys;
    std::vector<LFMVS::DisparityAndNormalPtr> dns;
    std::vector<float> centers;        // [V][2]
    std::vector<int> tilekeys;         // [V][2] (column, row)
    std::vector<int> nb_ids;           // [V][max_nb]
    std::vector<int> nb_counts;        // [V]
    int max_nb = 1;
    std::vector<uint8_t> gray;         // [V][mi_h][mi_w]
};
bool build_check_views(const LFMVS::QuadTreeTileInfoMap& info, const LFMVS::QuadTreeProblemMap& problems,
                       const LFMVS::QuadTreeDisNormalMap& dns, int mi_w, int mi_h, CheckViews* out,
                       std::string* err);

// Creates the engine frame of `v` on ctx with its micro-images filled.
pfd_status create_check_frame(pfd_ctx* ctx, const CheckViews& v, int mi_w, int mi_h, int* frame_id,
                              std::string* err);

}  // namespace pfd_host

#endif
