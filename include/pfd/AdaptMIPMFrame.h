/*
 * AdaptMIPMFrame.h -- whole-frame micro-image PatchMatch with cross-view
 * proposals, the class MIStereoMatch::StereoMatchingForMIA_FrameCrossViews
 * drives (MIStereo/MIStereoMatch.cpp:626-696), on the B200 engine.
 *
 * Same public interface and semantics as the reference's MIStereo/AdaptMIPMFrame.h:
 *   AdaptMIPMFrame(LightFieldParams&)                                     :20
 *   bool Initialize(QuadTreeTileInfoMap&, QuadTreeProblemMap&)            :23
 *   void RunPatchMatchCUDAForFrame()                                      :24
 *   void WriteBackResults(QuadTreeDisNormalMap&)                          :25
 *   void ReleaseMemory()                                                  :26
 *   int  GetValidViewCount() const                                        :28
 * Initialize keeps the reference's view selection (every problem that is not
 * garbage and needs matching and has an MLA_Info, in problem-map order), its
 * neighbour lists (the first 16 keys of m_NeighsSortVecForMatch that are
 * views, AdaptMIPMFrame.cpp:145-222) and its parameters
 * (InitGPUParamsFromCPUParams, :126-143).  The frame lives on the device of a
 * pfd context opened on the caller's current CUDA device.
 *
 * Differences, all on failure or outside the reference's interface:
 *  - no call exits the process; Initialize returns false and the other calls
 *    do nothing when a CUDA or engine call fails; LastError() tells why;
 *  - the random streams are Philox keyed by a seed (SetRandomSeed) instead of
 *    cuRAND seeded from clock64(), so runs repeat exactly;
 *  - GetParams() exposes the matching parameters after Initialize, for
 *    callers that run other patch sizes or iteration counts than the
 *    reference's fixed ones.
 */
#ifndef PFD_ADAPTMIPMFRAME_H
#define PFD_ADAPTMIPMFRAME_H

#include <cstdint>
#include <string>
#include <vector>

#include "lf_types.h"

struct pfd_ctx;

namespace LFMVS {

class AdaptMIPMFrame {
public:
    explicit AdaptMIPMFrame(LightFieldParams& params);
    ~AdaptMIPMFrame();
    AdaptMIPMFrame(const AdaptMIPMFrame&) = delete;
    AdaptMIPMFrame& operator=(const AdaptMIPMFrame&) = delete;

    bool Initialize(QuadTreeTileInfoMap& MLA_info_map, QuadTreeProblemMap& problem_map);
    void RunPatchMatchCUDAForFrame();
    void WriteBackResults(QuadTreeDisNormalMap& disNormals_map);
    void ReleaseMemory();

    int GetValidViewCount() const { return m_num_views; }

    /* Not in the reference. */
    void SetRandomSeed(uint64_t seed) { m_seed = seed; }
    PatchMatchParamsLF& GetParams() { return params; }
    const std::string& LastError() const { return m_last_error; }
    /* The engine context and frame id holding the device state (0 before
     * Initialize), for callers that chain further engine calls on it. */
    pfd_ctx* Context() const { return m_ctx; }
    int FrameId() const { return m_frame_id; }
    /* Views in frame order and their neighbour lists (view ids, -1 padded). */
    const QuadTreeTileKeyPtrVec& ViewKeys() const { return m_view_keys; }
    const std::vector<int>& NeighborIds() const { return m_neighbor_ids; }
    const std::vector<int>& NeighborCounts() const { return m_neighbor_counts; }
    int MaxNeighbors() const { return m_max_neighbors; }

protected:
    void InitGPUParamsFromCPUParams();
    bool BuildViewIndexMap(QuadTreeTileInfoMap& MLA_info_map, QuadTreeProblemMap& problem_map);
    bool InitializeGPU();
    bool Fail(const std::string& what);

    LightFieldParamsCUDA m_ParamsCUDA;
    PatchMatchParamsLF   params;
    int                  m_num_views = 0;
    int                  m_max_neighbors = 16;
    int                  m_pixels_per_view = 0;
    bool                 m_bReleased = false;
    uint64_t             m_seed = 0x5eed;

    QuadTreeTileKeyPtrVec m_view_keys;
    std::map<QuadTreeTileKeyPtr, int, QuadTreeTileKeyMapCmpLess> m_key_to_viewid;
    std::vector<uint8_t> m_images;        /* [views][mi_h][mi_w] gray */
    std::vector<uint8_t> m_blur;          /* [views][mi_h][mi_w] blur, empty when no view has one */
    std::vector<float>   m_centers;       /* [views][2] */
    std::vector<int>     m_tilekeys;      /* [views][2] (column, row) */
    std::vector<int>     m_neighbor_ids;  /* [views][m_max_neighbors] */
    std::vector<int>     m_neighbor_counts;

    pfd_ctx* m_ctx = nullptr;
    int      m_frame_id = 0;
    bool     m_has_results = false;
    std::vector<float4>       plane_final_host;
    std::vector<float>        cost_final_host;
    std::vector<float4>       disp_final_host;
    std::vector<unsigned int> selected_final_host;
    std::string m_last_error;
};

}  // namespace LFMVS

#endif
