/*
 * AdaptMIPMFrameACMM.h -- the ACMM whole-frame micro-image matcher, the class
 * MIStereoMatch::StereoMatchingForMIA_FrameCrossViews_ACMM drives
 * (MIStereo/MIStereoMatch.cpp:698-740), on the B200 engine.
 *
 * Same public interface and semantics as the reference's
 * MIStereo/AdaptMIPMFrameACMM.h:
 *   AdaptMIPMFrameACMM(LightFieldParams&)                                 :30
 *   bool Initialize(QuadTreeTileInfoMap&, QuadTreeProblemMap&)            :34
 *   void RunPatchMatchCUDAForFrameACMM()                                  :36
 *   void WriteBackResults(QuadTreeDisNormalMap&)                          :37
 *   void ReleaseMemory()                                                  :38
 *   int  GetValidViewCount() const, int GetNumLevels() const              :40-41
 * The view selection and neighbour lists are AdaptMIPMFrame's (the two
 * classes share BuildViewIndexMap, AdaptMIPMFrameACMM.cpp:207-280; Initialize
 * is :479-493).  The pyramid has as many levels as BuildBlurAlignedPyramids
 * gives (AdaptMIPMFrameACMM.cpp:312-321): one below a 24-pixel window, and then the
 * level's parameters are InitGPUParamsFromCPUParams's (:155-180): patch 5,
 * 5 iterations, top_k 6.  The matching is the engine's PFD_MATCHER_ACMM.
 *
 * Differences, beside those of AdaptMIPMFrame (no exits, Philox streams keyed
 * by SetRandomSeed, GetParams, LastError):
 *  - windows of 24 pixels and more (a two-level pyramid with a warm start in
 *    the reference) are refused: Initialize returns false;
 *  - BuildSingleLevelBlurAlignment does nothing in the reference either
 *    (:295-303), so no blur alignment exists to port.
 */
#ifndef PFD_ADAPTMIPMFRAMEACMM_H
#define PFD_ADAPTMIPMFRAMEACMM_H

#include "AdaptMIPMFrame.h"

namespace LFMVS {

const int MAX_ACMM_LEVELS = 4;

class AdaptMIPMFrameACMM : public AdaptMIPMFrame {
public:
    explicit AdaptMIPMFrameACMM(LightFieldParams& params) : AdaptMIPMFrame(params) {}

    bool Initialize(QuadTreeTileInfoMap& MLA_info_map, QuadTreeProblemMap& problem_map);
    void RunPatchMatchCUDAForFrameACMM();
    int GetNumLevels() const { return m_num_levels; }

protected:
    void InitGPUParamsFromCPUParams(int level_id);
    int m_num_levels = 0;
};

}  // namespace LFMVS

#endif
