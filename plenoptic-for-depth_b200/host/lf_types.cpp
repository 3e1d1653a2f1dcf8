// lf_types.cpp -- DisparityAndNormal's array ownership (MVStereo/LFDepthInfo.cpp:550-616).
#include "../../include/pfd/lf_types.h"

namespace LFMVS {

DisparityAndNormal::DisparityAndNormal(LightFieldParams& params) : m_Params(params)
{
    const size_t n = (size_t)m_Params.mi_width_for_match * m_Params.mi_height_for_match;
    c_cuda = new float[n];
    d_cuda = new float[n];
    ph_cuda = new float4[n];
    disp_v_cuda = new float4[n];
    selected_views = new unsigned int[n];
}

DisparityAndNormal::~DisparityAndNormal() { Release(); }

void DisparityAndNormal::Release()
{
    m_StereoStage = eSS_ACMH_Begin;
    delete[] ph_cuda;
    delete[] disp_v_cuda;
    delete[] c_cuda;
    delete[] d_cuda;
    delete[] selected_views;
    ph_cuda = disp_v_cuda = nullptr;
    c_cuda = d_cuda = nullptr;
    selected_views = nullptr;
}

}  // namespace LFMVS
