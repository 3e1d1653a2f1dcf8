/*
 * Stand-in for the reference's Common/Common.h when its three PatchMatch
 * kernel files (MIStereo/AdaptMIPMFrame.cu, CudaUtil.cu, AdaptMIPMUtil.cu) are
 * compiled from source as a test oracle.  The real header pulls in OpenCV and
 * Eigen for host-side types that these kernel files never touch; this one
 * declares only what the kernel files and the class declaration in
 * MIStereo/AdaptMIPMFrame.h name.  Test infrastructure: nothing in the engine
 * includes it.
 *
 * MAX_IMAGES is raised from the reference's 4096 (Common/Common.h:28) to the
 * launch grid's z limit, so that a 4080x3068 frame fits cudaTextureObjects
 * down to pitch 15 (about 64 000 micro-images); nothing else reads it in these
 * files.
 */
#ifndef PFD_REF_STUB_COMMON_H
#define PFD_REF_STUB_COMMON_H

#include <cstdint>
#include <string>
#include <vector>
#include <vector_types.h>

#include "pfd/lf_types.h"   /* PatchMatchParamsLF, LightFieldParams(CUDA), the map types */

namespace cv {
/* AdaptMIPMFrame.h declares std::vector<cv::Mat> members; the kernels never use them. */
class Mat {};
}

namespace LFMVS {
#define MAX_IMAGES 65535
}

#endif
