/*
 * Stand-in for the reference's MVStereo/LFDepthInfo.h (see Common/Common.h of
 * this directory): PatchMatchParamsLF and the map types come from the
 * engine's own restatement of them in include/pfd/lf_types.h, which keeps the
 * reference's member names, types and order (LFDepthInfo.h:19-46).
 */
#ifndef PFD_REF_STUB_LFDEPTHINFO_H
#define PFD_REF_STUB_LFDEPTHINFO_H

#include "Common/CommonCUDA.h"

#endif
