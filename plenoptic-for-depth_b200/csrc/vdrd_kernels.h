// vdrd_kernels.h -- virtual-to-real depth conversion and the behavioural-model
// fit, FP64 on the device (vdrd_kernels.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace pfd {

constexpr int kMaxVdSegments = 64;

// mode 0: VirtualToRealDepthFunc::convertVirtualToRealDepth (double out);
// mode 1: LFRefocus::ConvertVdToRd (float out).
cudaError_t launch_vd_to_rd(const float* vd, size_t n, double c0, double c1, double c2, int mode, void* out,
                            cudaStream_t st);
// LFRefocus::ConvertVdToRdSegment; segs: [nseg][5] (min, max, c0, c1, c2) on the device.
cudaError_t launch_vd_to_rd_segments(const float* vd, size_t n, const double* segs, int nseg, float* out,
                                     cudaStream_t st);
// Normal-equation sums of [a_L v, v, 1] c = a_L: 9 doubles per block into partial
// (A00 A01 A02 A11 A12 A22 b0 b1 b2), then folded in block order into sums[9].
int fit_blocks(size_t n);
cudaError_t launch_fit_sums(const float* real_depth, const float* vd, size_t n, double* partial, double* sums,
                            cudaStream_t st);

}  // namespace pfd
