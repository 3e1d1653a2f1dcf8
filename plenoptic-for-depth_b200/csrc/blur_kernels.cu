// blur_kernels.cu -- the blur channel of the frame path, computed on the device.
//
// The reference quantises blur with ImageQualityEstimate::QuantizeBlurByLaplacian
// (Util/ImageQualityEstimate.cpp:211-230): cv::Laplacian of the raw frame's
// BGR2GRAY image, ksize 1 (the aperture 0 1 0 / 1 -4 1 / 0 1 0), CV_32F output,
// default border (reflect without repeating the edge: -1 -> 1, W -> W - 2).
// DepthSolver::SliceAndIndicatlizeForMI (DepthSolver.cpp:2709-2754) then cuts
// every micro-image's window (the matching window, at GetLeftDownCorner) out of
// it into MLA_Problem::m_Image_Blureness, a cv::Mat_<uint8>: Mat::copyTo into a
// fixed-type 8-bit matrix converts with saturate_cast, so the channel holds the
// Laplacian clamped to [0, 255] (an integer already: no rounding happens).  The
// same window of cv::threshold(score, 10, 255, THRESH_BINARY) becomes
// m_Image_Blureness_Bianry, and MLA_Problem::ComputeBlurenessValue
// (MVStereo/LFDepthInfo.cpp:65-83) counts its 255s: the pixels whose Laplacian
// exceeds 10.
//
// One CTA per view; each thread computes pixels of the window from five raw
// bytes (the raw frame is read through the read-only cache: neighbouring
// windows and rows share lines).  The count is a CTA-wide __syncthreads_count
// per pass, so it is exact and independent of scheduling.
#include <cstdint>
#include "blur_kernels.h"

namespace pfd {

namespace {

__device__ __forceinline__ int reflect101(int p, int n) { return p < 0 ? -p : (p >= n ? 2 * n - 2 - p : p); }

}  // namespace

__global__ void __launch_bounds__(128) pm_blur_kernel(const uint8_t* __restrict__ raw, int raw_pitch, int W, int H,
                                                      const int2* __restrict__ origin, int mi_w, int mi_h,
                                                      int tile_stride, uint8_t* __restrict__ tiles,
                                                      uint32_t* __restrict__ counts)
{
    const int v = blockIdx.x;
    const int2 o = origin[v];
    const int ppv = mi_w * mi_h;
    uint8_t* tile = tiles + (size_t)v * tile_stride;
    uint32_t sharp = 0;
    for (int base = 0; base < tile_stride; base += blockDim.x) {
        const int e = base + threadIdx.x;
        int lap = 0;
        if (e < ppv) {
            const int x = o.x + e % mi_w, y = o.y + e / mi_w;
            const uint8_t* row = raw + (size_t)y * raw_pitch;
            const int c = __ldg(row + x);
            const int l = __ldg(row + reflect101(x - 1, W)), r = __ldg(row + reflect101(x + 1, W));
            const int u = __ldg(raw + (size_t)reflect101(y - 1, H) * raw_pitch + x);
            const int d = __ldg(raw + (size_t)reflect101(y + 1, H) * raw_pitch + x);
            lap = l + r + u + d - 4 * c;
        }
        if (e < tile_stride) tile[e] = (uint8_t)(lap < 0 ? 0 : (lap > 255 ? 255 : lap));
        if (counts) sharp += (uint32_t)__syncthreads_count(lap > 10);
    }
    if (counts && threadIdx.x == 0) counts[v] = sharp;
}

cudaError_t launch_blur(const uint8_t* raw, int raw_pitch, int W, int H, const int2* origin, int V, int mi_w,
                        int mi_h, int tile_stride, uint8_t* tiles, uint32_t* counts, cudaStream_t st)
{
    if (V <= 0) return cudaSuccess;
    pm_blur_kernel<<<V, 128, 0, st>>>(raw, raw_pitch, W, H, origin, mi_w, mi_h, tile_stride, tiles, counts);
    return cudaGetLastError();
}

}  // namespace pfd
