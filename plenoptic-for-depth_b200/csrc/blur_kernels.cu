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

// Richness channel.  ImageQualityEstimate::QuantizeRichnessByGLCM
// (Util/ImageQualityEstimate.cpp:310-340) gives every pixel with 4 <= row < H - 4
// and 4 <= col < W - 4 the GLCM contrast of the 8x8 window at (col - 4, row - 4)
// (calculate_matrix, :659-682): the sum over the 49 diagonal pairs of the window,
// (m(r, c) / 32, m(r + 1, c + 1) / 32), of (i - j)^2.  Every term is an integer
// and every partial sum stays below 2^24, so the reference's float sum is exact
// and equals the integer box sum computed here: D(y, x) = (q(y, x) - q(y + 1,
// x + 1))^2 with q = gray >> 5, summed over 7 x 7 starting at (row - 4, col - 4).
// Other pixels hold 0, so the map's minimum is 0, and cv::normalize(NORM_MINMAX,
// 0, 255) multiplies by scale = (float)(255 * (1 / max)) (double arithmetic; 0 for
// a map of zeros) and adds shift = 0.
//
// pm_glcm_kernel: one CTA per 64 x 16 output tile; the quantised raw, D and the
// horizontal 7-sums live in shared memory (6 KB), the vertical 7-sum gives the
// contrast (at most 49 * 49, a 16-bit map), and the CTA's maximum goes to *cmax
// by one atomicMax.  pm_richness_kernel: one CTA per view; scales its window of
// the map, thresholds it at 10 (cv::threshold, THRESH_BINARY, then the 8-bit copy
// of DepthSolver::SliceAndIndicatlizeForMI) and counts the 255s
// (MLA_Problem::ComputeRichnessValue) with __syncthreads_count.
constexpr int kGlcmTX = 64, kGlcmTY = 16, kGlcmThreads = 256;

__global__ void __launch_bounds__(kGlcmThreads) pm_glcm_kernel(const uint8_t* __restrict__ raw, int raw_pitch, int W,
                                                             int H, uint16_t* __restrict__ contrast,
                                                             unsigned* __restrict__ cmax)
{
    __shared__ uint8_t q[kGlcmTY + 7][kGlcmTX + 8];
    __shared__ uint8_t d[kGlcmTY + 6][kGlcmTX + 8];
    __shared__ uint16_t hs[kGlcmTY + 6][kGlcmTX];
    __shared__ unsigned wmax[kGlcmThreads / 32];
    const int c0 = blockIdx.x * kGlcmTX, r0 = blockIdx.y * kGlcmTY, t = threadIdx.x;
    for (int i = t; i < (kGlcmTY + 7) * (kGlcmTX + 7); i += kGlcmThreads) {
        const int iy = i / (kGlcmTX + 7), ix = i % (kGlcmTX + 7);
        const int y = r0 - 4 + iy, x = c0 - 4 + ix;
        q[iy][ix] = (y >= 0 && y < H && x >= 0 && x < W) ? (uint8_t)(__ldg(raw + (size_t)y * raw_pitch + x) >> 5) : 0;
    }
    __syncthreads();
    for (int i = t; i < (kGlcmTY + 6) * (kGlcmTX + 6); i += kGlcmThreads) {
        const int iy = i / (kGlcmTX + 6), ix = i % (kGlcmTX + 6);
        const int e = (int)q[iy][ix] - (int)q[iy + 1][ix + 1];
        d[iy][ix] = (uint8_t)(e * e);
    }
    __syncthreads();
    for (int i = t; i < (kGlcmTY + 6) * kGlcmTX; i += kGlcmThreads) {
        const int iy = i / kGlcmTX, ox = i % kGlcmTX;
        int s = 0;
#pragma unroll
        for (int k = 0; k < 7; ++k) s += d[iy][ox + k];
        hs[iy][ox] = (uint16_t)s;
    }
    __syncthreads();
    unsigned m = 0;
    for (int i = t; i < kGlcmTY * kGlcmTX; i += kGlcmThreads) {
        const int oy = i / kGlcmTX, ox = i % kGlcmTX;
        const int row = r0 + oy, col = c0 + ox;
        if (row >= H || col >= W) continue;
        int s = 0;
        if (row >= 4 && row < H - 4 && col >= 4 && col < W - 4) {
#pragma unroll
            for (int k = 0; k < 7; ++k) s += hs[oy + k][ox];
        }
        contrast[(size_t)row * W + col] = (uint16_t)s;
        m = max(m, (unsigned)s);
    }
    m = __reduce_max_sync(0xffffffffu, m);
    if ((t & 31) == 0) wmax[t >> 5] = m;
    __syncthreads();
    if (t < 32) {
        unsigned v = t < kGlcmThreads / 32 ? wmax[t] : 0u;
        v = __reduce_max_sync(0xffffffffu, v);
        if (t == 0 && v) atomicMax(cmax, v);
    }
}

__global__ void __launch_bounds__(128) pm_richness_kernel(const uint16_t* __restrict__ contrast, int W,
                                                          const int2* __restrict__ origin, int mi_w, int mi_h,
                                                          const unsigned* __restrict__ cmax, float* __restrict__ score,
                                                          uint8_t* __restrict__ binary, uint32_t* __restrict__ counts)
{
    const int v = blockIdx.x;
    const int2 o = origin[v];
    const int ppv = mi_w * mi_h;
    const unsigned mx = *cmax;
    const float scale = (float)(255.0 * (mx ? 1.0 / (double)mx : 0.0));
    uint32_t rich = 0;
    for (int base = 0; base < ppv; base += blockDim.x) {
        const int e = base + threadIdx.x;
        bool hit = false;
        if (e < ppv) {
            const int x = o.x + e % mi_w, y = o.y + e / mi_w;
            const float s = __fadd_rn(__fmul_rn((float)contrast[(size_t)y * W + x], scale), 0.0f);
            hit = s > 10.0f;
            if (score) score[(size_t)v * ppv + e] = s;
            if (binary) binary[(size_t)v * ppv + e] = hit ? 255 : 0;
        }
        if (counts) rich += (uint32_t)__syncthreads_count(hit);
    }
    if (counts && threadIdx.x == 0) counts[v] = rich;
}

cudaError_t launch_richness(const uint8_t* raw, int raw_pitch, int W, int H, const int2* origin, int V, int mi_w,
                            int mi_h, uint16_t* contrast, unsigned* cmax, float* score, uint8_t* binary,
                            uint32_t* counts, cudaStream_t st)
{
    const unsigned gx = (unsigned)((W + kGlcmTX - 1) / kGlcmTX), gy = (unsigned)((H + kGlcmTY - 1) / kGlcmTY);
    if (W <= 0 || H <= 0 || gy > 65535u) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(cmax, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    pm_glcm_kernel<<<dim3(gx, gy), kGlcmThreads, 0, st>>>(raw, raw_pitch, W, H, contrast, cmax);
    e = cudaGetLastError();
    if (e != cudaSuccess || V <= 0) return e;
    pm_richness_kernel<<<V, 128, 0, st>>>(contrast, W, origin, mi_w, mi_h, cmax, score, binary, counts);
    return cudaGetLastError();
}

cudaError_t launch_blur(const uint8_t* raw, int raw_pitch, int W, int H, const int2* origin, int V, int mi_w,
                        int mi_h, int tile_stride, uint8_t* tiles, uint32_t* counts, cudaStream_t st)
{
    if (V <= 0) return cudaSuccess;
    pm_blur_kernel<<<V, 128, 0, st>>>(raw, raw_pitch, W, H, origin, mi_w, mi_h, tile_stride, tiles, counts);
    return cudaGetLastError();
}

}  // namespace pfd
