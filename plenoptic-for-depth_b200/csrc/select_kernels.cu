// select_kernels.cu -- MISimilarityMeasure::MeasureSimilarity (Util/
// MISimilarityMeasure.cpp:173-284) for many (micro-image, candidate) pairs,
// one warp per pair.
//
// Both micro-images are binarised (threshold 128: 255 above, 0 otherwise).
// The candidate is shifted along the baseline in steps of 2 px; for every
// step the warp counts, over the overlap rectangle, the pixels where the
// reference micro-image equals the shifted candidate, and the similarity is
// the largest count.  The shift loop follows the reference as it runs (an
// OpenMP loop nested in a parallel region, hence sequential): step k uses the
// shift step k - 1 left behind (0 for steps 0 and 1), and once the shift
// leaves the image it stays there.  The shifted candidate is
// cv::warpAffine(INTER_NEAREST) of a translation, OpenCV's 10-bit fixed
// point: source column x + floor((rnd(-1024 sx) + 512) / 1024), source row
// floor((rnd(1024 (y - sy)) + 512) / 1024), rnd rounding half to even, 0
// outside.  Integer conversions of the host code follow x86 (NaN and
// out-of-range values give INT_MIN).
#include <climits>
#include <cstdint>
#include "select_kernels.h"

namespace pfd {

namespace {

__device__ __forceinline__ int trunc_x86(float x) { return fabsf(x) < 2147483648.0f ? __float2int_rz(x) : INT_MIN; }
__device__ __forceinline__ int round_x86(double x) { return fabs(x) < 2147483648.0 ? __double2int_rn(x) : INT_MIN; }

}  // namespace

__global__ void __launch_bounds__(128) pm_similarity_kernel(const uint8_t* __restrict__ gray, int tile_stride, int W,
                                                            int H, const float2* __restrict__ centers,
                                                            const int2* __restrict__ pairs, int n,
                                                            int* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int p = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (p >= n) return;
    const int2 pr = pairs[p];
    const uint8_t* src = gray + (size_t)pr.x * tile_stride;
    const uint8_t* nb = gray + (size_t)pr.y * tile_stride;
    float dx = __fsub_rn(centers[pr.y].x, centers[pr.x].x), dy = __fsub_rn(centers[pr.y].y, centers[pr.x].y);
    if (fabsf(dx) < 5.0f) dx = 0.0f;
    if (fabsf(dy) < 5.0f) dy = 0.0f;
    const float norm = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    const float dxs = __fmul_rn(__fdiv_rn(dx, norm), 2.0f), dys = __fmul_rn(__fdiv_rn(dy, norm), 2.0f);
    int dxc = trunc_x86(__fdiv_rn((float)W, fabsf(dxs)));
    int dyc = trunc_x86(__fdiv_rn((float)H, fabsf(dys)));
    if (dxs == 0.0f) dxc = 0;
    else if (dys == 0.0f) dyc = 0;
    const int steps = dxc > dyc ? dxc : dyc;
    int best = 0;
    float sx = 0.0f, sy = 0.0f;
    for (int step = 0; step < steps && step < 4096; ++step) {
        // once the shift leaves the image the reference skips every later step (its
        // shift is only advanced by a step that ran), so nothing more can count
        if (fabsf(sx) >= (float)W || fabsf(sy) >= (float)H) break;
        const int X0 = round_x86(__dmul_rn((double)(-sx), 1024.0)) + 512;
        const int x1 = (int)(0.0f < sx ? sx : 0.0f), y1 = (int)(0.0f < sy ? sy : 0.0f);
        const float ex = __fsub_rn(__fadd_rn(sx, (float)W), 1.0f), ey = __fsub_rn(__fadd_rn(sy, (float)H), 1.0f);
        const int x2 = (int)floorf(ex < (float)(W - 1) ? ex : (float)(W - 1));
        const int y2 = (int)floorf(ey < (float)(H - 1) ? ey : (float)(H - 1));
        int c = 0;
        if (x2 >= x1 && y2 >= y1) {
            const int rw = x2 - x1 + 1, area = rw * (y2 - y1 + 1);
            for (int e = lane; e < area; e += 32) {
                const int y = y1 + e / rw, x = x1 + e % rw;
                const int Y = (round_x86(__dmul_rn(__dadd_rn((double)y, (double)(-sy)), 1024.0)) + 512) >> 10;
                const int X = (X0 + x * 1024) >> 10;
                const uint8_t v = (X >= 0 && X < W && Y >= 0 && Y < H) ? (nb[Y * W + X] > 128 ? 255 : 0) : 0;
                c += ((src[y * W + x] > 128 ? 255 : 0) == v) ? 1 : 0;
            }
        }
        c = __reduce_add_sync(0xffffffffu, c);
        if (c > best) best = c;
        sx = __fmul_rn((float)step, dxs);
        sy = __fmul_rn((float)step, dys);
    }
    if (lane == 0) out[p] = best;
}

cudaError_t launch_similarity(const uint8_t* gray, int tile_stride, int W, int H, const float2* centers,
                              const int2* pairs, int n, int* out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    pm_similarity_kernel<<<(n + 3) / 4, 128, 0, st>>>(gray, tile_stride, W, H, centers, pairs, n, out);
    return cudaGetLastError();
}

}  // namespace pfd
