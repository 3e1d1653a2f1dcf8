// vdrd_kernels.cu -- virtual depth to real depth (FocalStack/LFRefocus.cpp:
// 2515-2593, FocalStack/VirtualToRealDepthFunc.cpp:3390-3450) in FP64.
//
// The conversions are elementwise and HBM-bound (4 bytes in, 8 or 4 out per
// pixel); each thread handles four consecutive pixels with one 16-byte load.
// Every expression is evaluated as written (the library is built with
// -fmad=false; double division is IEEE).
#include <algorithm>
#include <cstdint>
#include "vdrd_kernels.h"

namespace pfd {

namespace {

__device__ __forceinline__ double vd_map_one(float vdepth, double c0, double c1, double c2)
{
    const double v = (double)vdepth;
    const double num = __dadd_rn(__dmul_rn(v, c1), c2);
    const double den = __dsub_rn(1.0, __dmul_rn(v, c0));
    double z = __ddiv_rn(num, den);
    if (isnan(z) || isinf(z) || z < 0.0) z = 0.0;
    return z;
}

__device__ __forceinline__ float vd_point_one(float vdepth, double c0, double c1, double c2)
{
    const double v = (double)vdepth;
    const double denom = __dsub_rn(1.0, __dmul_rn(v, c0));
    if (fabs(denom) < 1.0e-12) return 0.0f;
    const double z = __ddiv_rn(__dadd_rn(__dmul_rn(v, c1), c2), denom);
    if (!isfinite(z) || z < 0.0) return 0.0f;
    return (float)z;
}

}  // namespace

__global__ void pm_vd_to_rd_kernel(const float* __restrict__ vd, size_t n, double c0, double c1, double c2, int mode,
                                   void* __restrict__ out)
{
    const size_t nv = n / 4;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const bool aligned = ((uintptr_t)vd & 15) == 0 && ((uintptr_t)out & 15) == 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (aligned ? nv : 0); i += stride) {
        const float4 v = ((const float4*)vd)[i];
        if (mode == 0) {
            double2* o = (double2*)out + 2 * i;
            o[0] = make_double2(vd_map_one(v.x, c0, c1, c2), vd_map_one(v.y, c0, c1, c2));
            o[1] = make_double2(vd_map_one(v.z, c0, c1, c2), vd_map_one(v.w, c0, c1, c2));
        } else {
            ((float4*)out)[i] = make_float4(vd_point_one(v.x, c0, c1, c2), vd_point_one(v.y, c0, c1, c2),
                                            vd_point_one(v.z, c0, c1, c2), vd_point_one(v.w, c0, c1, c2));
        }
    }
    for (size_t i = (aligned ? 4 * nv : 0) + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (mode == 0) ((double*)out)[i] = vd_map_one(vd[i], c0, c1, c2);
        else ((float*)out)[i] = vd_point_one(vd[i], c0, c1, c2);
    }
}

__global__ void pm_vd_to_rd_segments_kernel(const float* __restrict__ vd, size_t n, const double* __restrict__ segs,
                                            int nseg, float* __restrict__ out)
{
    __shared__ double sg[kMaxVdSegments * 5];
    for (int i = threadIdx.x; i < nseg * 5; i += blockDim.x) sg[i] = segs[i];
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float vdepth = vd[i];
        const double v = (double)vdepth;
        double z = 0.0;
        float r = -1.0f;                      // -1: no early return taken
        for (int s = 0; s < nseg; ++s) {
            const double* g = sg + 5 * s;
            if (v >= g[0] && v < g[1]) {
                const double denom = __dsub_rn(1.0, __dmul_rn(v, g[2]));
                if (fabs(denom) < 1.0e-12) { r = 0.0f; break; }
                z = __ddiv_rn(__dadd_rn(__dmul_rn(v, g[3]), g[4]), denom);
                break;
            }
        }
        if (r < 0.0f) r = (!isfinite(z) || z < 0.0) ? 0.0f : (float)z;
        out[i] = r;
    }
}

// Per block, the normal-equation sums over a contiguous chunk, reduced in a fixed
// tree order (deterministic for a given n and grid).
__global__ void pm_fit_sums_kernel(const float* __restrict__ real_depth, const float* __restrict__ vd, size_t n,
                                   size_t chunk, double* __restrict__ partial)
{
    double a[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    const size_t lo = (size_t)blockIdx.x * chunk, hi = min(n, lo + chunk);
    for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double aL = real_depth[i], v = vd[i];
        const double x0 = __dmul_rn(aL, v), x1 = v;
        a[0] = __dadd_rn(a[0], __dmul_rn(x0, x0));
        a[1] = __dadd_rn(a[1], __dmul_rn(x0, x1));
        a[2] = __dadd_rn(a[2], x0);
        a[3] = __dadd_rn(a[3], __dmul_rn(x1, x1));
        a[4] = __dadd_rn(a[4], x1);
        a[5] = __dadd_rn(a[5], 1.0);
        a[6] = __dadd_rn(a[6], __dmul_rn(x0, aL));
        a[7] = __dadd_rn(a[7], __dmul_rn(x1, aL));
        a[8] = __dadd_rn(a[8], aL);
    }
    __shared__ double red[9][256];
    for (int q = 0; q < 9; ++q) red[q][threadIdx.x] = a[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int q = 0; q < 9; ++q) red[q][threadIdx.x] = __dadd_rn(red[q][threadIdx.x], red[q][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x < 9) partial[(size_t)blockIdx.x * 9 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void pm_fit_fold_kernel(const double* __restrict__ partial, int nblocks, double* __restrict__ sums)
{
    if (threadIdx.x >= 9) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s = __dadd_rn(s, partial[(size_t)b * 9 + threadIdx.x]);
    sums[threadIdx.x] = s;
}

cudaError_t launch_vd_to_rd(const float* vd, size_t n, double c0, double c1, double c2, int mode, void* out,
                            cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (n / 4 + 255) / 256 + 1;
    const int grid = (int)std::min<size_t>(want, (size_t)sms * 8);
    pm_vd_to_rd_kernel<<<grid, 256, 0, st>>>(vd, n, c0, c1, c2, mode, out);
    return cudaGetLastError();
}

cudaError_t launch_vd_to_rd_segments(const float* vd, size_t n, const double* segs, int nseg, float* out,
                                     cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)148 * 8);
    pm_vd_to_rd_segments_kernel<<<grid, 256, 0, st>>>(vd, n, segs, nseg, out);
    return cudaGetLastError();
}

int fit_blocks(size_t n)
{
    return (int)std::max<size_t>(1, std::min<size_t>((n + 4095) / 4096, 1024));
}

cudaError_t launch_fit_sums(const float* real_depth, const float* vd, size_t n, double* partial, double* sums,
                            cudaStream_t st)
{
    const int nb = fit_blocks(n);
    const size_t chunk = (n + nb - 1) / nb;
    pm_fit_sums_kernel<<<nb, 256, 0, st>>>(real_depth, vd, n, chunk, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pm_fit_fold_kernel<<<1, 32, 0, st>>>(partial, nb, sums);
    return cudaGetLastError();
}

}  // namespace pfd
