// fuse_kernels.cu -- LFRefocus::FuseVirtualDepth_BackProject (FocalStack/
// LFRefocus.cpp:1553-1794) on the device.
//
// The reference visits the reference micro-images in map order and their
// pixels row by row; a pixel that finds at least two consistent neighbour
// pixels becomes a fused point and masks the neighbour pixels it used, which
// everything after it then skips.  Two micro-images depend on each other only
// through the masks of the micro-images they both touch (themselves and their
// list entries), so the host groups them into wavefront steps in which no two
// touch a common micro-image, ordered so that every dependent pair keeps the
// reference's order; a step runs one warp per micro-image, pixel after pixel,
// the warp's lanes taking the neighbour-list entries.  Consistent neighbours
// are summed in list order by shuffles, so every float is the reference's.
// Points that land on the same raw pixel overwrite each other in map order in
// the reference; here each records its sequence number (micro-image, pixel)
// with atomicMax and the maps are written from the last one afterwards.
#include <climits>
#include <cstdint>
#include "fuse_kernels.h"

namespace pfd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kInvalidImage = -9999.0f;         // g_Invalid_image, Common/Common.cpp:53

// x86 conversions of the reference's host code: (int) truncates, cvRound
// rounds half to even; NaN and out-of-range values give INT_MIN.
__device__ __forceinline__ int trunc_x86(float x) { return fabsf(x) < 2147483648.0f ? __float2int_rz(x) : INT_MIN; }
__device__ __forceinline__ int round_x86(float x) { return fabsf(x) < 2147483648.0f ? __float2int_rn(x) : INT_MIN; }
__device__ __forceinline__ uint8_t sat_u8(float v)
{
    const int i = round_x86(v);
    return (uint8_t)(i < 0 ? 0 : (i > 255 ? 255 : i));
}

// ComputeVirtualDepth (:2087-2098): a float base over a double disparity.
__device__ __forceinline__ float virtual_depth(float mla_base, float disp)
{
    const double d = (double)disp;
    if (d <= 0.0) return kInvalidImage;
    return __double2float_rn(__ddiv_rn((double)mla_base, d));
}

// ComputeVirtual3D (:2100-2117)
__device__ __forceinline__ float3 virtual_3d(float vd, int col, int row, float cm, float2 c)
{
    return make_float3(__fadd_rn(__fmul_rn(__fsub_rn((float)col, cm), vd), c.x),
                       __fadd_rn(__fmul_rn(__fsub_rn((float)row, cm), vd), c.y), vd);
}

// BackProject2MI (:2119-2125)
__device__ __forceinline__ float2 back_project(float3 P, float2 c, float cm)
{
    return make_float2(__fadd_rn(__fdiv_rn(__fsub_rn(P.x, c.x), P.z), cm),
                       __fadd_rn(__fdiv_rn(__fsub_rn(P.y, c.y), P.z), cm));
}

__device__ __forceinline__ float3 colour(const FuseFrame& F, int v, int idx)
{
    if (F.bgr) {
        const uint8_t* p = F.bgr + ((size_t)v * F.ppv + idx) * 3;
        return make_float3((float)p[0], (float)p[1], (float)p[2]);
    }
    const float g = (float)F.gray[(size_t)v * F.tile_stride + idx];
    return make_float3(g, g, g);
}

__device__ __forceinline__ bool valid_vd(float vd)
{
    return !(fabsf(__fsub_rn(vd, kInvalidImage)) < 1.0e-6f) && isfinite(vd);
}

}  // namespace

__global__ void __launch_bounds__(128) pm_fuse_step_kernel(FuseFrame F, const int* __restrict__ views, int n)
{
    const int lane = threadIdx.x & 31;
    const int wi = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (wi >= n) return;                              // whole warps leave together
    const int v = views[wi];
    const int m = F.m, ppv = F.ppv;
    const float cm = __fadd_rn(__fmul_rn((float)(m - 1), 0.5f), 1.0f);
    const float2 cr = F.centers[v];
    const int nl = min(F.list_counts[v], F.max_list);
    const int nch = (nl + 31) >> 5;
    int uj[kFuseMaxList / 32];
    float2 cj[kFuseMaxList / 32];
#pragma unroll
    for (int ch = 0; ch < kFuseMaxList / 32; ++ch) {
        const int j = ch * 32 + lane;
        uj[ch] = (j < nl) ? F.lists[(size_t)v * F.max_list + j] : -1;
        cj[ch] = uj[ch] >= 0 ? F.centers[uj[ch]] : make_float2(0.f, 0.f);
    }
    for (int idx = 0; idx < ppv; ++idx) {
        if (F.mask[(size_t)v * ppv + idx] == 1) continue;
        const float4 pl = F.plane[(size_t)v * ppv + idx];
        if (pl.w < F.min_ref_disp) continue;
        const float vdr = virtual_depth(F.mla_base, pl.w);
        if (!valid_vd(vdr)) continue;
        const int r = idx / m, c = idx - r * m;
        const float3 P = virtual_3d(vdr, c, r, cm, cr);
        float3 sp = P, sn = make_float3(pl.x, pl.y, pl.z), sc = colour(F, v, idx);
        int num = 0;
        bool ok[kFuseMaxList / 32];
        int usi[kFuseMaxList / 32];
#pragma unroll
        for (int ch = 0; ch < kFuseMaxList / 32; ++ch) {
            ok[ch] = false;
            usi[ch] = 0;
            if (ch >= nch) continue;                  // uniform
            const int u = uj[ch];
            float3 Ps = make_float3(0.f, 0.f, 0.f), Ns = Ps, Cs = Ps;
            if (u >= 0) {
                const float2 q = back_project(P, cj[ch], cm);
                const int src_r = trunc_x86(__fadd_rn(q.y, 0.5f)), src_c = trunc_x86(__fadd_rn(q.x, 0.5f));
                if (src_c >= 0 && src_c < m && src_r >= 0 && src_r < m) {
                    const int si = src_r * m + src_c;
                    if (F.mask[(size_t)u * ppv + si] != 1) {
                        const float4 ps = F.plane[(size_t)u * ppv + si];
                        if (!(ps.w <= 0.0f)) {
                            const float vds = virtual_depth(F.mla_base, ps.w);
                            if (valid_vd(vds)) {
                                Ps = virtual_3d(vds, src_c, src_r, cm, cj[ch]);
                                const float2 rq = back_project(Ps, cr, cm);
                                const float ex = __fsub_rn((float)c, rq.x), ey = __fsub_rn((float)r, rq.y);
                                const float err = __fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)));
                                const float den = vdr < 1.0e-6f ? 1.0e-6f : vdr;
                                const float rel = __fdiv_rn(fabsf(__fsub_rn(vds, vdr)), den);
                                if (err < F.max_reproj_px && rel < F.max_rel_vd) {
                                    ok[ch] = true;
                                    usi[ch] = si;
                                    Ns = make_float3(ps.x, ps.y, ps.z);
                                    Cs = colour(F, u, si);
                                }
                            }
                        }
                    }
                }
            }
            // the consistent entries of this chunk, summed in list order
            unsigned bits = __ballot_sync(kFull, ok[ch]);
            num += __popc(bits);
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                sp.x = __fadd_rn(sp.x, __shfl_sync(kFull, Ps.x, b));
                sp.y = __fadd_rn(sp.y, __shfl_sync(kFull, Ps.y, b));
                sp.z = __fadd_rn(sp.z, __shfl_sync(kFull, Ps.z, b));
                sn.x = __fadd_rn(sn.x, __shfl_sync(kFull, Ns.x, b));
                sn.y = __fadd_rn(sn.y, __shfl_sync(kFull, Ns.y, b));
                sn.z = __fadd_rn(sn.z, __shfl_sync(kFull, Ns.z, b));
                sc.x = __fadd_rn(sc.x, __shfl_sync(kFull, Cs.x, b));
                sc.y = __fadd_rn(sc.y, __shfl_sync(kFull, Cs.y, b));
                sc.z = __fadd_rn(sc.z, __shfl_sync(kFull, Cs.z, b));
            }
        }
        if (num >= F.min_consistent) {
            // cv::Vec3f /= float multiplies by the float reciprocal
            const float ia = __fdiv_rn(1.0f, __fadd_rn((float)num, 1.0f));
            sp = make_float3(__fmul_rn(sp.x, ia), __fmul_rn(sp.y, ia), __fmul_rn(sp.z, ia));
            sn = make_float3(__fmul_rn(sn.x, ia), __fmul_rn(sn.y, ia), __fmul_rn(sn.z, ia));
            sc = make_float3(__fmul_rn(sc.x, ia), __fmul_rn(sc.y, ia), __fmul_rn(sc.z, ia));
            const int vx = round_x86(sp.x), vy = round_x86(sp.y);
            if (lane == 0 && vy >= 0 && vy < F.raw_h && vx >= 0 && vx < F.raw_w) {
                const size_t seq = (size_t)v * ppv + idx;
                float* rec = F.rec + seq * 10;
                rec[0] = sp.x; rec[1] = sp.y; rec[2] = sp.z;
                rec[3] = sn.x; rec[4] = sn.y; rec[5] = sn.z;
                rec[6] = sc.x; rec[7] = sc.y; rec[8] = sc.z;
                rec[9] = (float)num;
                F.has_rec[seq] = 1u;
                atomicMax(&F.winner[(size_t)vy * F.raw_w + vx], (unsigned int)seq + 1u);
            }
#pragma unroll
            for (int ch = 0; ch < kFuseMaxList / 32; ++ch)
                if (ok[ch]) F.mask[(size_t)uj[ch] * ppv + usi[ch]] = 1;
        }
        __syncwarp();                                 // this pixel's masks before the next pixel reads them
    }
}

__global__ void pm_fuse_maps_kernel(FuseFrame F, float* __restrict__ vd_map, uint8_t* __restrict__ conf,
                                    uint8_t* __restrict__ aif)
{
    const size_t n = (size_t)F.raw_w * F.raw_h;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
        const unsigned s = F.winner[o];
        float z = 0.0f;
        uint8_t cf = 0, b = 0, g = 0, rr = 0;
        if (s) {
            const float* rec = F.rec + (size_t)(s - 1u) * 10;
            z = rec[2];
            const int k = ((int)rec[9] + 1) * 60;
            cf = (uint8_t)(k < 255 ? k : 255);
            b = sat_u8(rec[6]);
            g = sat_u8(rec[7]);
            rr = sat_u8(rec[8]);
        }
        vd_map[o] = z;
        conf[o] = cf;
        aif[3 * o + 0] = b;
        aif[3 * o + 1] = g;
        aif[3 * o + 2] = rr;
    }
}

__global__ void __launch_bounds__(kFuseScanBlock) pm_fuse_count_kernel(FuseFrame F, unsigned int* block_counts)
{
    const size_t n = (size_t)F.V * F.ppv;
    const size_t s = (size_t)blockIdx.x * kFuseScanBlock + threadIdx.x;
    const unsigned f = (s < n) ? F.has_rec[s] : 0u;
    const unsigned c = __syncthreads_count(f != 0u);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

__global__ void __launch_bounds__(kFuseScanBlock) pm_fuse_compact_kernel(FuseFrame F, const unsigned int* block_offsets,
                                                                          float* points)
{
    __shared__ unsigned warp_base[kFuseScanBlock / 32];
    const size_t n = (size_t)F.V * F.ppv;
    const size_t s = (size_t)blockIdx.x * kFuseScanBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool f = (s < n) && F.has_rec[s] != 0u;
    const unsigned bits = __ballot_sync(kFull, f);
    if (lane == 0) warp_base[w] = __popc(bits);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int i = 0; i < kFuseScanBlock / 32; ++i) { const unsigned t = warp_base[i]; warp_base[i] = acc; acc += t; }
    }
    __syncthreads();
    if (f) {
        const size_t o = (size_t)block_offsets[blockIdx.x] + warp_base[w] + __popc(bits & ((1u << lane) - 1u));
        const float* rec = F.rec + s * 10;
        for (int i = 0; i < 9; ++i) points[o * 9 + i] = rec[i];
    }
}

cudaError_t launch_fuse_step(const FuseFrame& F, const int* views, int n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    pm_fuse_step_kernel<<<(n + 3) / 4, 128, 0, st>>>(F, views, n);
    return cudaGetLastError();
}

cudaError_t launch_fuse_maps(const FuseFrame& F, float* vd_map, uint8_t* conf, uint8_t* aif, cudaStream_t st)
{
    const size_t n = (size_t)F.raw_w * F.raw_h;
    const int grid = (int)((n + 255) / 256 < (size_t)148 * 16 ? (n + 255) / 256 : (size_t)148 * 16);
    pm_fuse_maps_kernel<<<grid > 0 ? grid : 1, 256, 0, st>>>(F, vd_map, conf, aif);
    return cudaGetLastError();
}

cudaError_t launch_fuse_count(const FuseFrame& F, unsigned int* block_counts, cudaStream_t st)
{
    const size_t n = (size_t)F.V * F.ppv;
    const int nb = (int)((n + kFuseScanBlock - 1) / kFuseScanBlock);
    pm_fuse_count_kernel<<<nb, kFuseScanBlock, 0, st>>>(F, block_counts);
    return cudaGetLastError();
}

cudaError_t launch_fuse_compact(const FuseFrame& F, const unsigned int* block_offsets, float* points, cudaStream_t st)
{
    const size_t n = (size_t)F.V * F.ppv;
    const int nb = (int)((n + kFuseScanBlock - 1) / kFuseScanBlock);
    pm_fuse_compact_kernel<<<nb, kFuseScanBlock, 0, st>>>(F, block_offsets, points);
    return cudaGetLastError();
}

}  // namespace pfd
