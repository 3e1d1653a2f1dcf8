// refocus_kernels.cu -- focal-stack render on the device.
//
// The reference has no multi-slice render; this one is defined from its
// back-projection LFRefocus::BackProject2MI (FocalStack/LFRefocus.cpp:2119-2125):
// output pixel (ox, oy) of slice s lies at raw coordinates
// X = (ox + 0.5) * (W / out_w) - 0.5, and micro-image i sees it at
// u = (X - c_i) / vd_s + ((m-1)/2 + 1)  (the centre of FuseVirtualDepth_BackProject,
// :1635-1636).  Every micro-image whose u falls in [0, m-1]^2 contributes its
// bilinear gray sample; the output is the mean, summed in ascending view index.
//
// One CTA renders a 64 x 16 output tile of one slice.  The lenses that can reach
// the tile are gathered from a bucket grid of lens centres, sorted by view
// index (so the sum order is the oracle's), and their micro-images are staged
// through shared memory in chunks.  A warp owns output rows, so the row test of
// a lens is warp-uniform; each lane owns two columns.
#include <cstdint>
#include <cuda_runtime.h>
#include "refocus_kernels.h"

namespace pfd {

namespace {

constexpr int kTileW = 64, kTileH = 16, kThreads = 256;
constexpr int kChunk = 128;              // micro-images staged per pass

}  // namespace

__global__ void __launch_bounds__(kThreads) pm_refocus_kernel(RefocusFrame F, const float* slice_vd, int out_w,
                                                               int out_h, float sx, float sy, float* out, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    int* cand = (int*)smem;                                  // [kMaxRefocusCand] gathered
    int* sorted = cand + kMaxRefocusCand;                    // [kMaxRefocusCand] ascending
    float2* cc = (float2*)(sorted + kMaxRefocusCand);        // [kChunk] centres of the staged chunk
    uint8_t* tiles = (uint8_t*)(cc + kChunk);                // [kChunk][tile_stride]
    __shared__ int n_cand;

    const int s = blockIdx.z;
    const float v = slice_vd[s];
    const int ox0 = blockIdx.x * kTileW, oy0 = blockIdx.y * kTileH;
    const int m = F.m, mh = F.mh;
    const float cmx = (float)(m - 1) * 0.5f + 1.0f, cmy = (float)(mh - 1) * 0.5f + 1.0f;
    const float umax = (float)(m - 1), wmax = (float)(mh - 1);

    // ---- lenses that can reach the tile ------------------------------------
    const int ex = min(ox0 + kTileW, out_w) - 1, ey = min(oy0 + kTileH, out_h) - 1;
    const float X0 = ((float)ox0 + 0.5f) * sx - 0.5f, X1 = ((float)ex + 0.5f) * sx - 0.5f;
    const float Y0 = ((float)oy0 + 0.5f) * sy - 0.5f, Y1 = ((float)ey + 0.5f) * sy - 0.5f;
    const float bx0 = X0 - (umax - cmx) * v - 1.0f, bx1 = X1 + cmx * v + 1.0f;
    const float by0 = Y0 - (wmax - cmy) * v - 1.0f, by1 = Y1 + cmy * v + 1.0f;
    const float inv_cell = 1.0f / F.cell;
    const int gx0 = max(0, (int)floorf((bx0 - F.grid_x0) * inv_cell));
    const int gx1 = min(F.grid_w - 1, (int)floorf((bx1 - F.grid_x0) * inv_cell));
    const int gy0 = max(0, (int)floorf((by0 - F.grid_y0) * inv_cell));
    const int gy1 = min(F.grid_h - 1, (int)floorf((by1 - F.grid_y0) * inv_cell));
    if (threadIdx.x == 0) n_cand = 0;
    __syncthreads();
    if (gx1 >= gx0 && gy1 >= gy0) {
        const int gw = gx1 - gx0 + 1, ncell = gw * (gy1 - gy0 + 1);
        for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
            const int cell = (gy0 + c / gw) * F.grid_w + gx0 + c % gw;
            for (int k = F.cell_start[cell]; k < F.cell_start[cell + 1]; ++k) {
                const int id = F.cell_ids[k];
                const float2 p = F.centers[id];
                if (p.x < bx0 || p.x > bx1 || p.y < by0 || p.y > by1) continue;
                const int slot = atomicAdd(&n_cand, 1);
                if (slot < kMaxRefocusCand) cand[slot] = id;
            }
        }
    }
    __syncthreads();
    int n = n_cand;
    if (n > kMaxRefocusCand) {
        if (threadIdx.x == 0) atomicOr(err, PFD_DEVERR_REFOCUS_LENSES);
        n = kMaxRefocusCand;
    }
    // rank sort: ids are distinct
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int id = cand[i];
        int r = 0;
        for (int j = 0; j < n; ++j) r += cand[j] < id;
        sorted[r] = id;
    }

    // ---- accumulate ----------------------------------------------------------
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float sum[2][2] = { { 0.f, 0.f }, { 0.f, 0.f } };
    int cnt[2][2] = { { 0, 0 }, { 0, 0 } };
    float Xa[2], Yb[2];
    for (int a = 0; a < 2; ++a) Xa[a] = ((float)(ox0 + lane + 32 * a) + 0.5f) * sx - 0.5f;
    for (int b = 0; b < 2; ++b) Yb[b] = ((float)(oy0 + warp + 8 * b) + 0.5f) * sy - 0.5f;
    const int words = F.tile_stride / 16;
    for (int base = 0; base < n; base += kChunk) {
        const int nc = min(kChunk, n - base);
        __syncthreads();                                      // sorted[] ready / previous chunk consumed
        for (int e = threadIdx.x; e < nc * words; e += blockDim.x) {
            const int t = e / words, wd = e % words;
            const uint4* src = (const uint4*)(F.gray + (size_t)sorted[base + t] * F.tile_stride);
            ((uint4*)(tiles + (size_t)t * F.tile_stride))[wd] = src[wd];
        }
        for (int t = threadIdx.x; t < nc; t += blockDim.x) cc[t] = F.centers[sorted[base + t]];
        __syncthreads();
        for (int t = 0; t < nc; ++t) {
            const float2 c = cc[t];
            const uint8_t* T = tiles + (size_t)t * F.tile_stride;
            // the column coordinates do not depend on the row: one division per column
            float ua[2];
            for (int a = 0; a < 2; ++a) ua[a] = __fadd_rn(__fdiv_rn(__fsub_rn(Xa[a], c.x), v), cmx);
            for (int b = 0; b < 2; ++b) {
                const float w = __fadd_rn(__fdiv_rn(__fsub_rn(Yb[b], c.y), v), cmy);   // warp-uniform
                if (!(w >= 0.0f && w <= wmax)) continue;
                const int y0 = (int)floorf(w);
                const int y1 = min(y0 + 1, mh - 1);
                const float ay = __fsub_rn(w, (float)y0);
                for (int a = 0; a < 2; ++a) {
                    const float u = ua[a];
                    if (!(u >= 0.0f && u <= umax)) continue;
                    const int x0 = (int)floorf(u);
                    const int x1 = min(x0 + 1, m - 1);
                    const float ax = __fsub_rn(u, (float)x0);
                    const float t00 = (float)T[y0 * m + x0], t01 = (float)T[y0 * m + x1];
                    const float t10 = (float)T[y1 * m + x0], t11 = (float)T[y1 * m + x1];
                    const float top = __fmaf_rn(ax, __fsub_rn(t01, t00), t00);
                    const float bot = __fmaf_rn(ax, __fsub_rn(t11, t10), t10);
                    sum[b][a] = __fadd_rn(sum[b][a], __fmaf_rn(ay, __fsub_rn(bot, top), top));
                    cnt[b][a] += 1;
                }
            }
        }
    }
    float* o = out + (size_t)s * out_h * out_w;
    for (int b = 0; b < 2; ++b) {
        const int oy = oy0 + warp + 8 * b;
        if (oy >= out_h) continue;
        for (int a = 0; a < 2; ++a) {
            const int ox = ox0 + lane + 32 * a;
            if (ox >= out_w) continue;
            o[(size_t)oy * out_w + ox] = cnt[b][a] ? __fdiv_rn(sum[b][a], (float)cnt[b][a]) : 0.0f;
        }
    }
}

int refocus_smem_bytes(const RefocusFrame& F)
{
    return 2 * kMaxRefocusCand * 4 + kChunk * 8 + kChunk * F.tile_stride;
}

cudaError_t launch_refocus(const RefocusFrame& F, const float* slice_vd, int n_slices, int raw_w, int raw_h, int out_w,
                           int out_h, float* out, int* err, cudaStream_t st)
{
    if (n_slices <= 0) return cudaSuccess;
    const int smem = refocus_smem_bytes(F);
    cudaError_t e = cudaFuncSetAttribute(pm_refocus_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const float sx = (float)raw_w / (float)out_w, sy = (float)raw_h / (float)out_h;
    const dim3 grid((out_w + kTileW - 1) / kTileW, (out_h + kTileH - 1) / kTileH, n_slices);
    pm_refocus_kernel<<<grid, kThreads, smem, st>>>(F, slice_vd, out_w, out_h, sx, sy, out, err);
    return cudaGetLastError();
}

}  // namespace pfd
