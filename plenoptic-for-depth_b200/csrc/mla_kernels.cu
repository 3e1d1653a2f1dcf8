// mla_kernels.cu -- micro-lens centre detection from a white image
// (DepthSolver::ComputeMLACentersFromWhiteImage, DepthSolver.cpp:710-870).
//
//   pm_mla_hist_kernel     the histogram DepthSolver::Otsu (:486-546) reads:
//                          the first W bytes of every row of the 3-channel image
//   pm_mla_label_kernel    BGR2GRAY (OpenCV's 8-bit 15-bit fixed point), the
//                          binary threshold, and one label per foreground pixel
//   pm_mla_union_kernel    8-connected components by union-find: every root
//                          ends as the component's smallest raster index, its
//                          first pixel, where the contour search of
//                          findContours(RETR_EXTERNAL) starts its border
//   pm_mla_roots_kernel    the component roots
//   pm_mla_trace_kernel    one thread per component: Suzuki-Abe outer border
//                          following from the root and the contour's polygon
//                          moments (Green's theorem), whose sums are exact
//                          integers in double, so the centroid m10/m00,
//                          m01/m00 and the area equal OpenCV's
#include <cstdint>
#include "mla_kernels.h"

namespace pfd {

namespace {

__constant__ int kDR[8] = { 0, -1, -1, -1, 0, 1, 1, 1 };      // counter-clockwise on screen
__constant__ int kDC[8] = { 1, 1, 0, -1, -1, -1, 0, 1 };

__device__ __forceinline__ int find_root(const int* L, int x)
{
    for (int it = 0; it < (1 << 26); ++it) {
        const int p = __ldcg(L + x);
        if (p == x) return x;
        x = p;
    }
    return x;
}

__device__ __forceinline__ void unite(int* L, int a, int b, int* err)
{
    for (int it = 0; it < (1 << 20); ++it) {
        a = find_root(L, a);
        b = find_root(L, b);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }       // link the larger root under the smaller
        const int old = atomicMin(L + a, b);
        if (old == a) return;
        a = old;
    }
    atomicOr(err, PFD_DEVERR_MLA_UNION);
}

}  // namespace

__global__ void pm_mla_hist_kernel(const uint8_t* __restrict__ bgr, int W, int H, int step, unsigned int* hist)
{
    __shared__ unsigned int h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const size_t n = (size_t)W * H;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e / W, j = e - r * W;
        atomicAdd(&h[bgr[r * step + j]], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(hist + i, h[i]);
}

__global__ void pm_mla_label_kernel(const uint8_t* __restrict__ bgr, int W, int H, int step, int threshold,
                                    uint8_t* __restrict__ fg, int* __restrict__ L)
{
    const size_t n = (size_t)W * H;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e / W, c = e - r * W;
        const uint8_t* p = bgr + r * step + 3 * c;
        const int g = ((int)p[0] * 3735 + (int)p[1] * 19235 + (int)p[2] * 9798 + 16384) >> 15;
        const bool on = g > threshold;
        fg[e] = on ? 1 : 0;
        L[e] = on ? (int)e : -1;
    }
}

__global__ void pm_mla_union_kernel(const uint8_t* __restrict__ fg, int W, int H, int* L, int* err)
{
    const size_t n = (size_t)W * H;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        if (!fg[e]) continue;
        const int r = (int)(e / W), c = (int)(e - (size_t)r * W);
        // the four neighbours before this pixel in raster order cover every 8-adjacent pair once
        if (c > 0 && fg[e - 1]) unite(L, (int)e, (int)e - 1, err);
        if (r > 0) {
            const size_t u = e - W;
            if (c > 0 && fg[u - 1]) unite(L, (int)e, (int)u - 1, err);
            if (fg[u]) unite(L, (int)e, (int)u, err);
            if (c < W - 1 && fg[u + 1]) unite(L, (int)e, (int)u + 1, err);
        }
    }
}

__global__ void pm_mla_roots_kernel(const uint8_t* __restrict__ fg, int W, int H, const int* L, int* roots,
                                    unsigned int* n_roots, int max_roots)
{
    const size_t n = (size_t)W * H;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        if (!fg[e] || find_root(L, (int)e) != (int)e) continue;
        const unsigned k = atomicAdd(n_roots, 1u);
        if ((int)k < max_roots) roots[k] = (int)e;
    }
}

__global__ void pm_mla_trace_kernel(const uint8_t* __restrict__ fg, int W, int H, const int* __restrict__ starts,
                                    int n, double* __restrict__ sums, int* err)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = starts[k];
    const int r0 = s / W, c0 = s - r0 * W;
    auto on = [&](int r, int c) { return r >= 0 && r < H && c >= 0 && c < W && fg[(size_t)r * W + c] != 0; };
    double a00 = 0.0, a10 = 0.0, a01 = 0.0;
    // (3.1) clockwise from the left neighbour for the first foreground pixel
    int d1 = -1;
    for (int i = 0; i < 8; ++i) {
        const int d = (4 - i + 8) & 7;
        if (on(r0 + kDR[d], c0 + kDC[d])) { d1 = d; break; }
    }
    if (d1 >= 0) {
        const int r1 = r0 + kDR[d1], c1 = c0 + kDC[d1];
        int r3 = r0, c3 = c0, d2 = d1;                    // direction from (r3, c3) to (r2, c2) = (r1, c1)
        double xp = c0, yp = r0;                          // the vertex before the next one
        bool closed = false;
        for (long long step = 0; step < 4LL * W * H + 8; ++step) {
            // (3.3) counter-clockwise around (r3, c3), from the element after (r2, c2)
            int d4 = -1;
            for (int i = 1; i <= 8; ++i) {
                const int d = (d2 + i) & 7;
                if (on(r3 + kDR[d], c3 + kDC[d])) { d4 = d; break; }
            }
            const int r4 = r3 + kDR[d4], c4 = c3 + kDC[d4];
            // (3.5)
            if (r4 == r0 && c4 == c0 && r3 == r1 && c3 == c1) { closed = true; break; }
            d2 = (d4 + 4) & 7;                            // (r2, c2) <- (r3, c3), seen from (r4, c4)
            r3 = r4; c3 = c4;
            const double x = c3, y = r3;
            const double dxy = xp * y - x * yp;
            a00 += dxy; a10 += dxy * (xp + x); a01 += dxy * (yp + y);
            xp = x; yp = y;
        }
        if (!closed) atomicOr(err, PFD_DEVERR_MLA_TRACE);
        // close the polygon: last vertex -> start
        const double x = c0, y = r0;
        const double dxy = xp * y - x * yp;
        a00 += dxy; a10 += dxy * (xp + x); a01 += dxy * (yp + y);
    }
    sums[3 * (size_t)k + 0] = a00;
    sums[3 * (size_t)k + 1] = a10;
    sums[3 * (size_t)k + 2] = a01;
}

// Normal equations of the hexagonal lattice model
//   x = ox + (col + (row & 1) / 2) a - row (sqrt(3) / 2) b
//   y = oy + (col + (row & 1) / 2) b + row (sqrt(3) / 2) a
// (lens pitch |(a, b)|, rotation atan2(b, a)), linear in (ox, oy, a, b): per
// block the 10 upper-triangle sums of A^T A and the 4 of A^T z over a chunk of
// lenses, reduced in a fixed tree order.
__global__ void pm_mla_lattice_kernel(const pfd_mla_lens_dev* __restrict__ lens, int n, int chunk, double* partial)
{
    double acc[14];
    for (int q = 0; q < 14; ++q) acc[q] = 0.0;
    const int lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    const double h3 = 0.86602540378443864676;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const pfd_mla_lens_dev L = lens[i];
        const double u = __dadd_rn((double)L.col, (L.row & 1) ? 0.5 : 0.0), w = __dmul_rn((double)L.row, h3);
        // rows of A for x and y: [1, 0, u, -w] and [0, 1, w, u]
        const double rx[4] = { 1.0, 0.0, u, -w }, ry[4] = { 0.0, 1.0, w, u };
        int q = 0;
        for (int i0 = 0; i0 < 4; ++i0)
            for (int i1 = i0; i1 < 4; ++i1, ++q)
                acc[q] = __dadd_rn(acc[q], __dadd_rn(__dmul_rn(rx[i0], rx[i1]), __dmul_rn(ry[i0], ry[i1])));
        for (int i0 = 0; i0 < 4; ++i0)
            acc[10 + i0] = __dadd_rn(acc[10 + i0], __dadd_rn(__dmul_rn(rx[i0], (double)L.cx), __dmul_rn(ry[i0], (double)L.cy)));
    }
    __shared__ double red[14][128];
    for (int q = 0; q < 14; ++q) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if ((int)threadIdx.x < s2)
            for (int q = 0; q < 14; ++q) red[q][threadIdx.x] = __dadd_rn(red[q][threadIdx.x], red[q][threadIdx.x + s2]);
        __syncthreads();
    }
    if (threadIdx.x < 14) partial[(size_t)blockIdx.x * 14 + threadIdx.x] = red[threadIdx.x][0];
}

cudaError_t launch_mla_lattice(const pfd_mla_lens_dev* lens, int n, double* partial, int nblocks, cudaStream_t st)
{
    const int chunk = (n + nblocks - 1) / nblocks;
    pm_mla_lattice_kernel<<<nblocks, 128, 0, st>>>(lens, n, chunk, partial);
    return cudaGetLastError();
}

static int grid_for(size_t n)
{
    const size_t g = (n + 255) / 256;
    return (int)(g < (size_t)148 * 16 ? (g > 0 ? g : 1) : (size_t)148 * 16);
}

cudaError_t launch_mla_hist(const uint8_t* bgr, int W, int H, int step, unsigned int* hist, cudaStream_t st)
{
    pm_mla_hist_kernel<<<grid_for((size_t)W * H), 256, 0, st>>>(bgr, W, H, step, hist);
    return cudaGetLastError();
}

cudaError_t launch_mla_components(const uint8_t* bgr, int W, int H, int step, int threshold, uint8_t* fg, int* L,
                                  int* roots, unsigned int* n_roots, int max_roots, int* err, cudaStream_t st)
{
    const int g = grid_for((size_t)W * H);
    pm_mla_label_kernel<<<g, 256, 0, st>>>(bgr, W, H, step, threshold, fg, L);
    pm_mla_union_kernel<<<g, 256, 0, st>>>(fg, W, H, L, err);
    pm_mla_roots_kernel<<<g, 256, 0, st>>>(fg, W, H, L, roots, n_roots, max_roots);
    return cudaGetLastError();
}

cudaError_t launch_mla_trace(const uint8_t* fg, int W, int H, const int* starts, int n, double* sums, int* err,
                             cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    pm_mla_trace_kernel<<<(n + 127) / 128, 128, 0, st>>>(fg, W, H, starts, n, sums, err);
    return cudaGetLastError();
}

}  // namespace pfd
