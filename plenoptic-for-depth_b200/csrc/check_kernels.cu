// check_kernels.cu -- the consistency pass after PatchMatch, on the device:
//   pm_filter_kernel   MIDisparityFilterCPU::FilterTile (CheckModule/MIDisparityFilter.cpp:423-693)
//   pm_reproj_kernel   ComputeTileReprojectionErrorMap (MIDisparityFilter.cpp:695-842)
//   pm_cycle_kernel    MICycleCheckerCPU::CheckTile (CheckModule/MICycleCheck.cpp:282-725)
//
// The filter invalidates rejected pixels in place and walks the micro-images
// in key order, so a later micro-image reads the already filtered state of
// earlier neighbours (FilterGlobal, :962-986).  The device keeps exactly that
// dependency: micro-image (col, row) runs in wavefront step col + c * row, with
// c chosen on the host so that every neighbour earlier in key order falls in
// an earlier step and every later one in a later step.  Micro-images of one
// step are never neighbours of each other and run in parallel.
//
// Arithmetic is the reference's expressions evaluated as written, one
// rounding per operation (the library is built with -fmad=false), matching the
// CPU oracle (oracle/checks.c).
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <math_constants.h>
#include "check_kernels.h"

namespace pfd {

namespace {

__device__ __forceinline__ float hypot_canon(float x, float y)
{
    const double dx = (double)x, dy = (double)y;
    return (float)sqrt(dx * dx + dy * dy);
}

__device__ __forceinline__ bool bilinear_f32(const float* img, int W, int H, float x, float y, float& v)
{
    if (x < 0 || y < 0 || x > W - 1 || y > H - 1) return false;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = min(x0 + 1, W - 1), y1 = min(y0 + 1, H - 1);
    const float ax = x - (float)x0, ay = y - (float)y0;
    const float v00 = img[y0 * W + x0], v01 = img[y1 * W + x0], v10 = img[y0 * W + x1], v11 = img[y1 * W + x1];
    float s = ((1.0f - ax) * (1.0f - ay)) * v00;
    s = s + ((1.0f - ax) * ay) * v01;
    s = s + (ax * (1.0f - ay)) * v10;
    s = s + (ax * ay) * v11;
    v = s;
    return true;
}

// cv::meanStdDev of a 3x3 window (top-left x0, y0): double sums, row-major.
__device__ __forceinline__ void mean_std_3x3(const float* img, int W, int x0, int y0, float& mean, float& stdv)
{
    double s = 0.0, sq = 0.0;
    for (int y = y0; y < y0 + 3; ++y)
        for (int x = x0; x < x0 + 3; ++x) {
            const double v = (double)img[y * W + x];
            s += v;
            sq += v * v;
        }
    const double scale = 1.0 / 9.0;
    s *= scale;
    double var = sq * scale - s * s;
    if (var < 0.0) var = 0.0;
    mean = (float)s;
    stdv = (float)sqrt(var);
}

__device__ __forceinline__ bool patch_mean_std_centred(const float* img, int W, int H, float fx, float fy, float& m,
                                                       float& s)
{
    const int cx = (int)roundf(fx), cy = (int)roundf(fy);
    if (cx < 1 || cy < 1 || cx >= W - 1 || cy >= H - 1) return false;
    mean_std_3x3(img, W, cx - 1, cy - 1, m, s);
    return isfinite(m) && isfinite(s) && s > 1.0e-3f;
}

// ComputePhotoResidual, MIDisparityFilter.cpp:138-156
__device__ __forceinline__ float photo_residual(const float* ref, const float* nei, int W, int H, float px, float py,
                                               float qx, float qy)
{
    float Ir = 0.0f, In = 0.0f;
    if (!bilinear_f32(ref, W, H, px, py, Ir)) return CUDART_NAN_F;
    if (!bilinear_f32(nei, W, H, qx, qy, In)) return CUDART_NAN_F;
    float mr, sr, mn, sn;
    if (patch_mean_std_centred(ref, W, H, px, py, mr, sr) && patch_mean_std_centred(nei, W, H, qx, qy, mn, sn)) {
        const float Irn = (Ir - mr) / sr;
        const float Inn = (In - mn) / sn;
        return fabsf(Irn - Inn);
    }
    return fabsf(In - Ir);
}

// BilinearDisparity (MIDisparityFilter.cpp:80-118) over a neighbour's state.
__device__ __forceinline__ float bilinear_disp(const float4* plane, int W, int H, float x, float y, float min_valid)
{
    if (x < 0 || y < 0 || x > W - 1 || y > H - 1) return CUDART_NAN_F;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = min(x0 + 1, W - 1), y1 = min(y0 + 1, H - 1);
    const float ax = x - (float)x0, ay = y - (float)y0;
    const float d00 = plane[y0 * W + x0].w, d01 = plane[y1 * W + x0].w;
    const float d10 = plane[y0 * W + x1].w, d11 = plane[y1 * W + x1].w;
    if (!isfinite(d00) || d00 <= min_valid || !isfinite(d01) || d01 <= min_valid ||
        !isfinite(d10) || d10 <= min_valid || !isfinite(d11) || d11 <= min_valid)
        return CUDART_NAN_F;
    float r = ((1.0f - ax) * (1.0f - ay)) * d00;
    r = r + ((1.0f - ax) * ay) * d01;
    r = r + (ax * (1.0f - ay)) * d10;
    r = r + (ax * ay) * d11;
    return r;
}

__device__ __forceinline__ float bilinear_cost(const float* cost, int W, int H, float x, float y)
{
    if (x < 0 || y < 0 || x > W - 1 || y > H - 1) return CUDART_NAN_F;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = min(x0 + 1, W - 1), y1 = min(y0 + 1, H - 1);
    const float ax = x - (float)x0, ay = y - (float)y0;
    const float c00 = cost[y0 * W + x0], c01 = cost[y1 * W + x0], c10 = cost[y0 * W + x1], c11 = cost[y1 * W + x1];
    if (!isfinite(c00) || !isfinite(c01) || !isfinite(c10) || !isfinite(c11)) return CUDART_NAN_F;
    float r = ((1.0f - ax) * (1.0f - ay)) * c00;
    r = r + ((1.0f - ax) * ay) * c01;
    r = r + (ax * (1.0f - ay)) * c10;
    r = r + (ax * ay) * c11;
    return r;
}

struct NbDir { float dx, dy, scale; bool ok; };

__device__ __forceinline__ NbDir neighbour_dir(float2 c0, float2 c1, float unit)
{
    NbDir r{ 0.f, 0.f, 0.f, false };
    const float Bx = c0.x - c1.x, By = c0.y - c1.y;
    const float baseline = hypot_canon(Bx, By);
    if (baseline < 1.0e-6f) return r;
    r.dx = Bx / baseline;
    r.dy = By / baseline;
    r.scale = baseline / unit;
    r.ok = true;
    return r;
}

__device__ __forceinline__ int set_bits(uint32_t mask, int* out, int max_needed)
{
    int n = 0;
    for (int b = 0; mask && n < max_needed; ++b) {
        if (mask & 1u) out[n++] = b;
        mask >>= 1u;
    }
    return n;
}

// Stage 1 of FilterTile for one pixel; returns the reject reason (0 = keep).
// Also used, with geometry only, by the reprojection-error map.
__device__ __forceinline__ bool cost_ok(float c, const FilterCfg& cfg)
{
    if (!cfg.enable_cost_filter) return true;
    return !((!isfinite(c) || c < 0.0f) || (isfinite(c) && c > cfg.max_cost));
}

}  // namespace

// Gray micro-images are read as floats from the 8-bit tiles.
__global__ void pm_filter_kernel(CheckFrame F, FilterCfg cfg, StateDev st, const int* step_views, int n_step,
                                 uint8_t* reason, unsigned long long* stats)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int W = F.W, H = F.H, N = W * H;
    float* ref = (float*)smem;                        // [N]
    float* nei = ref + N;                              // [K][N] neighbour grays
    unsigned char* keep1 = (unsigned char*)(nei + (size_t)F.K * N);
    unsigned char* keepf = keep1 + N;
    __shared__ unsigned long long cnt[8];
    for (int item = blockIdx.x; item < n_step; item += gridDim.x) {
        const int v = step_views[item];
        const int nc = min(F.nb_counts[v], F.K);
        const size_t base = (size_t)v * N;
        if (threadIdx.x < 8) cnt[threadIdx.x] = 0;
        for (int e = threadIdx.x; e < N; e += blockDim.x) ref[e] = (float)F.gray[(size_t)v * F.tile_stride + e];
        for (int e = threadIdx.x; e < nc * N; e += blockDim.x) {
            const int k = e / N, r = e % N;
            const int nv = F.nb_ids[v * F.K + k];
            nei[e] = nv >= 0 ? (float)F.gray[(size_t)nv * F.tile_stride + r] : 0.0f;
        }
        __syncthreads();
        const float2 c0 = F.centers[v];
        for (int idx = threadIdx.x; idx < N; idx += blockDim.x) {
            const int x = idx % W, y = idx / W;
            keep1[idx] = 0;
            uint8_t why = kPrKeep;
            atomicAdd(&cnt[kFsTotal], 1ull);
            const float d = st.plane[base + idx].w;
            if (isfinite(d) && d > cfg.min_valid_disp) {
                atomicAdd(&cnt[kFsValidIn], 1ull);
                const float cost = st.cost[base + idx];
                if (!cost_ok(cost, cfg)) {
                    why = kPrCost;
                } else {
                    int vids[32];
                    int nv;
                    if (cfg.use_selected_views_only) nv = set_bits(st.sel[base + idx], vids, cfg.max_triplet);
                    else { nv = min(nc, cfg.max_triplet); for (int i = 0; i < nv; ++i) vids[i] = i; }
                    if (nv == 0) {
                        why = kPrNoSupport;
                    } else {
                        const float px = (float)x, py = (float)y;
                        int support = 0, good = 0;
                        for (int vi = 0; vi < nv; ++vi) {
                            const int b = vids[vi];
                            if (b < 0 || b >= nc) continue;
                            const int nvid = F.nb_ids[v * F.K + b];
                            if (nvid < 0) continue;
                            const NbDir g = neighbour_dir(c0, F.centers[nvid], F.baseline_unit);
                            if (!g.ok) continue;
                            const float qx = px + (g.dx * d) * g.scale;
                            const float qy = py + (g.dy * d) * g.scale;
                            if (qx < 0 || qy < 0 || qx > W - 1 || qy > H - 1) continue;
                            const size_t nbase = (size_t)nvid * N;
                            const float d_nei = bilinear_disp(st.plane + nbase, W, H, qx, qy, cfg.min_valid_disp);
                            if (!isfinite(d_nei)) continue;
                            if (cfg.enable_cost_filter && !cost_ok(bilinear_cost(st.cost + nbase, W, H, qx, qy), cfg)) continue;
                            ++support;
                            bool pass_geo = true, pass_photo = true;
                            if (cfg.enable_cycle_geo_filter) {
                                const float phx = qx - (g.dx * d_nei) * g.scale;
                                const float phy = qy - (g.dy * d_nei) * g.scale;
                                const float ge = hypot_canon(phx - px, phy - py);
                                pass_geo = isfinite(ge) && ge <= cfg.max_geo_err_px;
                            }
                            if (cfg.enable_cycle_photo_filter) {
                                const float pe = photo_residual(ref, nei + (size_t)b * N, W, H, px, py, qx, qy);
                                pass_photo = isfinite(pe) && pe <= cfg.max_photo_err_u;
                            }
                            if (pass_geo && pass_photo) ++good;
                        }
                        if (support < cfg.min_good_neighbors) why = kPrNoSupport;
                        else if (good < cfg.min_good_neighbors) why = kPrCycle;
                        else keep1[idx] = 1;
                    }
                }
                if (why == kPrCost) atomicAdd(&cnt[kFsCost], 1ull);
                if (why == kPrNoSupport) atomicAdd(&cnt[kFsNoSupport], 1ull);
                if (why == kPrCycle) atomicAdd(&cnt[kFsCycle], 1ull);
            }
            if (reason) reason[base + idx] = why;
        }
        __syncthreads();
        // spike pass (MIDisparityFilter.cpp:644-676): reads before any write
        for (int idx = threadIdx.x; idx < N; idx += blockDim.x) {
            keepf[idx] = keep1[idx];
            if (!cfg.enable_spike_filter || !keep1[idx]) continue;
            const int x = idx % W, y = idx / W;
            float nvals[8];
            int n = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    const int xn = x + dx, yn = y + dy;
                    if (xn < 0 || yn < 0 || xn >= W || yn >= H) continue;
                    const int ni = yn * W + xn;
                    if (!keep1[ni]) continue;
                    const float dv = st.plane[base + ni].w;
                    if (!isfinite(dv) || dv <= cfg.min_valid_disp) continue;
                    nvals[n++] = dv;
                }
            if (n < cfg.spike_min_neighbors) continue;
            for (int a = 1; a < n; ++a) {
                const float t = nvals[a];
                int b = a - 1;
                while (b >= 0 && nvals[b] > t) { nvals[b + 1] = nvals[b]; --b; }
                nvals[b + 1] = t;
            }
            const float med = nvals[n / 2];
            const float cur = st.plane[base + idx].w;
            if (!isfinite(cur)) continue;
            if (fabsf(cur - med) > cfg.spike_abs_diff) {
                keepf[idx] = 0;
                if (reason) reason[base + idx] = kPrSpike;
                atomicAdd(&cnt[kFsSpike], 1ull);
            }
        }
        __syncthreads();
        // InvalidatePixel (MIDisparityFilter.cpp:158-174) for every rejected valid pixel
        for (int idx = threadIdx.x; idx < N; idx += blockDim.x) {
            const float d = st.plane[base + idx].w;
            if (!isfinite(d) || d <= cfg.min_valid_disp) continue;
            if (keepf[idx]) { atomicAdd(&cnt[kFsKept], 1ull); continue; }
            atomicAdd(&cnt[kFsRemoved], 1ull);
            st.plane[base + idx] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
            st.cost[base + idx] = 2.0f;
            st.disp[base + idx] = make_float4(-1.0f, -1.0f, 0.0f, 0.0f);
            if (cfg.clear_selected_views_when_invalid) st.sel[base + idx] = 0u;
        }
        __syncthreads();
        if (threadIdx.x < 8 && stats) atomicAdd(&stats[threadIdx.x], cnt[threadIdx.x]);
        __syncthreads();
    }
}

// ComputeTileReprojectionErrorMap for every pixel of every view (read-only).
__global__ void pm_reproj_kernel(CheckFrame F, FilterCfg cfg, StateDev st, float* err)
{
    const int N = F.W * F.H;
    const size_t total = (size_t)F.V * N;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int v = (int)(t / N), idx = (int)(t % N);
        const int W = F.W, H = F.H, x = idx % W, y = idx / W;
        const int nc = min(F.nb_counts[v], F.K);
        float out = -1.0f;
        const float d = st.plane[t].w;
        if (isfinite(d) && d > cfg.min_valid_disp && cost_ok(st.cost[t], cfg)) {
            int vids[32];
            int nv;
            if (cfg.use_selected_views_only) nv = set_bits(st.sel[t], vids, cfg.max_triplet);
            else { nv = min(nc, cfg.max_triplet); for (int i = 0; i < nv; ++i) vids[i] = i; }
            const float px = (float)x, py = (float)y;
            float ge[32];
            int ng = 0;
            const float2 c0 = F.centers[v];
            for (int vi = 0; vi < nv; ++vi) {
                const int b = vids[vi];
                if (b < 0 || b >= nc) continue;
                const int nvid = F.nb_ids[v * F.K + b];
                if (nvid < 0) continue;
                const NbDir g = neighbour_dir(c0, F.centers[nvid], F.baseline_unit);
                if (!g.ok) continue;
                const float qx = px + (g.dx * d) * g.scale;
                const float qy = py + (g.dy * d) * g.scale;
                if (qx < 0 || qy < 0 || qx > W - 1 || qy > H - 1) continue;
                const size_t nbase = (size_t)nvid * N;
                const float d_nei = bilinear_disp(st.plane + nbase, W, H, qx, qy, cfg.min_valid_disp);
                if (!isfinite(d_nei)) continue;
                if (cfg.enable_cost_filter && !cost_ok(bilinear_cost(st.cost + nbase, W, H, qx, qy), cfg)) continue;
                const float phx = qx - (g.dx * d_nei) * g.scale;
                const float phy = qy - (g.dy * d_nei) * g.scale;
                const float e = hypot_canon(phx - px, phy - py);
                if (isfinite(e)) ge[ng++] = e;
            }
            if (ng >= cfg.min_good_neighbors) {
                for (int a = 1; a < ng; ++a) {
                    const float tv = ge[a];
                    int b = a - 1;
                    while (b >= 0 && ge[b] > tv) { ge[b + 1] = ge[b]; --b; }
                    ge[b + 1] = tv;
                }
                // QuantileFromSorted(v, 0.5), MIDisparityFilter.cpp:36-51
                const float pos = 0.5f * (float)(ng - 1);
                const int lo = (int)floorf(pos), hi = (int)ceilf(pos);
                const float tq = pos - (float)lo;
                out = (lo == hi) ? ge[lo] : ge[lo] * (1.0f - tq) + ge[hi] * tq;
            }
        }
        err[t] = out;
    }
}

namespace {

// cv::BORDER_REFLECT_101 (borderInterpolate)
__device__ __forceinline__ int reflect101(int i, int n)
{
    if (n == 1) return 0;
    while (i < 0 || i >= n) i = i < 0 ? -i : 2 * n - 2 - i;
    return i;
}

// patch_mean_std lambda (MICycleCheck.cpp:327-339): 3x3 window, top-left round(p) - 2
__device__ __forceinline__ bool patch_mean_std_cycle(const float* img, int W, int H, float fx, float fy, float& m,
                                                     float& s)
{
    const int cx = (int)roundf(fx), cy = (int)roundf(fy);
    if (cx < 2 || cy < 2 || cx >= W - 2 || cy >= H - 2) return false;
    mean_std_3x3(img, W, cx - 2, cy - 2, m, s);
    return isfinite(m) && isfinite(s) && s > 1e-3f;
}

// bilinear_disp lambda (MICycleCheck.cpp:306-325): non-finite corners replaced
__device__ __forceinline__ float bilinear_disp_cycle(const float4* plane, int W, int H, float fx, float fy)
{
    if (fx < 0 || fy < 0 || fx > W - 1 || fy > H - 1) return CUDART_NAN_F;
    const int x0 = (int)floorf(fx), y0 = (int)floorf(fy);
    const int x1 = min(x0 + 1, W - 1), y1 = min(y0 + 1, H - 1);
    const float ax = fx - (float)x0, ay = fy - (float)y0;
    float d00 = plane[y0 * W + x0].w, d01 = plane[y1 * W + x0].w;
    float d10 = plane[y0 * W + x1].w, d11 = plane[y1 * W + x1].w;
    if (!isfinite(d00)) d00 = 0.0f;
    if (!isfinite(d01)) d01 = d00;
    if (!isfinite(d10)) d10 = d00;
    if (!isfinite(d11)) d11 = d00;
    float r = ((1.0f - ax) * (1.0f - ay)) * d00;
    r = r + ((1.0f - ax) * ay) * d01;
    r = r + (ax * (1.0f - ay)) * d10;
    r = r + (ax * ay) * d11;
    return r;
}

__device__ __forceinline__ float min_std(float a, float b) { return (b < a) ? b : a; }   // std::min
__device__ __forceinline__ float max_std(float a, float b) { return (a < b) ? b : a; }   // std::max

}  // namespace

// One CTA per micro-image: BuildTextureMaskAndViz on the reference gray, the
// per-pixel cycle errors, then the tile's sums in pixel order (one thread per
// sum, so each double sum keeps the reference's order).
__global__ void pm_cycle_kernel(CheckFrame F, CycleCfg cfg, StateDev st, float* geo_err, float* pho_err,
                                uint8_t* texmask, CycleTileRec* recs, unsigned int* hist)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int W = F.W, H = F.H, N = W * H;
    float* ref = (float*)smem;                          // [N]
    float* nei = ref + N;                               // [K][N]
    float* gavg = nei + (size_t)F.K * N;                // [N] per-pixel mean geometric error
    float* pavg = gavg + N;                             // [N] per-pixel mean photometric error
    uint8_t* flag = (uint8_t*)(pavg + N);               // [N] bit 0 sample, bit 1 textured
    uint8_t* tm = flag + N;                             // [N] texture mask
    __shared__ int comp[4];
    for (int v = blockIdx.x; v < F.V; v += gridDim.x) {
        const int nc = min(F.nb_counts[v], F.K);
        const size_t base = (size_t)v * N;
        if (threadIdx.x < 4) comp[threadIdx.x] = 0;
        for (int e = threadIdx.x; e < N; e += blockDim.x) ref[e] = (float)F.gray[(size_t)v * F.tile_stride + e];
        for (int e = threadIdx.x; e < nc * N; e += blockDim.x) {
            const int k = e / N, r = e % N;
            const int nv = F.nb_ids[v * F.K + k];
            nei[e] = nv >= 0 ? (float)F.gray[(size_t)nv * F.tile_stride + r] : 0.0f;
        }
        __syncthreads();
        // texture mask: Sobel magnitude and 7x7 variance (integer gray, exact sums)
        for (int idx = threadIdx.x; idx < N; idx += blockDim.x) {
            const int x = idx % W, y = idx / W;
            const int xm = reflect101(x - 1, W), xp = reflect101(x + 1, W);
            const int ym = reflect101(y - 1, H), yp = reflect101(y + 1, H);
            const float gx = (ref[ym * W + xp] - ref[ym * W + xm]) + 2.0f * (ref[y * W + xp] - ref[y * W + xm]) +
                             (ref[yp * W + xp] - ref[yp * W + xm]);
            const float gy = (ref[yp * W + xm] - ref[ym * W + xm]) + 2.0f * (ref[yp * W + x] - ref[ym * W + x]) +
                             (ref[yp * W + xp] - ref[ym * W + xp]);
            const float mag = sqrtf(gx * gx + gy * gy);
            double s1 = 0.0, s2 = 0.0;
            for (int dy = -3; dy <= 3; ++dy) {
                const int yy = reflect101(y + dy, H) * W;
                for (int dx = -3; dx <= 3; ++dx) {
                    const float val = ref[yy + reflect101(x + dx, W)];
                    s1 += (double)val;
                    s2 += (double)(val * val);
                }
            }
            const float mean = (float)(s1 * (1.0 / 49.0)), mean2 = (float)(s2 * (1.0 / 49.0));
            const float var = mean2 - mean * mean;
            const bool m1 = mag > cfg.sobel_thresh, m2 = var > cfg.var_thresh;
            tm[idx] = (cfg.use_and ? (m1 && m2) : (m1 || m2)) ? 255 : 0;
        }
        __syncthreads();
        const float2 c0 = F.centers[v];
        for (int idx = threadIdx.x; idx < N; idx += blockDim.x) {
            const int x = idx % W, y = idx / W;
            float gcell = 0.0f, pcell = 0.0f;
            uint8_t fl = 0;
            const float d = st.plane[base + idx].w;
            int vids[32];
            const int nv = isfinite(d) ? set_bits(st.sel[base + idx], vids, cfg.max_triplet) : 0;
            if (nv > 0) {
                const float px = (float)x, py = (float)y;
                float gsum = 0.0f, psum = 0.0f, m_ref, s_ref;
                int cnt = 0, gate = 0, gate_geo = 0, gate_photo = 0;
                const bool ref_mask_ok = patch_mean_std_cycle(ref, W, H, px, py, m_ref, s_ref);
                for (int vi = 0; vi < nv; ++vi) {
                    const int b = vids[vi];
                    if (b < 0 || b >= nc) continue;
                    const int nvid = F.nb_ids[v * F.K + b];
                    if (nvid < 0) continue;                       // no gray image: the sample fails
                    const NbDir g = neighbour_dir(c0, F.centers[nvid], F.baseline_unit);
                    if (!g.ok) continue;
                    const float qx = px + (g.dx * d) * g.scale;
                    const float qy = py + (g.dy * d) * g.scale;
                    if (qx < 0 || qy < 0 || qx > W - 1 || qy > H - 1) continue;
                    const float d_nei = bilinear_disp_cycle(st.plane + (size_t)nvid * N, W, H, qx, qy);
                    const float phx = qx - (g.dx * d_nei) * g.scale;
                    const float phy = qy - (g.dy * d_nei) * g.scale;
                    const float geo_e = hypot_canon(phx - px, phy - py);
                    if (!(geo_e < (float)(W * 2))) continue;
                    const float* nimg = nei + (size_t)b * N;
                    float Ir, In;
                    if (!bilinear_f32(ref, W, H, px, py, Ir)) continue;
                    if (!bilinear_f32(nimg, W, H, qx, qy, In)) continue;
                    float mr, sr, mn, sn, phe;
                    if (patch_mean_std_cycle(ref, W, H, px, py, mr, sr) &&
                        patch_mean_std_cycle(nimg, W, H, qx, qy, mn, sn)) {
                        const float Irn = (Ir - mr) / sr, Inn = (In - mn) / sn;
                        phe = fabsf(Irn - Inn);
                    } else {
                        phe = fabsf(In - Ir);
                    }
                    const float phe_raw = phe;
                    if (isfinite(phe)) phe = min_std(phe, 3.0f);
                    const float geo_used = cfg.clamp_geo ? min_std(geo_e, cfg.geo_u_px) : geo_e;
                    const float phe_used = cfg.clamp_photo ? min_std(phe, cfg.photo_u) : phe;
                    const bool pg = cfg.gate_use_clamped ? (geo_used <= cfg.gate_geo_px) : (geo_e <= cfg.gate_geo_px);
                    const bool pp = cfg.gate_use_clamped ? (phe_used <= cfg.gate_photo_u) : (phe_raw <= cfg.gate_photo_u);
                    gate += (pg && pp);
                    gate_geo += pg;
                    gate_photo += pp;
                    const bool ok = cfg.pixel_gate_enabled ? (pg && pp) : true;
                    if (ok) { gsum = gsum + geo_used; psum = psum + phe_used; ++cnt; }
                    if (cnt > 0) { gcell = max_std(gcell, geo_used); pcell = max_std(pcell, phe_used); }
                }
                if (ref_mask_ok) {
                    atomicAdd(&comp[0], 1);
                    if (gate >= cfg.gate_min_good_neighbors) atomicAdd(&comp[1], 1);
                    if (gate_geo >= cfg.gate_min_good_neighbors) atomicAdd(&comp[2], 1);
                    if (gate_photo >= cfg.gate_min_good_neighbors) atomicAdd(&comp[3], 1);
                }
                if ((!cfg.pixel_gate_enabled && cnt > 0) || (cfg.pixel_gate_enabled && cnt >= cfg.gate_min_good_neighbors)) {
                    gavg[idx] = cnt > 0 ? gsum / (float)cnt : 0.0f;
                    pavg[idx] = cnt > 0 ? psum / (float)cnt : 0.0f;
                    fl = 1 | (tm[idx] ? 2 : 0);
                }
            }
            flag[idx] = fl;
            if (geo_err) geo_err[base + idx] = gcell;
            if (pho_err) pho_err[base + idx] = pcell;
            if (texmask) texmask[base + idx] = tm[idx];
        }
        __syncthreads();
        // tile sums, each by one thread in pixel order
        const int t = threadIdx.x;
        if (t < 8) {
            const bool photo = (t & 2) != 0, sq = (t & 1) != 0, masked_only = (t & 4) != 0;
            const float* a = photo ? pavg : gavg;
            double acc = 0.0;
            for (int i = 0; i < N; ++i) {
                const uint8_t f = flag[i];
                if (!(f & 1) || (masked_only && !(f & 2))) continue;
                acc += sq ? (double)(a[i] * a[i]) : (double)a[i];
            }
            CycleTileRec& r = recs[v];
            switch (t) {
                case 0: r.sum_geo = acc; break;
                case 1: r.sq_geo = acc; break;
                case 2: r.sum_photo = acc; break;
                case 3: r.sq_photo = acc; break;
                case 4: r.sum_geo_m = acc; break;
                case 5: r.sq_geo_m = acc; break;
                case 6: r.sum_photo_m = acc; break;
                default: r.sq_photo_m = acc; break;
            }
        } else if (t == 8) {
            int n = 0, nm = 0;
            float mn = CUDART_INF_F, mx = 0.0f;
            for (int i = 0; i < N; ++i) {
                const uint8_t f = flag[i];
                if (!(f & 1)) continue;
                ++n;
                if (!(f & 2)) continue;
                ++nm;
                const float gv = gavg[i];
                if (!isfinite(gv) || gv < 0.0f) continue;
                int bi = (int)floor((double)gv / 0.5);
                bi = max(0, min(bi, kCycleHistBins - 1));
                if (hist) atomicAdd(&hist[bi], 1u);
                if (gv < mn) mn = gv;
                if (gv > mx) mx = gv;
            }
            recs[v].n = n;
            recs[v].n_masked = nm;
            recs[v].min_geo_m = mn;
            recs[v].max_geo_m = mx;
            recs[v].comp_total = comp[0];
            recs[v].comp_good = comp[1];
            recs[v].comp_good_geo = comp[2];
            recs[v].comp_good_photo = comp[3];
        }
        __syncthreads();
    }
}

int cycle_smem_bytes(const CheckFrame& F)
{
    const int N = F.W * F.H;
    return (3 + F.K) * N * 4 + 2 * N;
}

cudaError_t launch_cycle(const CheckFrame& F, const CycleCfg& cfg, const StateDev& st, float* geo_err, float* pho_err,
                         uint8_t* texmask, CycleTileRec* recs, unsigned int* hist, cudaStream_t s)
{
    if (F.V <= 0) return cudaSuccess;
    const int smem = cycle_smem_bytes(F);
    cudaError_t e = cudaFuncSetAttribute(pm_cycle_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const int threads = F.W * F.H < 256 ? ((F.W * F.H + 31) / 32) * 32 : 256;
    pm_cycle_kernel<<<F.V, threads < 64 ? 64 : threads, smem, s>>>(F, cfg, st, geo_err, pho_err, texmask, recs, hist);
    return cudaGetLastError();
}

int filter_smem_bytes(const CheckFrame& F)
{
    const int N = F.W * F.H;
    return (1 + F.K) * N * 4 + 2 * N;
}

cudaError_t launch_filter_step(const CheckFrame& F, const FilterCfg& cfg, const StateDev& st, const int* step_views,
                               int n_step, uint8_t* reason, unsigned long long* stats, cudaStream_t s)
{
    if (n_step <= 0) return cudaSuccess;
    const int smem = filter_smem_bytes(F);
    const int threads = F.W * F.H < 256 ? ((F.W * F.H + 31) / 32) * 32 : 256;
    cudaError_t e = cudaFuncSetAttribute(pm_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    pm_filter_kernel<<<n_step, threads, smem, s>>>(F, cfg, st, step_views, n_step, reason, stats);
    return cudaGetLastError();
}

cudaError_t launch_reproj(const CheckFrame& F, const FilterCfg& cfg, const StateDev& st, float* err, cudaStream_t s)
{
    const size_t total = (size_t)F.V * F.W * F.H;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    pm_reproj_kernel<<<blocks, 256, 0, s>>>(F, cfg, st, err);
    return cudaGetLastError();
}

}  // namespace pfd
