// pm_kernels.cu -- sm_100a kernels of the whole-frame micro-image PatchMatch.
//
//   pm_slice_kernel   raw frame -> per-view micro-image tiles (Slice_RawMLAImage,
//                     DepthSolver.cpp:1951-1997)
//   pm_init_kernel    RandomInitializationForFrame (AdaptMIPMFrame.cu:474-518)
//   pm_ncc_kernel     per-hypothesis cost vectors (ComputeMultiViewCostVector_Frame)
//
// One CTA owns one reference micro-image (and a batch of its pixels).  Its own
// window and its neighbours' windows are brought into shared memory by the
// bulk-copy engine (cp.async.bulk + mbarrier) and expanded there into
// bilinear-ready row pairs; every NCC tap then reads shared memory only.  Each
// thread owns one pixel and evaluates its hypotheses against the neighbours in
// chunks of KCH, sharing the reference-side work of a tap across the chunk.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_device.cuh"
#include "pm_kernels.h"

namespace pfd {

// --------------------------------------------------------------------------
// Shared-memory plan, identical on host and device.
// --------------------------------------------------------------------------
__host__ __device__ inline int align16(int v) { return (v + 15) & ~15; }

// Row stride of the neighbour row pairs: even (conflict-free 8-byte loads for
// two rows of checkerboard pixels) and at least W + 1.
__host__ __device__ inline int pair_stride(int W) { return (W + 2) & ~1; }

struct SmemPlan {
    int off_Q, off_QB, off_R, off_RB, off_geo, off_ok, off_as, off_ac;
    int off_prevc, off_prevs, off_cost, off_stage, off_bar, total;
    int q_bytes;

    __host__ __device__ static SmemPlan make(int W, int H, int K, int npb, int ntap, bool blur,
                                             int cost_slots, bool sweep, int tile_stride)
    {
        SmemPlan p;
        int o = 0;
        p.q_bytes = (H + 2) * pair_stride(W) * 8;
        p.off_Q = o;    o += align16(K * p.q_bytes);
        p.off_QB = o;   o += blur ? align16(K * p.q_bytes) : 0;
        p.off_R = o;    o += align16(H * W * 4);
        p.off_RB = o;   o += blur ? align16(H * W * 4) : 0;
        p.off_geo = o;  o += align16(K * (int)sizeof(NbGeo));
        p.off_ok = o;   o += align16(K * 4);
        p.off_as = o;   o += align16(ntap * ntap * 4);
        p.off_ac = o;   o += 256 * 4;
        p.off_prevc = o; o += sweep ? align16(W * H * 4) : 0;
        p.off_prevs = o; o += sweep ? align16(W * H * 4) : 0;
        p.off_bar = o;  o += 16;
        p.off_cost = o;
        const int cost_bytes = align16(cost_slots * K * npb * 4);
        const int stage_bytes = (1 + K) * tile_stride * (blur ? 2 : 1);
        p.off_stage = o;                         // staging is dead before costs are written
        o += (cost_bytes > stage_bytes ? cost_bytes : stage_bytes);
        p.total = o;
        return p;
    }
};

// --------------------------------------------------------------------------
// mbarrier + bulk copy (TMA bulk engine) helpers
// --------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done != 0;
}
// Bounded wait: gives up after ~2^22 polls (seconds), records the failure and
// returns false.  A bulk copy from valid global memory completes in
// microseconds, so this only fires on a broken launch.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err)
{
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(128);
    }
    if (err) atomicOr(err, PFD_DEVERR_TMA_TIMEOUT);
    return false;
}

// --------------------------------------------------------------------------
// CTA prologue: stage the reference window and its neighbours' windows.
// --------------------------------------------------------------------------
template <bool BLUR>
__device__ __forceinline__ bool stage_tiles(unsigned char* smem, const SmemPlan& L, const FrameDev& F,
                                            const PmParams& P, int vid, int nc, Tiles& T, int* err)
{
    const int W = P.W, H = P.H, K = P.K;
    uint8_t* stage = (uint8_t*)(smem + L.off_stage);
    uint64_t* bar = (uint64_t*)(smem + L.off_bar);
    const int nt = 1 + nc;                 // reference + neighbours, in that order
    const int ts = P.tile_stride;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_arrive_expect_tx(bar, (uint32_t)(nt * ts * (BLUR ? 2 : 1)));
        for (int i = 0; i < nt; ++i) {
            const int v = (i == 0) ? vid : F.nb_ids[vid * K + i - 1];
            const int vv = v < 0 ? vid : v;      // invalid ids are masked below; copy something valid
            bulk_copy_g2s(stage + i * ts, F.gray + (size_t)vv * ts, (uint32_t)ts, bar);
            if (BLUR) bulk_copy_g2s(stage + (nt + i) * ts, F.blur + (size_t)vv * ts, (uint32_t)ts, bar);
        }
    }
    // per-neighbour geometry and the weight tables do not depend on the copies
    NbGeo* geo = (NbGeo*)(smem + L.off_geo);
    int* okk = (int*)(smem + L.off_ok);
    float* a_s = (float*)(smem + L.off_as);
    float* a_c = (float*)(smem + L.off_ac);
    const float2 c0 = F.centers[vid];
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int v = (k < nc) ? F.nb_ids[vid * K + k] : -1;
        okk[k] = (v >= 0);
        geo[k] = make_geo(c0, F.centers[v >= 0 ? v : vid], P);
    }
    const int ntap = P.ntap;
    for (int t = threadIdx.x; t < ntap * ntap; t += blockDim.x) {
        const float fi = (float)(-P.radius + (t / ntap) * P.inc);
        const float fj = (float)(-P.radius + (t % ntap) * P.inc);
        const float sd = __fsqrt_rn(__fmaf_rn(fj, fj, __fmul_rn(fi, fi)));
        a_s[t] = __fdiv_rn(-sd, P.ss2);
    }
    for (int c = threadIdx.x; c < 256; c += blockDim.x) a_c[c] = __fdiv_rn((float)c, P.cc2);
    __syncthreads();                         // barrier init visible before anyone polls it
    const bool ok = mbar_wait_bounded(bar, 0, err);
    if (__syncthreads_or(!ok)) return false;

    float* R = (float*)(smem + L.off_R);
    for (int e = threadIdx.x; e < W * H; e += blockDim.x) R[e] = (float)stage[e];
    if (BLUR) {
        float* RB = (float*)(smem + L.off_RB);
        for (int e = threadIdx.x; e < W * H; e += blockDim.x) RB[e] = (float)stage[nt * ts + e];
    }
    const int S = pair_stride(W);
    const int qs = (H + 2) * S;
    int2* Q = (int2*)(smem + L.off_Q);
    int2* QB = (int2*)(smem + L.off_QB);
    for (int e = threadIdx.x; e < nc * qs; e += blockDim.x) {
        const int k = e / qs, r = e % qs;
        const int y = r / S, x = r % S;
        const int yy = min(y, H - 1);
        const int x0 = min(x, W - 1), x1 = min(x + 1, W - 1);
        const uint8_t* src = stage + (1 + k) * ts + yy * W;
        Q[e] = make_int2((int)src[x0], (int)src[x1] - (int)src[x0]);
        if (BLUR) {
            const uint8_t* sb = stage + (nt + 1 + k) * ts + yy * W;
            QB[e] = make_int2((int)sb[x0], (int)sb[x1] - (int)sb[x0]);
        }
    }
    __syncthreads();
    T.R = R;
    T.RB = BLUR ? (const float*)(smem + L.off_RB) : nullptr;
    T.q_addr = smem_u32(smem + L.off_Q);
    T.qb_addr = BLUR ? smem_u32(smem + L.off_QB) : 0u;
    T.q_stride = S;
    T.q_bytes = L.q_bytes;
    T.geo = geo;
    T.nb_ok = okk;
    T.a_s = a_s;
    T.a_c = a_c;
    return true;
}

// --------------------------------------------------------------------------
// Slice: raw frame -> tiles.  Window origin trunc(c - (m-1)/2) is computed on
// the host (DepthSolver.cpp:1894-1895 and the cv::Rect conversion at :1977).
// --------------------------------------------------------------------------
__global__ void pm_slice_kernel(const uint8_t* raw, int raw_pitch, const int2* origin, int V, int W, int H,
                                int tile_stride, uint8_t* tiles)
{
    const int v = blockIdx.x;
    if (v >= V) return;
    const int2 o = origin[v];
    uint8_t* dst = tiles + (size_t)v * tile_stride;
    for (int e = threadIdx.x; e < tile_stride; e += blockDim.x) {
        uint8_t val = 0;
        if (e < W * H) val = raw[(size_t)(o.y + e / W) * raw_pitch + o.x + e % W];
        dst[e] = val;
    }
}

// --------------------------------------------------------------------------
// RandomInitializationForFrame.  One thread per pixel; every lane of a warp
// takes part in the warp-collective cost evaluation.
// --------------------------------------------------------------------------
// With refit set, the pixel keeps its plane from out.plane and only its cost,
// selected views and disp are recomputed: PostRefineMetadataFrame of the ACMM
// matcher (AdaptMIPMFrameACMM.cu:903-929), which is the same top-k evaluation.
template <bool BLUR, bool COUNT>
__global__ void __launch_bounds__(256) pm_init_kernel(FrameDev F, PmParams P, StateDev out, int* err, int refit)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int vid = blockIdx.x;
    const int npb = blockDim.x;
    const int t = threadIdx.x;
    const int nc = min(F.nb_counts[vid], P.K);
    const SmemPlan L = SmemPlan::make(P.W, P.H, P.K, npb, P.ntap, BLUR, 1, false, P.tile_stride);
    Tiles T;
    if (!stage_tiles<BLUR>(smem, L, F, P, vid, nc, T, err)) return;

    const int e = blockIdx.y * npb + t;
    const bool act = e < P.ppv;
    const int x = act ? e % P.W : 0, y = act ? e / P.W : 0;
    const size_t idx = (size_t)vid * P.ppv + (act ? e : 0);
    DrawStream g;
    g.init(P.seed, 0u, (uint32_t)idx);
    float4 h = make_float4(0.f, 0.f, 1.f, 0.f);
    if (act) h = refit ? out.plane[idx] : random_plane(g, P.depth_min, P.depth_max);
    float* cs = (float*)(smem + L.off_cost) + t;           // [k][npb]
    cost_vector<BLUR, COUNT>(T, P, x, y, act, h, nc, cs, npb);
    if (!act) return;

    // ComputeSelectedViewsTopK_Frame (AdaptMIPMFrame.cu:227-282)
    int best_idx = -1, valid = 0;
    for (int i = 0; i < nc; ++i) {
        const float c = cs[i * npb];
        if (c < 2.0f) {
            ++valid;
            if (best_idx < 0 || c < cs[best_idx * npb]) best_idx = i;
        }
    }
    float mean = 2.0f;
    uint32_t mask = 0;
    if (valid > 0) {
        const int kk = min(valid, P.top_k);
        float tmp[kMaxNb];
        for (int i = 0; i < kMaxNb; ++i) tmp[i] = (i < nc) ? cs[i * npb] : 2.0f;
        for (int i = 0; i < kk; ++i)
            for (int j = i + 1; j < nc; ++j)
                if (tmp[j] < tmp[i]) { const float s = tmp[i]; tmp[i] = tmp[j]; tmp[j] = s; }
        float m = 0.0f;
        for (int i = 0; i < kk; ++i) m = __fadd_rn(m, tmp[i]);
        mean = __fdiv_rn(m, (float)kk);
        const float thr = tmp[kk - 1];
        for (int i = 0; i < nc && i < 32; ++i)
            if (cs[i * npb] <= thr) mask |= (1u << i);
    }
    float4 disp = make_float4(0.f, 0.f, 0.f, 0.f);
    if (best_idx >= 0) disp = geo_disp(T.geo[best_idx], x, y, to_disparity(x, y, disparity_plane(x, y, h)));
    if (!refit) out.plane[idx] = h;
    out.cost[idx] = mean;
    out.disp[idx] = disp;
    out.sel[idx] = mask;
    if (P.cvec)
        for (int i = 0; i < nc; ++i) P.cvec[idx * P.K + i] = cs[i * npb];
}

// --------------------------------------------------------------------------
// Per-hypothesis cost vectors.  Segments group hypotheses of one view.
// --------------------------------------------------------------------------
template <bool BLUR, bool COUNT>
__global__ void __launch_bounds__(256) pm_ncc_kernel(FrameDev F, PmParams P, const int* seg_vid, const int* seg_start,
                                                     const int* seg_len, const int* hyp_pxy, const float4* hyp_plane,
                                                     const int* hyp_out, float* costs, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int s = blockIdx.x;
    const int vid = seg_vid[s];
    const int nc = min(F.nb_counts[vid], P.K);
    const SmemPlan L = SmemPlan::make(P.W, P.H, P.K, blockDim.x, P.ntap, BLUR, 1, false, P.tile_stride);
    Tiles T;
    if (!stage_tiles<BLUR>(smem, L, F, P, vid, nc, T, err)) return;
    const bool act = (int)threadIdx.x < seg_len[s];
    const int h = seg_start[s] + (act ? threadIdx.x : 0);
    const int px = act ? hyp_pxy[2 * h] : 0, py = act ? hyp_pxy[2 * h + 1] : 0;
    float* cs = (float*)(smem + L.off_cost) + threadIdx.x;
    cost_vector<BLUR, COUNT>(T, P, px, py, act, act ? hyp_plane[h] : make_float4(0.f, 0.f, 1.f, 0.f), nc, cs, blockDim.x);
    if (!act) return;
    float* out = costs + (size_t)hyp_out[h] * P.K;
    for (int k = 0; k < P.K; ++k) out[k] = (k < nc) ? cs[k * blockDim.x] : 2.0f;
}

// --------------------------------------------------------------------------
// Host launchers
// --------------------------------------------------------------------------
template <class Kern>
static cudaError_t launch(Kern k, dim3 grid, dim3 block, int smem, cudaStream_t st, void** args)
{
    cudaError_t e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernel((const void*)k, grid, block, args, (size_t)smem, st);
}

cudaError_t launch_slice(const uint8_t* raw, int raw_pitch, const int2* origin, int V, int W, int H, int tile_stride,
                         uint8_t* tiles, cudaStream_t st)
{
    if (V <= 0) return cudaSuccess;
    pm_slice_kernel<<<V, 128, 0, st>>>(raw, raw_pitch, origin, V, W, H, tile_stride, tiles);
    return cudaGetLastError();
}

cudaError_t launch_init(const FrameDev& F, const PmParams& P, const StateDev& out, int* err, cudaStream_t st,
                        bool refit)
{
    const bool blur = F.blur != nullptr;
    const int npb = P.ppv < 256 ? ((P.ppv + 31) / 32) * 32 : 256;
    const int smem = SmemPlan::make(P.W, P.H, P.K, npb, P.ntap, blur, 1, false, P.tile_stride).total;
    dim3 grid(F.V, (P.ppv + npb - 1) / npb);
    FrameDev f = F; PmParams p = P; StateDev o = out; int* e = err; int r = refit ? 1 : 0;
    void* args[] = { &f, &p, &o, &e, &r };
    if (P.tap_counter)
        return blur ? launch(pm_init_kernel<true, true>, grid, npb, smem, st, args)
                    : launch(pm_init_kernel<false, true>, grid, npb, smem, st, args);
    return blur ? launch(pm_init_kernel<true, false>, grid, npb, smem, st, args)
                : launch(pm_init_kernel<false, false>, grid, npb, smem, st, args);
}

cudaError_t launch_ncc(const FrameDev& F, const PmParams& P, int nseg, int npb, const int* seg_vid, const int* seg_start,
                       const int* seg_len, const int* hyp_pxy, const float4* hyp_plane, const int* hyp_out,
                       float* costs, int* err, cudaStream_t st)
{
    if (nseg <= 0) return cudaSuccess;
    const bool blur = F.blur != nullptr;
    const int smem = SmemPlan::make(P.W, P.H, P.K, npb, P.ntap, blur, 1, false, P.tile_stride).total;
    FrameDev f = F; PmParams p = P;
    void* args[] = { &f, &p, (void*)&seg_vid, (void*)&seg_start, (void*)&seg_len, (void*)&hyp_pxy,
                     (void*)&hyp_plane, (void*)&hyp_out, &costs, &err };
    return blur ? launch(pm_ncc_kernel<true, false>, nseg, npb, smem, st, args)
                : launch(pm_ncc_kernel<false, false>, nseg, npb, smem, st, args);
}

}  // namespace pfd
