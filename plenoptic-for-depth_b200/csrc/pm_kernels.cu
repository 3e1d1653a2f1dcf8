// pm_kernels.cu -- sm_100a kernels of the whole-frame micro-image PatchMatch.
//
//   pm_slice_kernel   raw frame -> per-view micro-image tiles (Slice_RawMLAImage,
//                     DepthSolver.cpp:1951-1997)
//   pm_init_kernel    RandomInitializationForFrame (AdaptMIPMFrame.cu:474-518)
//   pm_sweep_kernel   CheckerboardUpdateFrame (AdaptMIPMFrame.cu:520-947)
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

// The g-th pixel (row-major) whose colour (x + y) & 1 equals `colour`.
__device__ __forceinline__ bool nth_pixel(int g, int colour, int W, int H, int& x, int& y)
{
    for (int yy = 0; yy < H; ++yy) {
        const int x0 = (colour ^ yy) & 1;
        const int cnt = (W - x0 + 1) >> 1;
        if (g < cnt) { x = x0 + 2 * g; y = yy; return true; }
        g -= cnt;
    }
    return false;
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
template <bool BLUR, bool COUNT>
__global__ void __launch_bounds__(256) pm_init_kernel(FrameDev F, PmParams P, StateDev out, int* err)
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
    if (act) h = random_plane(g, P.depth_min, P.depth_max);
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
    out.plane[idx] = h;
    out.cost[idx] = mean;
    out.disp[idx] = disp;
    out.sel[idx] = mask;
}

// --------------------------------------------------------------------------
// CheckerboardUpdateFrame
// --------------------------------------------------------------------------
struct Cands {
    int flag[8];
    int pos[8];        // local pixel index of the candidate plane
    int src[8];        // slot whose cost vector this slot copies, or -1
};

// Candidate positions of AdaptMIPMFrame.cu:589-795: per direction the lowest
// prev-cost sample among the scan pattern.
__device__ __forceinline__ void find_candidates(const float* pc, int x, int y, int W, int H, Cands& C)
{
    const int center = y * W + x;
    for (int a = 0; a < 8; ++a) { C.flag[a] = 0; C.pos[a] = center; C.src[a] = -1; }
    auto scan = [&](int start, const int* pts, const bool* ok, int n) {
        float cm = pc[start];
        int cp = start;
        for (int i = 0; i < n; ++i)
            if (ok[i] && pc[pts[i]] < cm) { cm = pc[pts[i]]; cp = pts[i]; }
        return cp;
    };
    if (y > 2) {
        const int s = center - 3 * W; const int pts[1] = { s - W }; const bool ok[1] = { y > 3 };
        C.flag[1] = 1; C.pos[1] = scan(s, pts, ok, 1);
    }
    if (y < H - 3) {
        const int s = center + 3 * W; const int pts[1] = { s + W }; const bool ok[1] = { y < H - 4 };
        C.flag[3] = 1; C.pos[3] = scan(s, pts, ok, 1);
    }
    if (x > 2) {
        const int s = center - 3; const int pts[1] = { s - 1 }; const bool ok[1] = { x > 3 };
        C.flag[5] = 1; C.pos[5] = scan(s, pts, ok, 1);
    }
    if (x < W - 3) {
        const int s = center + 3; const int pts[1] = { s + 1 }; const bool ok[1] = { x < W - 4 };
        C.flag[7] = 1; C.pos[7] = scan(s, pts, ok, 1);
    }
    if (y > 0) {
        const int s = center - W;
        const int pts[4] = { s - W, s - W, s - 2 * W - 1, s - 2 * W + 1 };
        const bool ok[4] = { y > 1 && x > 0, y > 1 && x < W - 1, y > 2 && x > 1, y > 2 && x < W - 2 };
        C.flag[0] = 1; C.pos[0] = scan(s, pts, ok, 4);
    }
    if (y <= 2 && y > 0) { C.flag[1] = 1; C.pos[1] = C.pos[0]; C.src[1] = 0; }
    if (y < H - 1) {
        const int s = center + W;
        const int pts[4] = { s + W, s + W, s + 2 * W - 1, s + 2 * W + 1 };
        const bool ok[4] = { y < H - 2 && x > 0, y < H - 2 && x < W - 1, y < H - 3 && x > 1, y < H - 3 && x < W - 2 };
        C.flag[2] = 1; C.pos[2] = scan(s, pts, ok, 4);
    }
    if (y >= H - 3 && y < H - 1) { C.flag[3] = 1; C.pos[3] = C.pos[2]; C.src[3] = 2; }
    if (x > 0) {
        const int s = center - 1;
        const int pts[4] = { s - 1, s - 1, s - 2 - W, s - 2 + W };
        const bool ok[4] = { x > 1 && y > 0, x > 1 && y < H - 1, x > 2 && y > 1, x > 2 && y < H - 2 };
        C.flag[4] = 1; C.pos[4] = scan(s, pts, ok, 4);
    }
    if (x <= 2 && x > 0) { C.flag[5] = 1; C.pos[5] = C.pos[4]; C.src[5] = 4; }
    if (x < W - 1) {
        const int s = center + 1;
        const int pts[4] = { s + 1, s + 1, s + 2 - W, s + 2 + W };
        const bool ok[4] = { x < W - 2 && y > 0, x < W - 2 && y < H - 1, x < W - 3 && y > 1, x < W - 3 && y < H - 2 };
        C.flag[6] = 1; C.pos[6] = scan(s, pts, ok, 4);
    }
    if (x >= W - 3 && x < W - 1) { C.flag[7] = 1; C.pos[7] = C.pos[6]; C.src[7] = 6; }
}

// Position of the n-th (0-based) set bit of m, or -1.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int n)
{
    for (int i = 0; i < n && m; ++i) m &= m - 1;
    return m ? __ffs(m) - 1 : -1;
}

// One red or black half-sweep as a persistent kernel: the grid holds as many
// CTAs as fit on the device, and CTA b walks the (view, pixel batch) items
// b, b + gridDim.x, ...  Each CTA owns a slice of cost_scratch for the nine
// candidate cost vectors of its pixels, small enough (about 40 MB for the
// whole grid) to stay in L2.
//
// Every lane of a warp reaches each cost evaluation together (lanes without
// a pixel, or whose candidate slot is empty, ride along inactive); per-lane
// logic between evaluations is free to diverge.  Cross-view proposals and
// refinement candidates are walked by a warp-uniform loop in which every lane
// takes its own next hypothesis.
template <bool BLUR, bool COUNT>
__global__ void __launch_bounds__(128, 4) pm_sweep_kernel(FrameDev F, PmParams P, StateDev prev, StateDev next,
                                                          int iter, int phase, int nbatch, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int npb = blockDim.x;
    const int t = threadIdx.x;
    const int W = P.W, H = P.H, K = P.K;
    const SmemPlan L = SmemPlan::make(W, H, K, npb, P.ntap, BLUR, 0, true, P.tile_stride);
    float* cA = P.cost_scratch + (size_t)blockIdx.x * 9 * K * npb + t;     // [slot][k][npb]
#define COSTA(slot, k) cA[((slot) * K + (k)) * npb]
    const int n_items = F.V * nbatch;

    for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int vid = item / nbatch, batch = item % nbatch;
        const int nc = min(F.nb_counts[vid], K);
        const size_t vbase = (size_t)vid * P.ppv;

        int ux = 0, uy = 0, cx = 0, cy = 0;
        const bool has_u = nth_pixel(batch * npb + t, phase, W, H, ux, uy);
        const bool has_c = nth_pixel(batch * npb + t, phase ^ 1, W, H, cx, cy);

        // pixels of the other colour keep their state (AdaptMIPMFrame.cu:552-559)
        if (has_c) {
            const size_t i = vbase + cy * W + cx;
            next.plane[i] = prev.plane[i]; next.cost[i] = prev.cost[i];
            next.disp[i] = prev.disp[i];   next.sel[i] = prev.sel[i];
        }
        if (nc <= 0) {                   // AdaptMIPMFrame.cu:562-570
            if (has_u) {
                const size_t i = vbase + uy * W + ux;
                next.plane[i] = prev.plane[i]; next.cost[i] = prev.cost[i];
                next.disp[i] = prev.disp[i];   next.sel[i] = prev.sel[i];
            }
            continue;
        }

        Tiles T;
        if (!stage_tiles<BLUR>(smem, L, F, P, vid, nc, T, err)) return;
        float* pc = (float*)(smem + L.off_prevc);
        uint32_t* ps = (uint32_t*)(smem + L.off_prevs);
        for (int e = t; e < P.ppv; e += npb) { pc[e] = prev.cost[vbase + e]; ps[e] = prev.sel[vbase + e]; }
        __syncthreads();

        const int x = ux, y = uy;
        const int center = y * W + x;
        const size_t idx = vbase + center;

        // ---- propagation candidates and the current plane ----------------
        Cands C;
        if (has_u) find_candidates(pc, x, y, W, H, C);
        else for (int a = 0; a < 8; ++a) { C.flag[a] = 0; C.pos[a] = 0; C.src[a] = -1; }
        for (int s = 0; s < 8; ++s) {
            const bool act = has_u && C.flag[s] && C.src[s] < 0;
            const float4 h = act ? prev.plane[vbase + C.pos[s]] : make_float4(0.f, 0.f, 1.f, 0.f);
            cost_vector<BLUR, COUNT>(T, P, x, y, act, h, nc, &COSTA(s, 0), npb);
        }
        for (int s = 0; s < 8; ++s) {
            if (!has_u || !C.flag[s] || C.src[s] < 0) continue;
            for (int k = 0; k < nc; ++k) COSTA(s, k) = COSTA(C.src[s], k);
        }
        float4 best_plane = has_u ? prev.plane[idx] : make_float4(0.f, 0.f, 1.f, 0.f);
        cost_vector<BLUR, COUNT>(T, P, x, y, has_u, best_plane, nc, &COSTA(8, 0), npb);

        // ---- view-selection priors and sampling (AdaptMIPMFrame.cu:797-875)
        DrawStream g;
        g.init(P.seed, (uint32_t)(1 + 2 * iter + phase), (uint32_t)idx);
        uint32_t tsel = 0;
        uint64_t vw_lo = 0, vw_hi = 0;       // 4-bit view weights, views 0-15 and 16-31
        float best_cost = kCostMax;
        int best_min = -1;
        if (has_u) {
            const int dpos[4] = { (y > 0) ? center - W : -1, (y < H - 1) ? center + W : -1,
                                  (x > 0) ? center - 1 : -1, (x < W - 1) ? center + 1 : -1 };
            const float thr = __fmul_rn(0.8f, pfd_expf(__fdiv_rn((float)(iter * iter), -90.0f)));
            const float p_default = pfd_expf(__fdiv_rn(__fmul_rn(thr, thr), -0.32f));
            float cdf[kMaxNb];
            float psum = 0.0f;
            for (int i = 0; i < nc; ++i) {
                float prior = 0.0f;
                for (int ii = 0; ii < 4; ++ii) {
                    if (dpos[ii] < 0 || !C.flag[2 * ii]) continue;
                    prior = __fadd_rn(prior, ((ps[dpos[ii]] >> i) & 1u) ? 0.9f : 0.1f);
                }
                float count = 0.0f, tmpw = 0.0f;
                int count_false = 0;
                for (int j = 0; j < 8; ++j) {
                    if (!C.flag[j]) continue;
                    const float c = COSTA(j, i);
                    if (c < thr) { tmpw = __fadd_rn(tmpw, pfd_expf(__fdiv_rn(__fmul_rn(c, c), -0.18f))); count = __fadd_rn(count, 1.0f); }
                    if (c > 1.2f) count_false++;
                }
                float pr = 0.0f;
                if (count > 2.0f && count_false < 3) pr = __fdiv_rn(tmpw, count);
                else if (count_false < 3) pr = p_default;
                pr = __fmul_rn(pr, prior);
                cdf[i] = pr;
                psum = __fadd_rn(psum, pr);
            }
            {   // TransformPDFToCDF (CudaUtil.cu:491-507)
                const float inv = __fdiv_rn(1.0f, psum);
                float cum = 0.0f;
                for (int i = 0; i < nc; ++i) { cum = __fmaf_rn(cdf[i], inv, cum); cdf[i] = cum; }
            }
            for (int sample = 0; sample < 15; ++sample) {
                const float rp = __fsub_rn(g.uniform(), 1.1920928955078125e-07f);
                for (int id = 0; id < nc; ++id)
                    if (cdf[id] > rp) {
                        if (id < 16) vw_lo += 1ull << (id * 4); else vw_hi += 1ull << ((id - 16) * 4);
                        break;
                    }
            }
            for (int i = 0; i < nc; ++i)
                if (((i < 16 ? vw_lo >> (i * 4) : vw_hi >> ((i - 16) * 4)) & 15ull) != 0) tsel |= 1u << i;
            if (tsel == 0)
                for (int i = 0; i < nc; ++i) {
                    if (i < 16) vw_lo |= 1ull << (i * 4); else vw_hi |= 1ull << ((i - 16) * 4);
                    tsel |= 1u << i;
                }
        }
#define VW(k) ((float)(((k) < 16 ? vw_lo >> ((k) * 4) : vw_hi >> (((k) - 16) * 4)) & 15ull))
        if (has_u) {
            // weighted costs: current plane, then the 8 candidates
            {
                WeightedCost wc;
                for (int k = 0; k < nc; ++k) wc.add(k, COSTA(8, k), VW(k));
                best_cost = wc.result();
                best_min = wc.min_idx;
            }
            for (int s = 0; s < 8; ++s) {
                if (!C.flag[s]) continue;
                WeightedCost wc;
                for (int k = 0; k < nc; ++k) wc.add(k, COSTA(s, k), VW(k));
                const float c = wc.result();
                if (c < best_cost) { best_cost = c; best_plane = prev.plane[vbase + C.pos[s]]; best_min = wc.min_idx; }
            }
        }
        float* scratch = &COSTA(0, 0);                // candidate costs are dead from here on

        // ---- cross-view proposals (AdaptMIPMFrame.cu:907-936) ------------
        const int nsel = __popc(tsel);
        const int nmax = __reduce_max_sync(kFullMask, nsel);
        for (int n = 0; n < nmax; ++n) {
            const int k = (n < nsel) ? nth_set_bit(tsel, n) : -1;
            bool act = false;
            float4 proxy = make_float4(0.f, 0.f, 1.f, 0.f);
            if (k >= 0) {
                const int nvid = F.nb_ids[vid * K + k];
                if (nvid >= 0) {
                    const NbGeo& gk = T.geo[k];
                    const float dcur = to_disparity(x, y, disparity_plane(x, y, best_plane));
                    const float2 qf = geo_anchor(gk, x, y, dcur);
                    const float fqx = floorf(__fadd_rn(qf.x, 0.5f)), fqy = floorf(__fadd_rn(qf.y, 0.5f));
                    if (fqx >= 0.0f && fqx < (float)W && fqy >= 0.0f && fqy < (float)H) {
                        const int qx = (int)fqx, qy = (int)fqy;
                        const float4 hn = prev.plane[(size_t)nvid * P.ppv + qy * W + qx];
                        const float3 dpn = disparity_plane(qx, qy, hn);
                        float denom = __fmaf_rn(dpn.y, gk.by, __fmaf_rn(dpn.x, gk.bx, 1.0f));
                        denom = safe_denom(denom);
                        proxy = encode_plane(x, y, __fdiv_rn(dpn.x, denom), __fdiv_rn(dpn.y, denom), __fdiv_rn(dpn.z, denom));
                        act = true;
                    }
                }
            }
            cost_vector<BLUR, COUNT>(T, P, x, y, act, proxy, nc, scratch, npb);
            if (act) {
                WeightedCost wc;
                for (int kk = 0; kk < nc; ++kk) wc.add(kk, scratch[kk * npb], VW(kk));
                const float c = wc.result();
                if (c < best_cost) { best_cost = c; best_plane = proxy; best_min = wc.min_idx; }
            }
        }

        // ---- refinement (PlaneHypothesisRefinement_Frame, :400-471) -----
        float4 cand[5];
        if (has_u) {
            const float depth_now = best_plane.w;
            (void)g.uniform();                       // depth_rand: drawn, never used
            const float4 rn = random_normal(g);
            const float4 pn = perturbed_normal(x, y, best_plane, g, P.pert_pi);
            const float dmin_p = __fmul_rn(__fsub_rn(1.0f, 0.02f), depth_now);
            const float dmax_p = __fmul_rn(__fadd_rn(1.0f, 0.02f), depth_now);
            const float depth_perturbed = __fmaf_rn(g.uniform(), __fsub_rn(dmax_p, dmin_p), dmin_p);
            cand[0] = random_plane(g, P.depth_min, P.depth_max);
            cand[1] = rn;
            cand[2] = pn;
            cand[3] = best_plane;
            cand[4] = best_plane;
            cand[4].w = depth_perturbed;
            for (int i = 1; i < 5; ++i) cand[i].w = to_disparity(x, y, disparity_plane(x, y, cand[i]));
        } else {
            for (int i = 0; i < 5; ++i) cand[i] = make_float4(0.f, 0.f, 1.f, 0.f);
        }
        for (int i = 0; i < 5; ++i) {
            cost_vector<BLUR, COUNT>(T, P, x, y, has_u, cand[i], nc, scratch, npb);
            if (has_u) {
                WeightedCost wc;
                for (int kk = 0; kk < nc; ++kk) wc.add(kk, scratch[kk * npb], VW(kk));
                const float c = wc.result();
                if (c < best_cost) { best_cost = c; best_plane = cand[i]; best_min = wc.min_idx; }
            }
        }
#undef VW
        if (has_u) {
            float4 best_disp = make_float4(0.f, 0.f, 0.f, 0.f);
            if (best_min >= 0)
                best_disp = geo_disp(T.geo[best_min], x, y, to_disparity(x, y, disparity_plane(x, y, best_plane)));
            next.plane[idx] = best_plane;
            next.cost[idx] = best_cost;
            next.disp[idx] = best_disp;
            next.sel[idx] = tsel;
        }
        __syncthreads();                             // shared memory is restaged for the next item
    }
#undef COSTA
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
int sweep_smem_bytes(const PmParams& P, int npb, bool blur)
{
    return SmemPlan::make(P.W, P.H, P.K, npb, P.ntap, blur, 0, true, P.tile_stride).total;
}

constexpr int kSweepThreads = 128;

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

cudaError_t launch_init(const FrameDev& F, const PmParams& P, const StateDev& out, int* err, cudaStream_t st)
{
    const bool blur = F.blur != nullptr;
    const int npb = P.ppv < 256 ? ((P.ppv + 31) / 32) * 32 : 256;
    const int smem = SmemPlan::make(P.W, P.H, P.K, npb, P.ntap, blur, 1, false, P.tile_stride).total;
    dim3 grid(F.V, (P.ppv + npb - 1) / npb);
    FrameDev f = F; PmParams p = P; StateDev o = out; int* e = err;
    void* args[] = { &f, &p, &o, &e };
    if (P.tap_counter)
        return blur ? launch(pm_init_kernel<true, true>, grid, npb, smem, st, args)
                    : launch(pm_init_kernel<false, true>, grid, npb, smem, st, args);
    return blur ? launch(pm_init_kernel<true, false>, grid, npb, smem, st, args)
                : launch(pm_init_kernel<false, false>, grid, npb, smem, st, args);
}

size_t sweep_scratch_bytes(const PmParams& P, int n_sms, int ctas_per_sm)
{
    return (size_t)n_sms * (size_t)ctas_per_sm * 9u * (size_t)P.K * kSweepThreads * sizeof(float);
}

cudaError_t sweep_grid(const PmParams& P, bool blur, int* n_ctas)
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int smem = sweep_smem_bytes(P, kSweepThreads, blur);
    const void* k = blur ? (const void*)pm_sweep_kernel<true, false> : (const void*)pm_sweep_kernel<false, false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kSweepThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *n_ctas = sms * per_sm;
    return cudaSuccess;
}

cudaError_t launch_sweep(const FrameDev& F, const PmParams& P, const StateDev& prev, const StateDev& next,
                         int iter, int phase, int n_ctas, int* err, cudaStream_t st)
{
    const bool blur = F.blur != nullptr;
    const int updated = (P.ppv + 1) / 2;
    const int npb = kSweepThreads;
    const int nbatch = (updated + npb - 1) / npb;
    const int smem = sweep_smem_bytes(P, npb, blur);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    const int grid = std::min(n_ctas, F.V * nbatch);
    FrameDev f = F; PmParams p = P; StateDev a = prev, b = next; int it = iter, ph = phase, nb = nbatch; int* e = err;
    void* args[] = { &f, &p, &a, &b, &it, &ph, &nb, &e };
    if (P.tap_counter)
        return blur ? launch(pm_sweep_kernel<true, true>, grid, npb, smem, st, args)
                    : launch(pm_sweep_kernel<false, true>, grid, npb, smem, st, args);
    return blur ? launch(pm_sweep_kernel<true, false>, grid, npb, smem, st, args)
                : launch(pm_sweep_kernel<false, false>, grid, npb, smem, st, args);
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
