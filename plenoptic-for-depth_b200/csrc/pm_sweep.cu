// pm_sweep.cu -- CheckerboardUpdateFrame (MIStereo/AdaptMIPMFrame.cu:520-947)
// with one warp per updated pixel.
//
// A CTA stages one micro-image and its neighbours at a time; its warps take the
// updated pixels of that micro-image one by one.  For a pixel, every cost
// evaluation the reference makes (the 8 propagation candidates and the
// current plane, the cross-view proposals, the 5 refinement candidates) is a
// set of (hypothesis, neighbour) NCCs; the warp lays them across its lanes,
// one NCC per lane, and walks the pixel's patch window (patch intersected
// with the micro-image, the same for every lane) tap by tap.  The
// reference-side values of a tap (bilateral weight w, w * r, r and the blur
// term) are computed once per pixel into a per-warp table and read as a
// broadcast.  Each lane accumulates its NCC's six moments in the reference's
// tap order (x offset outer, y offset inner); a tap whose source sample
// leaves the neighbour window is skipped, as in the reference.
//
// Cross-view proposals depend on the best plane so far (AdaptMIPMFrame.cu:
// 907-936), and the refinement candidates on the best plane after them
// (:400-471).  Both are built speculatively from the best plane after
// propagation and evaluated together, then walked in order; a proposal whose
// neighbour-window sample position changed because an earlier one won is
// rebuilt and evaluated again, and so are the refinement candidates that
// follow the best plane, so the result is the sequential one.  A refinement
// candidate bit-identical to the best plane has its cost and is not evaluated.
//
// Neighbour samples come from the texture unit: the frame's micro-images are
// layered float textures with the reference's filter settings, and a tap is
// one tex2DLayered fetch, the reference's own tex2D.  The other form (TEX
// false, used by the tap-counting calibration) stages the neighbours in shared
// memory as 32-bit quads, entry (iy, ix) packing the four texels of a bilinear
// footprint, T(iy,ix), T(iy,ix+1), T(iy+1,ix), T(iy+1,ix+1), indices clamped
// to the window, and blends them as the texture unit does (measured, and equal
// to the fetches bit for bit).
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>
#include "pm_device.cuh"
#include "pm_kernels.h"

namespace pfd {

namespace {

// Launch shapes: (warps per CTA, CTAs per SM the registers are sized for).
// Shape 0 is the default; the others are the autotuner's alternatives
// (pfd_set_autotune), which trade resident CTAs for warps per CTA and
// registers per thread as the frame's shared-memory plan allows.
template <int S> struct ShapeOf;
template <> struct ShapeOf<0> { static constexpr int warps = 7, min_ctas = 4; };
template <> struct ShapeOf<1> { static constexpr int warps = 8, min_ctas = 3; };
template <> struct ShapeOf<2> { static constexpr int warps = 4, min_ctas = 6; };
template <> struct ShapeOf<3> { static constexpr int warps = 10, min_ctas = 2; };
constexpr int kShapeWarps[kSweepShapes] = { ShapeOf<0>::warps, ShapeOf<1>::warps, ShapeOf<2>::warps, ShapeOf<3>::warps };
constexpr int kShapeCtas[kSweepShapes] = { ShapeOf<0>::min_ctas, ShapeOf<1>::min_ctas, ShapeOf<2>::min_ctas,
                                           ShapeOf<3>::min_ctas };

struct Quad {
    const float* R;          // [H][W] reference texels
    const float* RB;         // [H][W] reference blur or nullptr
    uint32_t q_addr;         // shared address of neighbour quads [K][H+1][W+1] (shared-memory fetches)
    uint32_t qb_addr;        // same for blur
    int qs;                  // W + 1
    int q_bytes;             // (H + 1) * (W + 1) * 4
    const NbGeo* geo;        // [K]
    const int* nb_ok;        // [K]
    const float* a_s;        // [ntap * ntap]
    const float* a_c;        // [256]
    const cudaTextureObject_t* txh;    // [K] neighbour k's gray texture (texture fetches)
    const cudaTextureObject_t* txbh;   // [K] its blur texture
    const int* txl;                    // [K] its layer
};

// Per-warp scratch.  The tap table and the hypotheses, read on every tap, are
// in shared memory; the cost vectors and their bookkeeping, written once per
// NCC, are in the warp's slice of global scratch (P.cost_scratch), where they
// stay in L1/L2 and leave shared memory to more resident warps.
struct WarpBlock {
    float4* tab;             // [tab_n] (w, w * r, r, r_blur / 255) of the current pixel's window (shared)
    float4* plane;           // [maxh] hypotheses (shared)
    float4* dp;              // [maxh] disparity plane (x, y, z) and disparity at the pixel (w) (shared)
    float* cost;             // [maxh][K] (global)
    uint16_t* pair;          // [maxh * K] compacted (hypothesis, neighbour) indices (global)
    float* wres;             // [maxh] weighted cost (global)
    int* wmin;               // [maxh] index of the lowest cost (global)
    int* aux;                // [maxh] proposal sample position, or -1 (global)
};

// Hypotheses one evaluation can hold: 9 propagation slots, or every selected
// view's proposal, the 5 refinement candidates and one rebuilt proposal.
__host__ __device__ inline int sweep_maxh(int K) { return K + 6 > 9 ? K + 6 : 9; }
// 4-byte words of global scratch per warp: costs, 16-bit pair indices, wres/wmin/aux.
__host__ __device__ inline int sweep_warp_words(int K)
{
    const int mh = sweep_maxh(K);
    return ((mh * K + (mh * K + 1) / 2 + 3 * mh) + 31) & ~31;
}

struct Plan {
    int off_Q, off_QB, off_R, off_RB, off_geo, off_ok, off_as, off_ac, off_pc, off_ps, off_stage, off_bar, off_ctl;
    int off_txh, off_txbh, off_txl;
    int off_warp, warp_bytes, tab_n, maxh;
    int total;

    __host__ __device__ static int a16(int v) { return (v + 15) & ~15; }
    // tex: neighbours are fetched from textures (no quads; only the reference tile is staged)
    __host__ __device__ static Plan make(int W, int H, int K, int ntap, bool blur, int tile_stride, int warps, bool tex)
    {
        Plan p;
        int o = 0;
        // the staging barrier and the control words first: at the same offsets for
        // every frame, so one barrier serves a launch over several frames
        p.off_bar = o;   o += 16;
        p.off_ctl = o;   o += 16;
        const int qb = tex ? 0 : (H + 1) * (W + 1) * 4;
        p.off_Q = o;     o += a16(K * qb);
        p.off_QB = o;    o += blur ? a16(K * qb) : 0;
        p.off_txh = o;   o += tex ? a16(K * 8) : 0;
        p.off_txbh = o;  o += (tex && blur) ? a16(K * 8) : 0;
        p.off_txl = o;   o += tex ? a16(K * 4) : 0;
        p.off_R = o;     o += a16(W * H * 4);
        p.off_RB = o;    o += blur ? a16(W * H * 4) : 0;
        p.off_geo = o;   o += a16(K * (int)sizeof(NbGeo));
        p.off_ok = o;    o += a16(K * 4);
        p.off_as = o;    o += a16(ntap * ntap * 4);
        p.off_ac = o;    o += 256 * 4;
        p.off_pc = o;    o += a16(W * H * 4);
        p.off_ps = o;    o += a16(W * H * 4);
        p.tab_n = (ntap < W ? ntap : W) * (ntap < H ? ntap : H);
        p.maxh = sweep_maxh(K);
        p.warp_bytes = a16(p.tab_n * 16) + a16(2 * p.maxh * 16);
        // the staging buffer shares the warps' area: it is filled (by bulk copies)
        // and read only between views, while no warp holds a pixel
        p.off_warp = o;
        p.off_stage = o;
        const int stage_bytes = a16((tex ? 1 : 1 + K) * tile_stride * (blur ? 2 : 1));
        o += (warps * p.warp_bytes > stage_bytes) ? warps * p.warp_bytes : stage_bytes;
        p.total = o;
        return p;
    }
    // stride: floats of global scratch per warp; a launch over several frames uses
    // the largest frame's, so CTAs on different frames never share a region
    __device__ WarpBlock warp_block(unsigned char* smem, float* gscratch, int w, int warps, int K, int stride) const
    {
        unsigned char* b = smem + off_warp + w * warp_bytes;
        WarpBlock S;
        S.tab = (float4*)b;                  b += a16(tab_n * 16);
        S.plane = (float4*)b;
        S.dp = S.plane + maxh;
        float* g = gscratch + ((size_t)blockIdx.x * warps + w) * (size_t)stride;
        S.cost = g;
        S.pair = (uint16_t*)(g + maxh * K);
        S.wres = g + maxh * K + (maxh * K + 1) / 2;
        S.wmin = (int*)(S.wres + maxh);
        S.aux = S.wmin + maxh;
        return S;
    }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float4 lds_f4(uint32_t addr)
{
    float4 v;
    asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
    return v;
}

__device__ __forceinline__ uint32_t lds_u32(uint32_t addr)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

// Linear-filter fetch of the measured texture unit (see Tiles in pm_device.cuh)
// from a quad entry: 256 s = 256 T00 + a (T10 - T00) + b (T01 - T00) + w11 (T11 - T01 - T10 + T00)
// with w11 = (a b + 128) >> 8, regrouped per texel as
// 256 s = T00 w00 + T10 w10 + T01 w01 + T11 w11, w10 = a - w11, w01 = b - w11,
// w00 = 256 - w10 - b: all four weights lie in [0, 256], so two 16-bit pairs of
// weights against the quad's four bytes make the sum with two dp2a, exactly.
struct QuadWeights {
    uint32_t lo;             // w00 | w10 << 16, against T00, T10 (the quad's low bytes)
    uint32_t hi;             // w01 | w11 << 16, against T01, T11
};

// hi = w01 + 65536 w11 = b + 65535 w11, and lo + hi = 256 + 65535 a (w00 + w01 =
// 256 - a, w10 + w11 = a), so lo = 256 + 65535 a - hi: no weight is negative, so
// no half borrows from the other.
__device__ __forceinline__ QuadWeights quad_weights(int tbx, int tby)
{
    const uint32_t a = (uint32_t)tbx & 0xFFu, b = (uint32_t)tby & 0xFFu;
    const uint32_t w11 = (a * b + 128u) >> 8;
    QuadWeights q;
    q.hi = w11 * 65535u + b;
    q.lo = a * 65535u + 256u - q.hi;
    return q;
}

__device__ __forceinline__ float quad_blend(const QuadWeights& w, uint32_t q)
{
    const uint32_t s256 = __dp2a_lo(w.lo, q, __dp2a_hi(w.hi, q, 0u));
    return __fsub_rn(__uint_as_float(s256 | 0x47000000u), 32768.0f);
}

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
// Bounded wait (about 2^22 polls): records PFD_DEVERR_TMA_TIMEOUT and gives up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err)
{
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(128);
    }
    if (err) atomicOr(err, PFD_DEVERR_TMA_TIMEOUT);
    return false;
}

// Stages micro-image vid and its neighbours: bulk copies of the 8-bit tiles,
// then the reference as floats and the neighbours as quads.  The mbarrier is
// reused with alternating parity, one phase per staged view.
template <bool BLUR, bool TEX>
__device__ bool stage_view(unsigned char* smem, const Plan& L, const FrameDev& F, const PmParams& P, int vid, int nc,
                           uint32_t parity, int* err, Quad& T)
{
    const int W = P.W, H = P.H, K = P.K, ts = P.tile_stride;
    uint8_t* stage = (uint8_t*)(smem + L.off_stage);
    uint64_t* bar = (uint64_t*)(smem + L.off_bar);
    const int nt = TEX ? 1 : 1 + nc;
    if (threadIdx.x == 0) {
        // the warps' writes to the shared area before the last barrier, ordered
        // before the bulk copies that overwrite it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(bar, (uint32_t)(nt * ts * (BLUR ? 2 : 1)));
        for (int i = 0; i < nt; ++i) {
            const int v = (i == 0) ? vid : F.nb_ids[vid * K + i - 1];
            const int vv = (v < 0 || v >= F.V) ? vid : v;
            bulk_copy_g2s(stage + i * ts, F.gray + (size_t)vv * ts, (uint32_t)ts, bar);
            if (BLUR) bulk_copy_g2s(stage + (nt + i) * ts, F.blur + (size_t)vv * ts, (uint32_t)ts, bar);
        }
    }
    NbGeo* geo = (NbGeo*)(smem + L.off_geo);
    int* okk = (int*)(smem + L.off_ok);
    cudaTextureObject_t* txh = (cudaTextureObject_t*)(smem + L.off_txh);
    cudaTextureObject_t* txbh = (cudaTextureObject_t*)(smem + L.off_txbh);
    int* txl = (int*)(smem + L.off_txl);
    const float2 c0 = F.centers[vid];
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        int v = (k < nc) ? F.nb_ids[vid * K + k] : -1;
        if (v >= F.V) { atomicOr(err, PFD_DEVERR_SWEEP_CHECK); v = -1; }
        okk[k] = (v >= 0);
        geo[k] = make_geo(c0, F.centers[v >= 0 ? v : vid], P);
        if (TEX) {
            const int vv = v >= 0 ? v : vid;
            txh[k] = F.tex[vv / F.tex_layers];
            if (BLUR) txbh[k] = F.tex_blur[vv / F.tex_layers];
            txl[k] = vv % F.tex_layers;
        }
    }
    const bool ok = mbar_wait_bounded(bar, parity, err);
    if (__syncthreads_or(!ok)) return false;
    float* R = (float*)(smem + L.off_R);
    for (int e = threadIdx.x; e < W * H; e += blockDim.x) R[e] = (float)stage[e];
    if (BLUR) {
        float* RB = (float*)(smem + L.off_RB);
        for (int e = threadIdx.x; e < W * H; e += blockDim.x) RB[e] = (float)stage[nt * ts + e];
    }
    const int qs = W + 1, qn = (H + 1) * qs;
    uint32_t* Q = (uint32_t*)(smem + L.off_Q);
    uint32_t* QB = (uint32_t*)(smem + L.off_QB);
    for (int e = threadIdx.x; e < (TEX ? 0 : nc * qn); e += blockDim.x) {
        const int k = e / qn, r = e % qn;
        const int iy = r / qs, ix = r % qs;
        const int y0 = min(iy, H - 1), y1 = min(iy + 1, H - 1);
        const int x0 = min(ix, W - 1), x1 = min(ix + 1, W - 1);
        const uint8_t* s = stage + (1 + k) * ts;
        Q[e] = (uint32_t)s[y0 * W + x0] | ((uint32_t)s[y0 * W + x1] << 8) | ((uint32_t)s[y1 * W + x0] << 16) |
               ((uint32_t)s[y1 * W + x1] << 24);
        if (BLUR) {
            const uint8_t* sb = stage + (nt + 1 + k) * ts;
            QB[e] = (uint32_t)sb[y0 * W + x0] | ((uint32_t)sb[y0 * W + x1] << 8) |
                    ((uint32_t)sb[y1 * W + x0] << 16) | ((uint32_t)sb[y1 * W + x1] << 24);
        }
    }
    T.R = R;
    T.RB = BLUR ? (const float*)(smem + L.off_RB) : nullptr;
    T.q_addr = smem_u32(Q);
    T.qb_addr = BLUR ? smem_u32(QB) : 0u;
    T.qs = qs;
    T.q_bytes = qn * 4;
    T.geo = geo;
    T.nb_ok = okk;
    T.a_s = (const float*)(smem + L.off_as);
    T.a_c = (const float*)(smem + L.off_ac);
    T.txh = txh;
    T.txbh = txbh;
    T.txl = txl;
    return true;
}

// The pixel's patch window: the patch's taps (x offset i, y offset j, step inc)
// that fall inside the micro-image, as a rectangle of nX x nY taps.
struct PixWin {
    int x0, y0, nX, nY;      // first tap position and tap counts
    int ii0, jj0;            // offset index of the first tap ((x0 - px + r) / inc)
};

__device__ __forceinline__ PixWin pixel_window(const PmParams& P, int px, int py)
{
    PixWin w;
    const int r = P.radius, inc = P.inc;
    const int sx = max(0, (r - px + inc - 1) / inc), sy = max(0, (r - py + inc - 1) / inc);
    w.ii0 = sx;
    w.jj0 = sy;
    w.x0 = px - r + sx * inc;
    w.y0 = py - r + sy * inc;
    const int ex = min(P.ntap - 1, (P.W - 1 - px + r) / inc), ey = min(P.ntap - 1, (P.H - 1 - py + r) / inc);
    w.nX = max(0, ex - sx + 1);
    w.nY = max(0, ey - sy + 1);
    return w;
}

// Reference-side table of the pixel: (w, w r, r, r_blur / 255) per tap, x outer.
template <bool BLUR>
__device__ __forceinline__ void build_table(const Quad& T, const PmParams& P, const PixWin& pw, int px, int py,
                                            float4* tab, int lane)
{
    const int W = P.W, inc = P.inc;
    const float rc = T.R[py * W + px];
    const float sh = P.shifted ? rc : 0.0f;      // shifted moments: texels minus the centre texel (exact)
    const int n = pw.nX * pw.nY;
    for (int t = lane; t < n; t += 32) {
        const int ix = t / pw.nY, iy = t - ix * pw.nY;
        const int X = pw.x0 + ix * inc, Y = pw.y0 + iy * inc;
        const float rv = T.R[Y * W + X];
        const float cd = fabsf(__fsub_rn(rv, rc));
        const int cdi = __float_as_int(__fadd_rn(cd, 8388608.0f)) & 0xFF;
        const int ti = (pw.ii0 + ix) * P.ntap + (pw.jj0 + iy);
        const float w = pfd_expf_nonpos(__fsub_rn(T.a_s[ti], T.a_c[cdi]));
        const float rb = BLUR ? __fdiv_rn(T.RB[Y * W + X], 255.0f) : 0.0f;
        const float rvs = __fsub_rn(rv, sh);
        tab[t] = make_float4(w, __fmul_rn(w, rvs), rvs, rb);
    }
}

// One lane's NCC (ComputeBilateralNCC_Frame, AdaptMIPMFrame.cu:73-179) of the
// pixel under plane dp against neighbour k.  Every lane of the warp walks the
// same taps; a lane skips the taps it does not keep.  The loop's invariants
// (window bounds wb / hb as float bits, quad row stride, tap step) arrive as
// values, not as fields of the caller's structures (see eval_hyps).
template <bool BLUR, bool COUNT, bool SHIFT>
__device__ __forceinline__ float ncc_lane(const Quad& T, const PmParams& P, const float4* tab, const PixWin pw,
                                          float3 dp, int k, bool active, float sh, unsigned& ntaps, uint32_t wb,
                                          uint32_t hb, uint32_t q_stride, float finc)
{
    const NbGeo& g = T.geo[k];
    const float stx = g.stx, sty = g.sty;
    const uint32_t fold = 0x4B0000u * (q_stride + 1u) * 4u;
    const uint32_t base = T.q_addr + (uint32_t)(k * T.q_bytes) - fold;
    const uint32_t bbase = BLUR ? T.qb_addr + (uint32_t)(k * T.q_bytes) - fold : 0u;
    const uint32_t qs = q_stride;
    const uint32_t tab_s = smem_u32(tab);
    float sr = 0.f, srr = 0.f, ss = 0.f, sss = 0.f, srs = 0.f, sw = 0.f, bsx = 0.f, bsy = 0.f;
    float fxr = (float)pw.x0;
    int t = 0;
    for (int ix = 0; ix < pw.nX; ++ix, fxr = __fadd_rn(fxr, finc)) {
        const float axr = __fmul_rn(dp.x, fxr);
        float fyr = (float)pw.y0;
        // two taps per iteration, the table read through its shared-window address
#pragma unroll 2
        for (int iy = 0; iy < pw.nY; ++iy, ++t, fyr = __fadd_rn(fyr, finc)) {
            const float4 e = lds_f4(tab_s + (uint32_t)t * 16u);
            const float d = __fadd_rn(__fmaf_rn(dp.y, fyr, axr), dp.z);
            const float sx = __fmaf_rn(stx, d, fxr);
            const float sy = __fmaf_rn(sty, d, fyr);
            const bool v = active && (__float_as_uint(sx) < wb) && (__float_as_uint(sy) < hb);
            if (COUNT) ntaps += v ? 1u : 0u;
            if (v) {                         // a skipped tap leaves the sums as they are
                const int tbx = tex_coord_bits(sx), tby = tex_coord_bits(sy);
                const uint32_t rel = (((uint32_t)(tby >> 8) * qs + (uint32_t)(tbx >> 8)) << 2);
                const QuadWeights qw = quad_weights(tbx, tby);
                float s = quad_blend(qw, lds_u32(base + rel));
                if (SHIFT) s = __fsub_rn(s, sh);
                const float wv = e.x, wrv = e.y, rv = e.z;
                const float ws = __fmul_rn(wv, s);
                sr = __fmaf_rn(wv, rv, sr);
                srr = __fmaf_rn(wrv, rv, srr);
                ss = __fmaf_rn(wv, s, ss);
                sss = __fmaf_rn(ws, s, sss);
                srs = __fmaf_rn(wrv, s, srs);
                sw = __fadd_rn(sw, wv);
                if (BLUR) {
                    const float sb = quad_blend(qw, lds_u32(bbase + rel));
                    bsx = __fadd_rn(bsx, e.w);
                    bsy = __fadd_rn(bsy, __fdiv_rn(sb, 255.0f));
                }
            }
        }
    }
    float c = kCostMax;
    if (sw > 1e-6f) {
        const float inv = __fdiv_rn(1.0f, sw);
        const float m_r = __fmul_rn(sr, inv), m_rr = __fmul_rn(srr, inv);
        const float m_s = __fmul_rn(ss, inv), m_ss = __fmul_rn(sss, inv);
        const float m_rs = __fmul_rn(srs, inv);
        const float var_r = __fmaf_rn(-m_r, m_r, m_rr);
        const float var_s = __fmaf_rn(-m_s, m_s, m_ss);
        if (!(var_r < 1e-5f || var_s < 1e-5f)) {
            const float cov = __fmaf_rn(-m_r, m_s, m_rs);
            const float vv = __fsqrt_rn(__fmul_rn(var_r, var_s));
            c = clamp_cost(__fsub_rn(1.0f, __fdiv_rn(cov, vv)));
        }
    }
    if (BLUR) {
        const float tb = __fsub_rn(bsx, bsy);
        const float bw = pfd_expf(__fmul_rn(__fmul_rn(-0.007368f, tb), tb));
        c = clamp_cost(__fmaf_rn(P.blur_gain, __fsub_rn(1.0f, bw), c));
    }
    return c;
}

// ncc_lane with the neighbour samples fetched by the texture unit, as the
// reference's tex2D(images[id], x + 0.5, y + 0.5) fetches them.  A lane fetches
// only the taps inside the neighbour window (the fetch is predicated); a tap
// outside it adds +0 to each sum, which leaves the sum as it is (a sum starts
// at +0 and never becomes -0), so the sums are the ones of the skipped taps
// without a branch around the accumulation.
template <bool BLUR, bool COUNT, bool SHIFT>
__device__ __forceinline__ float ncc_lane_tex(const Quad& T, const PmParams& P, const float4* tab, const PixWin pw,
                                              float3 dp, int k, bool active, float sh, unsigned& ntaps, uint32_t wb,
                                              uint32_t hb, float finc)
{
    const NbGeo& g = T.geo[k];
    const float stx = g.stx, sty = g.sty;
    const cudaTextureObject_t tx = T.txh[k];
    const cudaTextureObject_t txb = BLUR ? T.txbh[k] : 0;
    const int layer = T.txl[k];
    float sr = 0.f, srr = 0.f, ss = 0.f, sss = 0.f, srs = 0.f, sw = 0.f, bsx = 0.f, bsy = 0.f;
    float fxr = (float)pw.x0;
    int t = 0;
    for (int ix = 0; ix < pw.nX; ++ix, fxr = __fadd_rn(fxr, finc)) {
        const float axr = __fmul_rn(dp.x, fxr);
        float fyr = (float)pw.y0;
#pragma unroll 4
        for (int iy = 0; iy < pw.nY; ++iy, ++t, fyr = __fadd_rn(fyr, finc)) {
            const float4 e = tab[t];
            const float d = __fadd_rn(__fmaf_rn(dp.y, fyr, axr), dp.z);
            const float sx = __fmaf_rn(stx, d, fxr);
            const float sy = __fmaf_rn(sty, d, fyr);
            const bool v = active && (__float_as_uint(sx) < wb) && (__float_as_uint(sy) < hb);
            if (COUNT) ntaps += v ? 1u : 0u;
            const float cx = __fadd_rn(sx, 0.5f), cy = __fadd_rn(sy, 0.5f);
            float s = 0.0f;
            if (v) s = tex2DLayered<float>(tx, cx, cy, layer);      // no request for a skipped tap
            if (SHIFT) s = v ? __fsub_rn(s, sh) : 0.0f;
            const float wv = v ? e.x : 0.0f, wrv = v ? e.y : 0.0f;
            const float ws = __fmul_rn(wv, s);
            sr = __fmaf_rn(wv, e.z, sr);
            srr = __fmaf_rn(wrv, e.z, srr);
            ss = __fmaf_rn(wv, s, ss);
            sss = __fmaf_rn(ws, s, sss);
            srs = __fmaf_rn(wrv, s, srs);
            sw = __fadd_rn(sw, wv);
            if (BLUR) {
                float fb = 0.0f;
                if (v) fb = tex2DLayered<float>(txb, cx, cy, layer);
                bsx = __fadd_rn(bsx, v ? e.w : 0.0f);
                bsy = __fadd_rn(bsy, __fdiv_rn(fb, 255.0f));       // 0 / 255 = +0 for a skipped tap
            }
        }
    }
    float c = kCostMax;
    if (sw > 1e-6f) {
        const float inv = __fdiv_rn(1.0f, sw);
        const float m_r = __fmul_rn(sr, inv), m_rr = __fmul_rn(srr, inv);
        const float m_s = __fmul_rn(ss, inv), m_ss = __fmul_rn(sss, inv);
        const float m_rs = __fmul_rn(srs, inv);
        const float var_r = __fmaf_rn(-m_r, m_r, m_rr);
        const float var_s = __fmaf_rn(-m_s, m_s, m_ss);
        if (!(var_r < 1e-5f || var_s < 1e-5f)) {
            const float cov = __fmaf_rn(-m_r, m_s, m_rs);
            const float vv = __fsqrt_rn(__fmul_rn(var_r, var_s));
            c = clamp_cost(__fsub_rn(1.0f, __fdiv_rn(cov, vv)));
        }
    }
    if (BLUR) {
        const float tb = __fsub_rn(bsx, bsy);
        const float bw = pfd_expf(__fmul_rn(__fmul_rn(-0.007368f, tb), tb));
        c = clamp_cost(__fmaf_rn(P.blur_gain, __fsub_rn(1.0f, bw), c));
    }
    return c;
}

// Cost vectors (ComputeMultiViewCostVector_Frame, AdaptMIPMFrame.cu:181-225) of
// hypotheses S.plane[0..nh) at (px, py), except those whose bit is set in
// skip: S.cost[h * K + k] for the neighbours k < nc whose bit is set in vmask
// (the other entries are left as they are).  A neighbour whose anchor leaves
// the window gets 2 without evaluation.
//
// Not inlined (its seven call sites would overflow the instruction cache), so
// what its tap loop reads on every tap arrives by value: the window, its bounds
// (wb, hb: (float)W and (float)H as bits), the quad row stride, the tap step and
// the tap table.  Read through references into the caller's frame they were
// reloaded from local memory on every tap (2.0e9 local loads in one half-sweep
// of a 2048x1536 frame, 3.2e8 with the values passed; 8% of the sweep's time).
template <bool BLUR, bool COUNT, bool SHIFT, bool TEX>
__device__ __noinline__ void eval_hyps(const Quad& T, const PmParams& P, const WarpBlock& S, const PixWin pw,
                                       uint32_t wb, uint32_t hb, uint32_t q_stride, float finc, const float4* tab,
                                       int px, int py, int nh, int nc, int lane, uint64_t skip, uint32_t vmask)
{
    const int K = P.K;
    for (int h = lane; h < nh; h += 32) {
        const float3 dp = disparity_plane(px, py, S.plane[h]);
        S.dp[h] = make_float4(dp.x, dp.y, dp.z, to_disparity(px, py, dp));
    }
    __syncwarp();
    const int total = nh * nc;
    int np = 0;
    for (int n0 = 0; n0 < total; n0 += 32) {
        const int n = n0 + lane;
        bool need = false;
        const int hn = n / nc;
        if (n < total && !((skip >> hn) & 1ull) && ((vmask >> (n - hn * nc)) & 1u)) {
            const int h = hn, k = n - h * nc;
            if (T.nb_ok[k]) {
                const float2 a = geo_anchor(T.geo[k], px, py, S.dp[h].w);
                need = (__float_as_uint(a.x) < P.W_bits) && (__float_as_uint(a.y) < P.H_bits);
            }
            if (!need) S.cost[h * K + k] = kCostMax;
        }
        const unsigned m = __ballot_sync(kFullMask, need);
        if (need) S.pair[np + __popc(m & ((1u << lane) - 1u))] = (uint16_t)n;
        np += __popc(m);
    }
    __syncwarp();
    unsigned ntaps = 0;
    const float sh = SHIFT ? T.R[py * P.W + px] : 0.0f;
    for (int p0 = 0; p0 < np; p0 += 32) {
        const bool act = p0 + lane < np;
        const int n = act ? S.pair[p0 + lane] : 0;
        const int h = n / nc, k = n - h * nc;
        const float4 d = S.dp[h];
        const float3 dp = make_float3(d.x, d.y, d.z);
        const float c = TEX ? ncc_lane_tex<BLUR, COUNT, SHIFT>(T, P, tab, pw, dp, k, act, sh, ntaps, wb, hb, finc)
                            : ncc_lane<BLUR, COUNT, SHIFT>(T, P, tab, pw, dp, k, act, sh, ntaps, wb, hb, q_stride, finc);
        if (act) S.cost[h * K + k] = c;
    }
    if (COUNT) {
        const unsigned tot = __reduce_add_sync(kFullMask, ntaps);
        if (lane == 0 && tot) atomicAdd(P.tap_counter, (unsigned long long)tot);
    }
    __syncwarp();
}

// ComputeWeightedCost_Frame (AdaptMIPMFrame.cu:284-317) of hypotheses [0, nh),
// one lane per hypothesis; view weights packed 4 bits per view.  Only the
// views in vmask are read: the weighted cost is exact whenever vmask holds
// every view of non-zero weight, the lowest-cost index covers vmask's views.
__device__ __noinline__ void weigh_hyps(const WarpBlock& S, int K, int nh, int nc, uint64_t vw_lo, uint64_t vw_hi,
                                        int lane, uint32_t vmask)
{
    for (int h = lane; h < nh; h += 32) {
        WeightedCost wc;
        for (int k = 0; k < nc; ++k) {
            if (!((vmask >> k) & 1u)) continue;
            const float w = (float)((k < 16 ? vw_lo >> (k * 4) : vw_hi >> ((k - 16) * 4)) & 15ull);
            wc.add(k, S.cost[h * K + k], w);
        }
        S.wres[h] = wc.result();
        S.wmin[h] = wc.min_idx;
    }
    __syncwarp();
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

__device__ __forceinline__ int nth_set_bit(uint32_t m, int n)
{
    for (int i = 0; i < n && m; ++i) m &= m - 1;
    return m ? __ffs(m) - 1 : -1;
}

struct Cands {
    int flag[8];
    int pos[8];
    int src[8];
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

// BuildCrossViewPlaneProposal (AdaptMIPMFrame.cu:350-398): the sample position
// q (local index) of pixel (x, y) under `cur` in neighbour k, or -1.  This and
// proposal_plane are called from three places each and kept out of line: less
// code between the NCC passes (1.5% of the half-sweep's time, measured).
__device__ __noinline__ int proposal_pos(const NbGeo& gk, int x, int y, int W, int H, float4 cur)
{
    const float dcur = to_disparity(x, y, disparity_plane(x, y, cur));
    const float2 qf = geo_anchor(gk, x, y, dcur);
    const float fqx = floorf(__fadd_rn(qf.x, 0.5f)), fqy = floorf(__fadd_rn(qf.y, 0.5f));
    if (!(fqx >= 0.0f && fqx < (float)W && fqy >= 0.0f && fqy < (float)H)) return -1;
    return (int)fqy * W + (int)fqx;
}

__device__ __noinline__ float4 proposal_plane(const NbGeo& gk, const float4* nb_plane, int q, int x, int y, int W)
{
    const int qx = q % W, qy = q / W;
    const float4 hn = nb_plane[q];
    const float3 dpn = disparity_plane(qx, qy, hn);
    float denom = __fmaf_rn(dpn.y, gk.by, __fmaf_rn(dpn.x, gk.bx, 1.0f));
    denom = safe_denom(denom);
    return encode_plane(x, y, __fdiv_rn(dpn.x, denom), __fdiv_rn(dpn.y, denom), __fdiv_rn(dpn.z, denom));
}

// The five candidates of PlaneHypothesisRefinement_Frame (AdaptMIPMFrame.cu:
// 400-471) for the best plane `best`, from the draws already taken (c0: the
// random plane, rn: the random normal, u1-u3: the perturbation, u4: the depth
// perturbation).
__device__ __noinline__ void refine_candidates(int x, int y, float4 best, float4 c0, float4 rn, float u1, float u2,
                                               float u3, float u4, float pert, float4 (&cand)[5])
{
    const float depth_now = best.w;
    const float4 pn = perturbed_normal_u(x, y, best, u1, u2, u3, pert);
    const float dmin_p = __fmul_rn(__fsub_rn(1.0f, 0.02f), depth_now);
    const float dmax_p = __fmul_rn(__fadd_rn(1.0f, 0.02f), depth_now);
    const float depth_perturbed = __fmaf_rn(u4, __fsub_rn(dmax_p, dmin_p), dmin_p);
    cand[0] = c0;
    cand[1] = rn;
    cand[2] = pn;
    cand[3] = best;
    cand[4] = best;
    cand[4].w = depth_perturbed;
    for (int i = 1; i < 5; ++i) cand[i].w = to_disparity(x, y, disparity_plane(x, y, cand[i]));
}

}  // namespace

// One half-sweep of one frame by this CTA: it takes the frame's micro-images
// from P.view_queue until none is left.  parity: the staging barrier's phase,
// carried across frames.  Returns false when a staging wait gave up.
template <bool BLUR, bool COUNT, bool SHIFT, bool TEX, int WARPS>
__device__ __forceinline__ bool sweep_frame(unsigned char* smem, const FrameDev& F, const PmParams& P,
                                            const StateDev& prev, const StateDev& next, int iter, int phase, int* err,
                                            uint32_t& parity)
{
    const int W = P.W, H = P.H, K = P.K;
    const Plan L = Plan::make(W, H, K, P.ntap, BLUR, P.tile_stride, WARPS, TEX);
    {
        // the frame's shared-memory plan and its warps' scratch must fit what the
        // launch has (checked once per frame; the decision is the same in every thread)
        uint32_t dyn;
        asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        const bool fits = L.total <= (int)dyn && P.view_queue != nullptr && P.cost_scratch != nullptr &&
                          (!TEX || (F.tex != nullptr && F.tex_layers > 0 && (!BLUR || F.tex_blur != nullptr))) &&
                          P.scratch_stride >= sweep_warp_words(K) &&
                          (size_t)gridDim.x * WARPS * (size_t)P.scratch_stride <= P.scratch_floats;
        if (!fits) {
            if (threadIdx.x == 0) atomicOr(err, PFD_DEVERR_SWEEP_CHECK);
            return false;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const WarpBlock S = L.warp_block(smem, P.cost_scratch, warp, WARPS, K, P.scratch_stride);
    float* pc = (float*)(smem + L.off_pc);
    uint32_t* ps = (uint32_t*)(smem + L.off_ps);
    int* ctl = (int*)(smem + L.off_ctl);
    const int n_upd = (P.ppv + (phase == 0 ? 1 : 0)) / 2;      // pixels with (x + y) & 1 == phase
    const uint32_t sweep_id = (uint32_t)(1 + 2 * iter + phase);

    // per-launch tables and the staging barrier
    {
        float* a_s = (float*)(smem + L.off_as);
        float* a_c = (float*)(smem + L.off_ac);
        for (int t = threadIdx.x; t < P.ntap * P.ntap; t += blockDim.x) {
            const float fi = (float)(-P.radius + (t / P.ntap) * P.inc);
            const float fj = (float)(-P.radius + (t % P.ntap) * P.inc);
            const float sd = __fsqrt_rn(__fmaf_rn(fj, fj, __fmul_rn(fi, fi)));
            a_s[t] = __fdiv_rn(-sd, P.ss2);
        }
        for (int c = threadIdx.x; c < 256; c += blockDim.x) a_c[c] = __fdiv_rn((float)c, P.cc2);
        __syncthreads();
    }

    // the CTAs take micro-images one at a time from a shared counter, so a CTA that
    // drew cheap ones takes more (their cost varies with the neighbour count and the
    // candidates); which CTA updates a micro-image does not change its result
    for (;;) {
        __syncthreads();                         // every thread has read the previous id
        if (threadIdx.x == 0) ctl[1] = atomicAdd(P.view_queue, 1);
        __syncthreads();
        const int vid = ctl[1];
        if (vid >= F.V) break;
        const int nc = min(F.nb_counts[vid], K);
        const size_t vbase = (size_t)vid * P.ppv;
        // the other colour keeps its state; so does every pixel of a view without neighbours
        for (int e = threadIdx.x; e < P.ppv; e += blockDim.x) {
            const int ex = e % W, ey = e / W;
            pc[e] = prev.cost[vbase + e];
            ps[e] = prev.sel[vbase + e];
            if (nc > 0 && ((ex + ey) & 1) == phase) continue;
            next.plane[vbase + e] = prev.plane[vbase + e];
            next.cost[vbase + e] = prev.cost[vbase + e];
            next.disp[vbase + e] = prev.disp[vbase + e];
            next.sel[vbase + e] = prev.sel[vbase + e];
        }
        if (nc <= 0) { __syncthreads(); continue; }
        Quad T;
        if (!stage_view<BLUR, TEX>(smem, L, F, P, vid, nc, parity, err, T)) return false;
        parity ^= 1u;
        if (threadIdx.x == 0) ctl[0] = 0;
        __syncthreads();

        for (;;) {
            int g = 0;
            if (lane == 0) g = atomicAdd(&ctl[0], 1);
            g = __shfl_sync(kFullMask, g, 0);
            if (g >= n_upd) break;
            int x = 0, y = 0;
            nth_pixel(g, phase, W, H, x, y);
            const int center = y * W + x;
            const size_t idx = vbase + center;
            const PixWin pw = pixel_window(P, x, y);
            build_table<BLUR>(T, P, pw, x, y, S.tab, lane);
            // NCC passes of this pixel: hypotheses [0, nh) on the views in vmask, except
            // the hypotheses in skip (the tap loop's invariants by value, see eval_hyps)
            auto eval = [&](int nh_, uint64_t skip, uint32_t vmask) {
                eval_hyps<BLUR, COUNT, SHIFT, TEX>(T, P, S, pw, P.W_bits, P.H_bits, (uint32_t)T.qs, (float)P.inc, S.tab,
                                                   x, y, nh_, nc, lane, skip, vmask);
            };

            // ---- propagation candidates and the current plane --------------
            // Row 0 holds the current plane, then one row per distinct candidate plane:
            // a cost vector depends only on the pixel and the plane, so candidates whose
            // planes are bit-identical (to each other or to the current plane) share a
            // row.  The current plane's vector is the one stored when this pixel was last
            // updated, when that store is valid; otherwise it is evaluated.
            Cands C;
            find_candidates(pc, x, y, W, H, C);
            const float4 cur_plane = prev.plane[idx];
            uint64_t slots = 0;                          // row of slot s in bits [4s, 4s + 4); slot 8 = row 0
            int nh = 1;
            if (lane == 0) {
                S.plane[0] = cur_plane;
                for (int s = 0; s < 8; ++s) {
                    if (!C.flag[s] || C.src[s] >= 0) continue;
                    const float4 q = prev.plane[vbase + C.pos[s]];
                    int r = COUNT ? nh : 0;                  // tap counting evaluates every candidate, as the reference
                    for (; r < nh; ++r) {
                        const float4 o = S.plane[r];
                        if (__float_as_uint(o.x) == __float_as_uint(q.x) && __float_as_uint(o.y) == __float_as_uint(q.y) &&
                            __float_as_uint(o.z) == __float_as_uint(q.z) && __float_as_uint(o.w) == __float_as_uint(q.w))
                            break;
                    }
                    if (r == nh) S.plane[nh++] = q;
                    slots |= (uint64_t)r << (4 * s);
                }
                for (int s = 0; s < 8; ++s)
                    if (C.flag[s] && C.src[s] >= 0) slots |= ((slots >> (4 * C.src[s])) & 15ull) << (4 * s);
            }
            slots = __shfl_sync(kFullMask, slots, 0);
            nh = __shfl_sync(kFullMask, nh, 0);
            const bool use_cvec = !COUNT && P.cvec_ok;
            if (use_cvec && lane < nc) S.cost[lane] = P.cvec[idx * K + lane];
            __syncwarp();
            eval(nh, use_cvec ? 1ull : 0ull, ~0u);
#define SLOT(s) ((int)((slots >> (4 * (s))) & 15ull))
#define COSTA(s, k) S.cost[SLOT(s) * K + (k)]

            // ---- view-selection priors and sampling (AdaptMIPMFrame.cu:797-875)
            DrawStream g2;
            g2.init(P.seed, sweep_id, (uint32_t)idx);
            uint32_t tsel = 0;
            uint64_t vw_lo = 0, vw_hi = 0;
            {
                const int dpos[4] = { (y > 0) ? center - W : -1, (y < H - 1) ? center + W : -1,
                                      (x > 0) ? center - 1 : -1, (x < W - 1) ? center + 1 : -1 };
                const float thr = __fmul_rn(0.8f, pfd_expf(__fdiv_rn((float)(iter * iter), -90.0f)));
                const float p_default = pfd_expf(__fdiv_rn(__fmul_rn(thr, thr), -0.32f));
                // lane i works out view i's probability; the sums over views then run in
                // view order on every lane, as the reference's loop does
                float pr = 0.0f;
                if (lane < nc) {
                    const int i = lane;
                    float prior = 0.0f;
                    for (int ii = 0; ii < 4; ++ii) {
                        if (dpos[ii] < 0 || !C.flag[2 * ii]) continue;
                        prior = __fadd_rn(prior, ((ps[dpos[ii]] >> i) & 1u) ? 0.9f : 0.1f);
                    }
                    float cj[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) cj[j] = C.flag[j] ? COSTA(j, i) : 0.0f;
                    float count = 0.0f, tmpw = 0.0f;
                    int count_false = 0;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        if (!C.flag[j]) continue;
                        const float c = cj[j];
                        if (c < thr) {
                            tmpw = __fadd_rn(tmpw, pfd_expf(__fdiv_rn(__fmul_rn(c, c), -0.18f)));
                            count = __fadd_rn(count, 1.0f);
                        }
                        if (c > 1.2f) count_false++;
                    }
                    if (count > 2.0f && count_false < 3) pr = __fdiv_rn(tmpw, count);
                    else if (count_false < 3) pr = p_default;
                    pr = __fmul_rn(pr, prior);
                }
                float psum = 0.0f;
                for (int i = 0; i < nc; ++i) psum = __fadd_rn(psum, __shfl_sync(kFullMask, pr, i));
                float cdf_l = 0.0f;
                {   // TransformPDFToCDF (CudaUtil.cu:491-507)
                    const float inv = __fdiv_rn(1.0f, psum);
                    float cum = 0.0f;
                    for (int i = 0; i < nc; ++i) {
                        cum = __fmaf_rn(__shfl_sync(kFullMask, pr, i), inv, cum);
                        if (lane == i) cdf_l = cum;
                    }
                }
                for (int sample = 0; sample < 15; ++sample) {
                    const float rp = __fsub_rn(g2.uniform(), 1.1920928955078125e-07f);
                    const unsigned hit = __ballot_sync(kFullMask, lane < nc && cdf_l > rp);
                    if (hit) {
                        const int id = __ffs(hit) - 1;        // the first view whose CDF exceeds rp
                        if (id < 16) vw_lo += 1ull << (id * 4); else vw_hi += 1ull << ((id - 16) * 4);
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
#undef COSTA
            // weighted costs: current plane, then the candidates in slot order
            weigh_hyps(S, K, nh, nc, vw_lo, vw_hi, lane, ~0u);
            float best_cost = S.wres[0];
            int best_min = S.wmin[0];
            float4 best_plane = cur_plane;
            int best_row = 0;
            for (int s = 0; s < 8; ++s) {
                if (!C.flag[s]) continue;
                const float c = S.wres[SLOT(s)];
                if (c < best_cost) { best_cost = c; best_plane = S.plane[SLOT(s)]; best_min = S.wmin[SLOT(s)]; best_row = SLOT(s); }
            }
#undef SLOT
            // this lane's entry of the best vector so far (the rows are reused below)
            float best_vec = lane < nc ? S.cost[best_row * K + lane] : 0.0f;
            __syncwarp();

            // ---- cross-view proposals (AdaptMIPMFrame.cu:907-936) and refinement
            // (PlaneHypothesisRefinement_Frame, :400-471), evaluated together.  Proposals
            // are built from the best plane so far and the refinement candidates from the
            // best plane after the proposals; both are built here from the current best
            // and rebuilt below when a proposal wins.  The refinement's random draws do
            // not depend on the best plane, so they are taken now, in their order.
            const int nsel = __popc(tsel);
            (void)g2.uniform();                          // depth_rand: drawn, never used
            const float4 rn = random_normal(g2);
            const float u1 = g2.uniform(), u2 = g2.uniform(), u3 = g2.uniform();
            const float u4 = g2.uniform();
            const float4 c0 = random_plane(g2, P.depth_min, P.depth_max);
            bool partial = false;
            if constexpr (!COUNT) {
                int qn = -1, kn = -1;
                if (lane < nsel) {
                    kn = nth_set_bit(tsel, lane);
                    const int nvid = F.nb_ids[vid * K + kn];
                    if (nvid >= 0) qn = proposal_pos(T.geo[kn], x, y, W, H, best_plane);
                }
                const unsigned actm = __ballot_sync(kFullMask, qn >= 0);
                if (qn >= 0) {
                    const int nvid = F.nb_ids[vid * K + kn];
                    S.plane[__popc(actm & ((1u << lane) - 1u))] =
                        proposal_plane(T.geo[kn], prev.plane + (size_t)nvid * P.ppv, qn, x, y, W);
                }
                if (lane < nsel) S.aux[lane] = qn;
                const int nact = __popc(actm);
                float4 cand[5];
                refine_candidates(x, y, best_plane, c0, rn, u1, u2, u3, u4, P.pert_pi, cand);
                // the candidate equal to the best plane has the best cost and cannot win
                bool skip3 = __float_as_uint(cand[3].w) == __float_as_uint(best_plane.w);
                const int r0 = nact;                         // rows of the refinement candidates
                if (lane == 0)
                    for (int i = 0; i < 5; ++i) S.plane[r0 + i] = cand[i];
                __syncwarp();
                eval(r0 + 5, skip3 ? (1ull << (r0 + 3)) : 0ull, tsel);
                weigh_hyps(S, K, r0 + 5, nc, vw_lo, vw_hi, lane, tsel);

                bool changed = false;
                int hs = 0;                                  // speculative row of proposal n
                for (int n = 0; n < nsel; ++n) {
                    const int k = nth_set_bit(tsel, n);
                    const int nvid = F.nb_ids[vid * K + k];
                    const int spec_q = S.aux[n];
                    int q = spec_q;
                    if (changed) q = (nvid >= 0) ? proposal_pos(T.geo[k], x, y, W, H, best_plane) : -1;
                    float c = kCostMax;
                    int cmin = -1;
                    float4 proxy = make_float4(0.f, 0.f, 1.f, 0.f);
                    if (q >= 0 && q == spec_q) {
                        c = S.wres[hs];
                        cmin = S.wmin[hs];
                        proxy = S.plane[hs];
                    } else if (q >= 0) {
                        // the best plane moved the sample position: rebuild this proposal in its
                        // own row (or the spare row after the refinement candidates) and evaluate it
                        const int row = (spec_q >= 0) ? hs : r0 + 5;
                        proxy = proposal_plane(T.geo[k], prev.plane + (size_t)nvid * P.ppv, q, x, y, W);
                        __syncwarp();
                        if (lane == 0) S.plane[row] = proxy;
                        __syncwarp();
                        eval(row + 1, (1ull << row) - 1ull, tsel);
                        weigh_hyps(S, K, row + 1, nc, vw_lo, vw_hi, lane, tsel);
                        c = S.wres[row];
                        cmin = S.wmin[row];
                    }
                    if (spec_q >= 0) ++hs;
                    if (q >= 0 && c < best_cost) { best_cost = c; best_plane = proxy; best_min = cmin; changed = true; partial = true; }
                }
                if (changed) {
                    // candidates 2-4 follow the best plane: rebuild and evaluate them again
                    refine_candidates(x, y, best_plane, c0, rn, u1, u2, u3, u4, P.pert_pi, cand);
                    skip3 = __float_as_uint(cand[3].w) == __float_as_uint(best_plane.w);
                    __syncwarp();
                    if (lane == 0)
                        for (int i = 2; i < 5; ++i) S.plane[r0 + i] = cand[i];
                    __syncwarp();
                    const uint64_t redo = (7ull << (r0 + 2)) & ~(skip3 ? (1ull << (r0 + 3)) : 0ull);
                    eval(r0 + 5, ~redo, tsel);
                    weigh_hyps(S, K, r0 + 5, nc, vw_lo, vw_hi, lane, tsel);
                }
                for (int i = 0; i < 5; ++i) {
                    if (i == 3 && skip3) continue;
                    const float c = S.wres[r0 + i];
                    if (c < best_cost) { best_cost = c; best_plane = cand[i]; best_min = S.wmin[r0 + i]; partial = true; }
                }
            } else {
                // tap counting: the reference's own evaluations, proposals one by one from the
                // best plane so far, then all five refinement candidates, on every view
                for (int n = 0; n < nsel; ++n) {
                    const int k = nth_set_bit(tsel, n);
                    const int nvid = F.nb_ids[vid * K + k];
                    const int q = (nvid >= 0) ? proposal_pos(T.geo[k], x, y, W, H, best_plane) : -1;
                    if (q < 0) continue;
                    const float4 proxy = proposal_plane(T.geo[k], prev.plane + (size_t)nvid * P.ppv, q, x, y, W);
                    __syncwarp();
                    if (lane == 0) S.plane[0] = proxy;
                    __syncwarp();
                    eval(1, 0ull, ~0u);
                    weigh_hyps(S, K, 1, nc, vw_lo, vw_hi, lane, ~0u);
                    const float c = S.wres[0];
                    if (c < best_cost) { best_cost = c; best_plane = proxy; best_min = S.wmin[0]; }
                }
                float4 cand[5];
                refine_candidates(x, y, best_plane, c0, rn, u1, u2, u3, u4, P.pert_pi, cand);
                __syncwarp();
                if (lane == 0)
                    for (int i = 0; i < 5; ++i) S.plane[i] = cand[i];
                __syncwarp();
                eval(5, 0ull, ~0u);
                weigh_hyps(S, K, 5, nc, vw_lo, vw_hi, lane, ~0u);
                for (int i = 0; i < 5; ++i) {
                    const float c = S.wres[i];
                    if (c < best_cost) { best_cost = c; best_plane = cand[i]; best_min = S.wmin[i]; }
                }
            }
            if (partial || (COUNT && P.acmm)) {
                // proposals and refinement candidates were evaluated on the selected views
                // only, which fixes their weighted cost; the winner's lowest-cost view runs
                // over every view, and its vector is stored, so the whole vector is
                // evaluated again (one NCC per lane, a single pass over the taps).  Tap
                // counting in the ACMM matcher evaluates it always: that matcher's
                // write-back evaluates the final plane on every view.
                __syncwarp();
                if (lane == 0) S.plane[0] = best_plane;
                __syncwarp();
                eval(1, 0ull, ~0u);
                weigh_hyps(S, K, 1, nc, vw_lo, vw_hi, lane, ~0u);
                best_min = S.wmin[0];
                best_vec = lane < nc ? S.cost[lane] : 0.0f;
                best_row = -1;
            }
            // the stored vector of the new current plane (unchanged when the current
            // plane stays and its stored vector was used)
            if (!COUNT && P.cvec && lane < nc && !(best_row == 0 && P.cvec_ok)) P.cvec[idx * K + lane] = best_vec;
            // ACMM write-back (AdaptMIPMFrameACMM.cu:880-900, RecomputeSupportCostDisp_Frame
            // :259-280): the final plane's vector over every view (best_vec) gives the
            // stored cost (mean of the top-k), the selected views (the top-k mask) and the
            // disp of the lowest-cost view; DetailRestorer_FrameACMM does nothing
            // without a warm start
            float acv[kMaxNb];
            if (P.acmm)
                for (int i = 0; i < nc; ++i) acv[i] = __shfl_sync(kFullMask, best_vec, i);
            if (lane == 0) {
                uint32_t sel_out = tsel;
                float cost_out = best_cost;
                int disp_view = best_min;
                if (P.acmm) {
                    disp_view = -1;
                    int valid = 0;
                    for (int i = 0; i < nc; ++i)
                        if (acv[i] < 2.0f) {
                            ++valid;
                            if (disp_view < 0 || acv[i] < acv[disp_view]) disp_view = i;
                        }
                    cost_out = 2.0f;
                    sel_out = 0;
                    if (valid > 0) {
                        const int kk = min(valid, P.top_k);
                        float tmp[kMaxNb];
                        for (int i = 0; i < nc; ++i) tmp[i] = acv[i];
                        for (int i = 0; i < kk; ++i)
                            for (int j = i + 1; j < nc; ++j)
                                if (tmp[j] < tmp[i]) { const float t = tmp[i]; tmp[i] = tmp[j]; tmp[j] = t; }
                        float m = 0.0f;
                        for (int i = 0; i < kk; ++i) m = __fadd_rn(m, tmp[i]);
                        cost_out = __fdiv_rn(m, (float)kk);
                        for (int i = 0; i < nc; ++i)
                            if (acv[i] <= tmp[kk - 1]) sel_out |= 1u << i;
                    }
                }
                float4 best_disp = make_float4(0.f, 0.f, 0.f, 0.f);
                if (disp_view >= 0)
                    best_disp = geo_disp(T.geo[disp_view], x, y, to_disparity(x, y, disparity_plane(x, y, best_plane)));
                next.plane[idx] = best_plane;
                next.cost[idx] = cost_out;
                next.disp[idx] = best_disp;
                next.sel[idx] = sel_out;
            }
            __syncwarp();
        }
        __syncthreads();                         // shared memory is restaged for the next view
    }
    return true;
}

// The staging barrier (offset 0 of every plan), once per launch.
__device__ __forceinline__ void init_barrier(unsigned char* smem)
{
    if (threadIdx.x == 0) mbar_init((uint64_t*)smem, 1);
    __syncthreads();
}

template <bool BLUR, bool COUNT, bool SHIFT, int SHAPE, bool TEX>
__global__ void __launch_bounds__(32 * ShapeOf<SHAPE>::warps, ShapeOf<SHAPE>::min_ctas)
pm_sweep_warp_kernel(FrameDev F, PmParams P, StateDev prev, StateDev next, int iter, int phase, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    init_barrier(smem);
    uint32_t parity = 0;
    sweep_frame<BLUR, COUNT, SHIFT, TEX, ShapeOf<SHAPE>::warps>(smem, F, P, prev, next, iter, phase, err, parity);
}

// Several frames' half-sweeps in one launch, in list order: a CTA that finds a
// frame's queue empty moves on to the next frame at once, so one frame's tail
// overlaps the next one's start.  The dynamic shared memory is the largest of
// the frames' plans.
template <bool BLUR, bool SHIFT, int SHAPE, bool TEX>
__global__ void __launch_bounds__(32 * ShapeOf<SHAPE>::warps, ShapeOf<SHAPE>::min_ctas)
pm_sweep_batch_kernel(const SweepItem* items, int n, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    init_barrier(smem);
    uint32_t parity = 0;
    for (int b = 0; b < n; ++b) {
        const SweepItem it = items[b];
        if (!sweep_frame<BLUR, false, SHIFT, TEX, ShapeOf<SHAPE>::warps>(smem, it.F, it.P, it.prev, it.next, it.iter,
                                                                         it.phase, err, parity))
            return;
    }
}

int sweep_shape_warps(int shape) { return kShapeWarps[(shape >= 0 && shape < kSweepShapes) ? shape : 0]; }

// Tap counting stages the neighbours in shared memory; the other sweeps fetch
// them from the frame's textures when it has them.
static bool uses_tex(const FrameDev& F, const PmParams& P) { return F.tex != nullptr && P.tap_counter == nullptr; }

int sweep_warp_smem_bytes(const PmParams& P, bool blur, int shape, bool tex)
{
    return Plan::make(P.W, P.H, P.K, P.ntap, blur, P.tile_stride, sweep_shape_warps(shape), tex && !P.tap_counter).total;
}

int sweep_warp_stride(int K) { return sweep_warp_words(K); }

size_t sweep_warp_scratch_bytes(const PmParams& P, int n_ctas, int shape)
{
    return (size_t)n_ctas * sweep_shape_warps(shape) * (size_t)sweep_warp_words(P.K) * 4u;
}

// Dynamic shared memory of a sweep kernel, and for the texture-fetch kernels the
// carveout they ask for: the shared memory of the CTAs per SM the shape's
// registers allow (with the 1 KB each CTA reserves), so the rest of the SM's
// 256 KB stays L1 and texture cache.  The shared-memory kernels keep the
// driver's choice.
static cudaError_t set_smem(const void* k, int smem, int shape, bool tex)
{
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess || !tex) return e;
    const int ctas = kShapeCtas[(shape >= 0 && shape < kSweepShapes) ? shape : 0];
    const long need = (long)ctas * (smem + 1024);
    const int pct = (int)std::min<long>(100, (need * 100 + 228 * 1024 - 1) / (228 * 1024) + 1);
    return cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

template <class Kern>
static cudaError_t launch_k(Kern k, dim3 grid, dim3 block, int smem, int shape, bool tex, cudaStream_t st,
                            void** args)
{
    cudaError_t e = set_smem((const void*)k, smem, shape, tex);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernel((const void*)k, grid, block, args, (size_t)smem, st);
}

// The half-sweep kernel of one variant; tap counting exists in shape 0 with
// shared-memory fetches only.
template <int SHAPE, bool TEX>
static const void* warp_kernel_of(bool blur, bool shift)
{
    if (shift) return blur ? (const void*)pm_sweep_warp_kernel<true, false, true, SHAPE, TEX>
                           : (const void*)pm_sweep_warp_kernel<false, false, true, SHAPE, TEX>;
    return blur ? (const void*)pm_sweep_warp_kernel<true, false, false, SHAPE, TEX>
                : (const void*)pm_sweep_warp_kernel<false, false, false, SHAPE, TEX>;
}

template <int SHAPE>
static const void* warp_kernel_of(bool blur, bool shift, bool tex)
{
    return tex ? warp_kernel_of<SHAPE, true>(blur, shift) : warp_kernel_of<SHAPE, false>(blur, shift);
}

static const void* warp_kernel(int shape, bool blur, bool count, bool shift, bool tex)
{
    if (count) {
        if (shift) return blur ? (const void*)pm_sweep_warp_kernel<true, true, true, 0, false>
                               : (const void*)pm_sweep_warp_kernel<false, true, true, 0, false>;
        return blur ? (const void*)pm_sweep_warp_kernel<true, true, false, 0, false>
                    : (const void*)pm_sweep_warp_kernel<false, true, false, 0, false>;
    }
    switch (shape) {
    case 1: return warp_kernel_of<1>(blur, shift, tex);
    case 2: return warp_kernel_of<2>(blur, shift, tex);
    case 3: return warp_kernel_of<3>(blur, shift, tex);
    default: return warp_kernel_of<0>(blur, shift, tex);
    }
}

template <int SHAPE, bool TEX>
static const void* batch_kernel_of(bool blur, bool shift)
{
    if (blur) return shift ? (const void*)pm_sweep_batch_kernel<true, true, SHAPE, TEX>
                           : (const void*)pm_sweep_batch_kernel<true, false, SHAPE, TEX>;
    return shift ? (const void*)pm_sweep_batch_kernel<false, true, SHAPE, TEX>
                 : (const void*)pm_sweep_batch_kernel<false, false, SHAPE, TEX>;
}

template <int SHAPE>
static const void* batch_kernel_of(bool blur, bool shift, bool tex)
{
    return tex ? batch_kernel_of<SHAPE, true>(blur, shift) : batch_kernel_of<SHAPE, false>(blur, shift);
}

static const void* batch_kernel(int shape, bool blur, bool shift, bool tex)
{
    switch (shape) {
    case 1: return batch_kernel_of<1>(blur, shift, tex);
    case 2: return batch_kernel_of<2>(blur, shift, tex);
    case 3: return batch_kernel_of<3>(blur, shift, tex);
    default: return batch_kernel_of<0>(blur, shift, tex);
    }
}

static cudaError_t grid_for(const void* k, int threads, int smem, int shape, bool tex, int* n_ctas)
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = set_smem(k, smem, shape, tex);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *n_ctas = sms * per_sm;
    return cudaSuccess;
}

cudaError_t sweep_warp_grid(const FrameDev& F, const PmParams& P, int* n_ctas, int shape)
{
    const bool blur = F.blur != nullptr, tex = uses_tex(F, P);
    if (P.tap_counter) shape = 0;
    return grid_for(warp_kernel(shape, blur, P.tap_counter != nullptr, P.shifted != 0, tex),
                    32 * sweep_shape_warps(shape), sweep_warp_smem_bytes(P, blur, shape, tex), shape, tex, n_ctas);
}

cudaError_t launch_sweep_warp(const FrameDev& F, const PmParams& P, const StateDev& prev, const StateDev& next,
                              int iter, int phase, int n_ctas, int* err, cudaStream_t st, int shape)
{
    const bool blur = F.blur != nullptr, tex = uses_tex(F, P);
    if (P.tap_counter) shape = 0;
    const int smem = sweep_warp_smem_bytes(P, blur, shape, tex);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    const int grid = std::max(1, std::min(n_ctas, F.V));
    cudaError_t qe = cudaMemsetAsync(P.view_queue, 0, sizeof(int), st);
    if (qe != cudaSuccess) return qe;
    FrameDev f = F; PmParams p = P; StateDev a = prev, b = next; int it = iter, ph = phase; int* e = err;
    void* args[] = { &f, &p, &a, &b, &it, &ph, &e };
    return launch_k(warp_kernel(shape, blur, P.tap_counter != nullptr, P.shifted != 0, tex), grid,
                    32 * sweep_shape_warps(shape), smem, shape, tex, st, args);
}

// One thread per texel; a write outside a surface is dropped (boundary mode
// zero), though none is made: v % layers < the layers of surface v / layers.
__global__ void __launch_bounds__(256) tex_fill_kernel(const uint8_t* tiles, int V, int W, int H, int ts,
                                                       const cudaSurfaceObject_t* surfs, int layers)
{
    const int per = W * H;
    const size_t n = (size_t)V * per;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int v = (int)(e / per), r = (int)(e - (size_t)v * per);
        const int y = r / W, x = r - y * W;
        surf2DLayeredwrite<float>((float)tiles[(size_t)v * ts + r], surfs[v / layers], x * (int)sizeof(float), y,
                                  v % layers, cudaBoundaryModeZero);
    }
}

cudaError_t launch_tex_fill(const uint8_t* tiles, int V, int W, int H, int tile_stride,
                            const cudaSurfaceObject_t* surfs, int layers, cudaStream_t st)
{
    if (V <= 0 || W <= 0 || H <= 0 || layers <= 0) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t n = (size_t)V * W * H;
    const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)std::max(sms, 1) * 8);
    tex_fill_kernel<<<grid, 256, 0, st>>>(tiles, V, W, H, tile_stride, surfs, layers);
    return cudaGetLastError();
}

cudaError_t sweep_batch_grid(int smem, bool blur, bool shift, bool tex, int* n_ctas, int shape)
{
    return grid_for(batch_kernel(shape, blur, shift, tex), 32 * sweep_shape_warps(shape), smem, shape, tex, n_ctas);
}

cudaError_t launch_sweep_batch(const SweepItem* items, int n, bool blur, bool shift, bool tex, int smem, int n_ctas,
                               int* err, cudaStream_t st, int shape)
{
    if (n <= 0) return cudaSuccess;
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    const SweepItem* it = items; int nn = n; int* e = err;
    void* args[] = { &it, &nn, &e };
    return launch_k(batch_kernel(shape, blur, shift, tex), dim3(std::max(1, n_ctas)), 32 * sweep_shape_warps(shape),
                    smem, shape, tex, st, args);
}

}  // namespace pfd
