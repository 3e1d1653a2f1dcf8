// pm_device.cuh -- device building blocks of the micro-image PatchMatch:
// plane geometry, hexagonal-baseline mapping, shared-memory micro-image tiles,
// and the bilateral NCC evaluated for one plane against a chunk of neighbour
// micro-images at once.
//
// Reference: MIStereo/AdaptMIPMFrame.cu:24-317,350-471, MIStereo/CudaUtil.cu:
// 13-170,341-361,491-507, MIStereo/AdaptMIPMUtil.cu:463-501,625-649.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "canon.cuh"

namespace pfd {

constexpr int kMaxNb = 32;           // selected-view bitmask width (CudaUtil.cu:13-21)
constexpr float kCostMax = 2.0f;

// Per-launch constants (PatchMatchParamsLF, LFDepthInfo.h:19-46, as the Frame
// path sets them in AdaptMIPMFrame.cpp:126-143).
struct PmParams {
    int W, H, ppv;          // micro-image window (mi_width_for_match) and pixels per view
    int K;                  // neighbour-id stride (m_max_neighbors)
    int radius, inc, ntap;  // patch radius, radius_increment, taps per patch side
    int top_k;
    float ss2, cc2;         // (2 sigma_s) sigma_s and (2 sigma_c) sigma_c
    float depth_min, depth_max;
    float base, inv_base;   // Base and 1 / max(Base, 1e-6)
    float pert_pi;          // (float)(0.02 * pi)
    uint32_t W_bits, H_bits;   // __float_as_uint((float)W), ... for unsigned bound tests
    int tile_stride;        // bytes per micro-image tile in HBM (W*H rounded up to 16)
    uint64_t seed;
    unsigned long long* tap_counter;   // calibration runs only: in-bounds NCC taps evaluated
    float* cost_scratch;    // sweep: per warp, the cost vectors of its current pixel
    size_t scratch_floats;  // sweep: floats cost_scratch holds (checked against the grid)
    int scratch_stride;     // sweep: floats of cost_scratch per warp, the same for every frame of a launch
    float* cvec;            // [V * ppv][K]: cost vector of each pixel's current plane (init and sweeps write it)
    int cvec_ok;            // sweep: cvec holds the vectors of the updated colour's current planes
    int shifted;            // 0: the reference's raw NCC moments; 1: moments of (pixel - centre pixel)
    int* view_queue;        // sweep: micro-images are handed out in order from this counter (zeroed per launch)
    float blur_gain;        // blur penalty gain: 2 (Frame matcher), 0.8 (ACMM matcher)
    int acmm;               // 1: ACMM write-back (top-k cost, views and disp of the final plane)
};

struct FrameDev {
    const uint8_t* gray;    // [V][tile_stride]
    const uint8_t* blur;    // [V][tile_stride] or nullptr
    const float2* centers;  // [V]
    const int* nb_ids;      // [V][K]
    const int* nb_counts;   // [V]
    int V;
    // The tiles again as layered float textures (linear filter, unnormalised
    // coordinates, clamped), the reference's micro-image textures with
    // tex_layers micro-images per texture: view v is layer v % tex_layers of
    // texture v / tex_layers.  nullptr where the frame has none.
    const cudaTextureObject_t* tex;        // gray
    const cudaTextureObject_t* tex_blur;   // blur, or nullptr
    int tex_layers;
};

struct StateDev {
    float4* plane;          // nx, ny, nz, disparity
    float* cost;
    float4* disp;           // d, d_real, baseline, baseline / d_real
    uint32_t* sel;
};

// Per (reference, neighbour) pair constants of DisparityGeometricMapOperate_Hex
// (AdaptMIPMUtil.cu:625-649) and the NCC's source step (AdaptMIPMFrame.cu:106-108).
struct NbGeo {
    float bx, by;           // c_ref - c_nb
    float baseline;         // |c_nb - c_ref|
    float dxn, dyn;         // (c_ref - c_nb) / baseline
    float scale;            // baseline / Base
    float stx, sty;         // (c_ref - c_nb) * inv_base
};

__device__ __forceinline__ NbGeo make_geo(float2 c0, float2 c1, const PmParams& P)
{
    NbGeo g;
    const float ey = __fsub_rn(c1.y, c0.y), ex = __fsub_rn(c1.x, c0.x);
    g.baseline = __fsqrt_rn(__fmaf_rn(ex, ex, __fmul_rn(ey, ey)));
    g.bx = __fsub_rn(c0.x, c1.x);
    g.by = __fsub_rn(c0.y, c1.y);
    g.dxn = __fdiv_rn(g.bx, g.baseline);
    g.dyn = __fdiv_rn(g.by, g.baseline);
    g.scale = __fdiv_rn(g.baseline, P.base);
    g.stx = __fmul_rn(g.bx, P.inv_base);
    g.sty = __fmul_rn(g.by, P.inv_base);
    return g;
}

// DisparityPlane, CudaUtil.cu:158-170
__device__ __forceinline__ float3 disparity_plane(int px, int py, float4 h)
{
    float3 d;
    d.x = __fdiv_rn(-h.x, h.z);
    d.y = __fdiv_rn(-h.y, h.z);
    float num = __fmaf_rn(h.y, (float)py, __fmul_rn(h.x, (float)px));
    num = __fmaf_rn(h.z, h.w, num);
    d.z = __fdiv_rn(num, h.z);
    return d;
}

// to_disparity, CudaUtil.cu:152-156
__device__ __forceinline__ float to_disparity(int px, int py, float3 dp)
{
    return __fadd_rn(__fmaf_rn(dp.y, (float)py, __fmul_rn(dp.x, (float)px)), dp.z);
}

// NormalizeVec3, CudaUtil.cu:49-56
__device__ __forceinline__ float4 normalize3(float4 v)
{
    const float n2 = __fmaf_rn(v.z, v.z, __fmaf_rn(v.y, v.y, __fmul_rn(v.x, v.x)));
    const float inv = pfd_rsqrtf(n2);
    v.x = __fmul_rn(v.x, inv); v.y = __fmul_rn(v.y, inv); v.z = __fmul_rn(v.z, inv);
    return v;
}

// Anchor of p in the neighbour window (DisparityGeometricMapOperate_Hex p1).
__device__ __forceinline__ float2 geo_anchor(const NbGeo& g, int px, int py, float d)
{
    return make_float2(__fmaf_rn(__fmul_rn(g.dxn, d), g.scale, (float)px),
                       __fmaf_rn(__fmul_rn(g.dyn, d), g.scale, (float)py));
}

// disparity_basline of DisparityGeometricMapOperate_Hex (d, d_real, baseline, ratio).
__device__ __forceinline__ float4 geo_disp(const NbGeo& g, int px, int py, float d)
{
    const float2 a = geo_anchor(g, px, py, d);
    const float dr2 = __fmaf_rn(g.by, __fsub_rn((float)py, a.y), __fmul_rn(g.bx, __fsub_rn((float)px, a.x)));
    const float d_real = __fsqrt_rn(dr2);
    const double ratio = __ddiv_rn((double)g.baseline, __dadd_rn((double)d_real, 1e-7));
    return make_float4(d, d_real, g.baseline, __double2float_rn(ratio));
}

// GenerateRandomNormal_MIPM (AdaptMIPMUtil.cu:463-492); the rejection loop is
// bounded at 64 pairs (probability of reaching it ~1e-43), then +z.
__device__ __forceinline__ float4 random_normal(DrawStream& g)
{
    float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
    int attempts = 0;
    while (s >= 1.0f) {
        if (attempts++ == 64) { q1 = 0.0f; q2 = 0.0f; s = 0.0f; break; }
        q1 = __fmaf_rn(2.0f, g.uniform(), -1.0f);
        q2 = __fmaf_rn(2.0f, g.uniform(), -1.0f);
        s = __fmaf_rn(q2, q2, __fmul_rn(q1, q1));
    }
    const float sq = __fsqrt_rn(__fsub_rn(1.0f, s));
    float4 n = make_float4(__fmul_rn(__fmul_rn(2.0f, q1), sq), __fmul_rn(__fmul_rn(2.0f, q2), sq),
                           __fmaf_rn(-2.0f, s, 1.0f), 0.0f);
    return normalize3(n);
}

// GenerateRandomPlaneHypothesis_MIPM (AdaptMIPMUtil.cu:494-501)
__device__ __forceinline__ float4 random_plane(DrawStream& g, float dmin, float dmax)
{
    const float depth = __fmaf_rn(g.uniform(), __fsub_rn(dmax, dmin), dmin);
    float4 h = random_normal(g);
    h.w = depth;
    return h;
}

// GeneratePerturbedNormalLF (CudaUtil.cu:105-142) from the three uniforms it
// draws (u1, u2, u3 in draw order).  The perturbed normal keeps n.w (the
// reference leaves .w uninitialised there).
__device__ __forceinline__ float4 perturbed_normal_u(int px, int py, float4 n, float u1, float u2, float u3, float pert)
{
    const float X0 = (float)px, X1 = (float)py, X2 = 1.0f;
    const float norm = __fsqrt_rn(__fmaf_rn(X2, X2, __fmaf_rn(X1, X1, __fmul_rn(X0, X0))));
    const float vx = __fdiv_rn(X0, norm), vy = __fdiv_rn(X1, norm), vz = __fdiv_rn(X2, norm);
    const float a1 = __fmul_rn(__fsub_rn(u1, 0.5f), pert);
    const float a2 = __fmul_rn(__fsub_rn(u2, 0.5f), pert);
    const float a3 = __fmul_rn(__fsub_rn(u3, 0.5f), pert);
    const float s1 = pfd_sin_small(a1), s2 = pfd_sin_small(a2), s3 = pfd_sin_small(a3);
    const float c1 = pfd_cos_small(a1), c2 = pfd_cos_small(a2), c3 = pfd_cos_small(a3);
    const float R0 = __fmul_rn(c2, c3);
    const float R1 = __fmaf_rn(-c1, s3, __fmul_rn(__fmul_rn(c3, s1), s2));
    const float R2 = __fmaf_rn(__fmul_rn(c1, c3), s2, __fmul_rn(s1, s3));
    const float R3 = __fmul_rn(c2, s3);
    const float R4 = __fmaf_rn(__fmul_rn(s1, s2), s3, __fmul_rn(c1, c3));
    const float R5 = __fmaf_rn(-c3, s1, __fmul_rn(__fmul_rn(c1, s2), s3));
    const float R6 = -s2;
    const float R7 = __fmul_rn(c2, s1);
    const float R8 = __fmul_rn(c1, c2);
    float4 q;
    q.x = __fmaf_rn(R2, n.z, __fmaf_rn(R1, n.y, __fmul_rn(R0, n.x)));
    q.y = __fmaf_rn(R5, n.z, __fmaf_rn(R4, n.y, __fmul_rn(R3, n.x)));
    q.z = __fmaf_rn(R8, n.z, __fmaf_rn(R7, n.y, __fmul_rn(R6, n.x)));
    q.w = n.w;
    const float dot = __fmaf_rn(q.z, vz, __fmaf_rn(q.y, vy, __fmul_rn(q.x, vx)));
    if (dot >= 0.0f) q = n;
    return normalize3(q);
}

// GeneratePerturbedNormalLF drawing its uniforms from g.
__device__ __forceinline__ float4 perturbed_normal(int px, int py, float4 n, DrawStream& g, float pert)
{
    const float u1 = g.uniform();
    const float u2 = g.uniform();
    const float u3 = g.uniform();
    return perturbed_normal_u(px, py, n, u1, u2, u3, pert);
}

// EncodePlaneHypothesisFromDispPlaneDevice (AdaptMIPMFrame.cu:36-53)
__device__ __forceinline__ float4 encode_plane(int ax, int ay, float alpha, float beta, float gamma)
{
    float nx = -alpha, ny = -beta, nz = 1.0f;
    const float inv = pfd_rsqrtf(__fadd_rn(__fmaf_rn(nz, nz, __fmaf_rn(ny, ny, __fmul_rn(nx, nx))), 1e-12f));
    nx = __fmul_rn(nx, inv); ny = __fmul_rn(ny, inv); nz = __fmul_rn(nz, inv);
    const float d = __fadd_rn(__fmaf_rn(beta, (float)ay, __fmul_rn(alpha, (float)ax)), gamma);
    return make_float4(nx, ny, nz, d);
}

__device__ __forceinline__ float clamp_cost(float v) { return fminf(2.0f, fmaxf(0.0f, v)); }

__device__ __forceinline__ float safe_denom(float v)
{
    if (fabsf(v) < 1e-6f) return (v >= 0.0f) ? 1e-6f : -1e-6f;
    return v;
}

// ---------------------------------------------------------------------------
// Shared-memory image of one reference micro-image and its neighbours.
//
// Neighbour windows are held as integer "row pairs": entry (y, x), y in
// [0, H+1], x in [0, S) with S even and >= W+1, is (T, T' - T) with
// T = I(y, x), T' = I(y, x+1), indices clamped to the window.  A fetch at
// texel (ix, iy) reads entries (iy, ix) and (iy+1, ix), which hold the four
// texels of the bilinear footprint.
//
// The fetch reproduces the texture unit's linear filter as measured on B200
// for integer texels (see the oracle's canon_tex_fetch): coordinates rounded
// half up to 1/256 (one FFMA rounding toward -inf against 2^23 - 127.5), and
// weights w11 = (a b + 128) >> 8, w10 = a - w11, w01 = b - w11,
// w00 = 256 - a - b + w11, i.e.
//   256 s = 256 T00 + a (T10-T00) + b (T01-T00) + w11 (T11-T10-T01+T00),
// an integer below 2^16 that is turned into a float exactly.
// ---------------------------------------------------------------------------
struct Tiles {
    const float* R;         // [H][W] reference texels (as floats)
    const float* RB;        // [H][W] reference blur or nullptr
    uint32_t q_addr;        // shared address of neighbour row pairs, [K][H+2][S] int2
    uint32_t qb_addr;       // same for blur (0 if none)
    int q_stride;           // S, row stride in entries
    int q_bytes;            // bytes per neighbour tile
    const NbGeo* geo;       // [K]
    const int* nb_ok;       // [K] neighbour id valid (>= 0)
    const float* a_s;       // [ntap*ntap] (-sqrt(i^2+j^2)) / ss2, i outer, j inner
    const float* a_c;       // [256] cd / cc2
};

constexpr uint32_t kFullMask = 0xffffffffu;

__device__ __forceinline__ int2 lds_int2(uint32_t addr)
{
    int2 v;
    asm volatile("ld.shared.v2.s32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(addr));
    return v;
}

// 2^23 + floor(256 (s + 0.5) - 127.5), as float bits: the texel index in the
// upper bits, the 8-bit fraction in the low byte.
__device__ __forceinline__ int tex_coord_bits(float s)
{
    return __float_as_int(__fmaf_rd(__fadd_rn(s, 0.5f), 256.0f, 8388480.5f));
}

__device__ __forceinline__ float tex_blend(int tbx, int tby, int2 p0, int2 p1)
{
    const int a = tbx & 0xFF, b = tby & 0xFF;
    const int w11 = (a * b + 128) >> 8;
    const int s256 = (p0.x << 8) + a * p0.y + b * (p1.x - p0.x) + w11 * (p1.y - p0.y);
    return __fsub_rn(__int_as_float(s256 | 0x47000000), 32768.0f);
}

// Bilateral NCC (ComputeBilateralNCC_Frame, AdaptMIPMFrame.cu:73-179) of each
// lane's plane against the neighbours ks[0..nks) (warp-uniform list).  The
// reference-side work of a tap (disparity, texel, bilateral weight) is done
// once and shared by the chunk; every neighbour keeps its own six moment sums
// in the reference's tap order (x offset outer, y offset inner).  The body is
// branch-free: a tap that falls outside either window contributes exact
// zeros (fma(0, s, acc) == acc), so the sums equal the reference's skipping.
// okmask: per lane, bit k set when neighbour k's anchor lies in the window.
template <int KCH, bool BLUR, bool COUNT>
__device__ __forceinline__ void ncc_chunk(const Tiles& T, const PmParams& P, int px, int py, float3 dp,
                                          const int (&ks)[16], int nks, uint32_t okmask, float (&cost)[KCH],
                                          unsigned& ntaps)
{
    const int W = P.W, H = P.H, S = T.q_stride;
    const uint32_t fold = (uint32_t)0x4B0000u * (uint32_t)(S + 1) * 8u;
    float stx[KCH], sty[KCH];
    uint32_t base[KCH], bbase[KCH];
    bool okc[KCH];
    float sr[KCH], srr[KCH], ss[KCH], sss[KCH], srs[KCH], sw[KCH], bsx[KCH], bsy[KCH];
#pragma unroll
    for (int c = 0; c < KCH; ++c) {
        const int k = (c < nks) ? ks[c] : ks[0];
        okc[c] = (c < nks) && ((okmask >> k) & 1u);
        stx[c] = T.geo[k].stx;
        sty[c] = T.geo[k].sty;
        base[c] = T.q_addr + (uint32_t)(k * T.q_bytes) - fold;
        bbase[c] = BLUR ? T.qb_addr + (uint32_t)(k * T.q_bytes) - fold : 0u;
        sr[c] = srr[c] = ss[c] = sss[c] = srs[c] = sw[c] = 0.0f;
        bsx[c] = bsy[c] = 0.0f;
    }
    const float rc = T.R[py * W + px];
    // shifted moments: texels and samples minus the centre texel; both are
    // multiples of 1/256 below 2^16, so the subtraction is exact, and with
    // shift 0 every sum is bit for bit the reference's
    const float sh = P.shifted ? rc : 0.0f;
    const int r = P.radius, inc = P.inc, ntap = P.ntap;
    // Taps are visited by absolute window position (X, Y), X outer, Y inner,
    // over the union of the warp's patches.  Each lane keeps only positions
    // inside its own patch, so it accumulates its taps in exactly the
    // reference order (x offset outer, y offset inner), while the warp's lanes
    // see nearly the same source-window validity and read the same texels.
    bool any_ok = false;
#pragma unroll
    for (int c = 0; c < KCH; ++c) any_ok |= okc[c];
    const int x_lo = max(0, __reduce_min_sync(kFullMask, any_ok ? px : W) - r);
    const int x_hi = min(W - 1, (int)__reduce_max_sync(kFullMask, any_ok ? px : -r - 1) + r);
    const int y_lo = max(0, __reduce_min_sync(kFullMask, any_ok ? py : H) - r);
    const int y_hi = min(H - 1, (int)__reduce_max_sync(kFullMask, any_ok ? py : -r - 1) + r);
    for (int X = x_lo; X <= x_hi; ++X) {
        const int i = X - px;
        const bool rowok = any_ok && i >= -r && i <= r && (inc == 1 || (i + r) % inc == 0);
        if (!__any_sync(kFullMask, rowok)) continue;
        const int xr = X, xrc = X;
        const float fxr = (float)X;
        const float axr = __fmul_rn(dp.x, fxr);
        const int ii = (inc == 1) ? (i + r) : (i + r) / inc;
        float fyr = (float)y_lo;
        for (int Y = y_lo; Y <= y_hi; ++Y, fyr = __fadd_rn(fyr, 1.0f)) {
            const int j = Y - py;
            const bool refok = rowok && j >= -r && j <= r && (inc == 1 || (j + r) % inc == 0);
            if (!__any_sync(kFullMask, refok)) continue;
            const int t = refok ? ii * ntap + ((inc == 1) ? (j + r) : (j + r) / inc) : 0;
            const int yrc = Y;
            const float rv = T.R[Y * W + X];
            const float cd = fabsf(__fsub_rn(rv, rc));
            const int cdi = __float_as_int(__fadd_rn(cd, 8388608.0f)) & 0xFF;
            const float w = refok ? pfd_expf_nonpos(__fsub_rn(T.a_s[t], T.a_c[cdi])) : 0.0f;
            const float rvs = __fsub_rn(rv, sh);
            const float wr = __fmul_rn(w, rvs);
            const float d = __fadd_rn(__fmaf_rn(dp.y, fyr, axr), dp.z);
            (void)xr;
            float rb = 0.0f;
            if (BLUR) rb = __fdiv_rn(T.RB[yrc * W + xrc], 255.0f);
#pragma unroll
            for (int c = 0; c < KCH; ++c) {
                const float sx = __fmaf_rn(stx[c], d, fxr);
                const float sy = __fmaf_rn(sty[c], d, fyr);
                const bool v = okc[c] && refok && (__float_as_uint(sx) < P.W_bits) && (__float_as_uint(sy) < P.H_bits);
                // a tap that no lane of the warp keeps for this neighbour is skipped whole
                if (!__any_sync(kFullMask, v)) continue;
                if (COUNT) ntaps += v ? 1u : 0u;
                const int tbx = tex_coord_bits(sx), tby = tex_coord_bits(sy);
                const uint32_t rel = (uint32_t)(((tby >> 8) * S + (tbx >> 8)) << 3);
                const uint32_t addr = v ? base[c] + rel : T.q_addr;
                const int2 p0 = lds_int2(addr), p1 = lds_int2(addr + (uint32_t)S * 8u);
                const float s = __fsub_rn(tex_blend(tbx, tby, p0, p1), sh);
                const float wv = v ? w : 0.0f;
                const float wrv = v ? wr : 0.0f;
                const float ws = __fmul_rn(wv, s);
                sr[c]  = __fmaf_rn(wv, rvs, sr[c]);
                srr[c] = __fmaf_rn(wrv, rvs, srr[c]);
                ss[c]  = __fmaf_rn(wv, s, ss[c]);
                sss[c] = __fmaf_rn(ws, s, sss[c]);
                srs[c] = __fmaf_rn(wrv, s, srs[c]);
                sw[c]  = __fadd_rn(sw[c], wv);
                if (BLUR) {
                    const uint32_t baddr = v ? bbase[c] + rel : T.qb_addr;
                    const int2 b0 = lds_int2(baddr), b1 = lds_int2(baddr + (uint32_t)S * 8u);
                    const float sb = tex_blend(tbx, tby, b0, b1);
                    bsx[c] = __fadd_rn(bsx[c], v ? rb : 0.0f);
                    bsy[c] = __fadd_rn(bsy[c], v ? __fdiv_rn(sb, 255.0f) : 0.0f);
                }
            }
        }
    }
#pragma unroll
    for (int c = 0; c < KCH; ++c) {
        float v = kCostMax;
        if (okc[c] && sw[c] > 1e-6f) {
            const float inv = __fdiv_rn(1.0f, sw[c]);
            const float m_r = __fmul_rn(sr[c], inv), m_rr = __fmul_rn(srr[c], inv);
            const float m_s = __fmul_rn(ss[c], inv), m_ss = __fmul_rn(sss[c], inv);
            const float m_rs = __fmul_rn(srs[c], inv);
            const float var_r = __fmaf_rn(-m_r, m_r, m_rr);
            const float var_s = __fmaf_rn(-m_s, m_s, m_ss);
            if (!(var_r < 1e-5f || var_s < 1e-5f)) {
                const float cov = __fmaf_rn(-m_r, m_s, m_rs);
                const float vv = __fsqrt_rn(__fmul_rn(var_r, var_s));
                v = clamp_cost(__fsub_rn(1.0f, __fdiv_rn(cov, vv)));
            }
        }
        if (BLUR) {
            const float tb = __fsub_rn(bsx[c], bsy[c]);
            const float bw = pfd_expf(__fmul_rn(__fmul_rn(-0.007368f, tb), tb));
            v = clamp_cost(__fmaf_rn(P.blur_gain, __fsub_rn(1.0f, bw), v));
        }
        cost[c] = v;
    }
}

// ComputeMultiViewCostVector_Frame (AdaptMIPMFrame.cu:181-225) for the plane of
// every lane of the warp; must be called by all 32 lanes together.  Lanes with
// active == false only keep the warp company.  Cost of neighbour k (k < nc)
// goes to out[k * out_stride]; neighbours whose anchor leaves the window for
// every lane are not evaluated (their cost is 2, as the reference returns).
template <bool BLUR, bool COUNT>
__device__ __noinline__ void cost_vector(const Tiles& T, const PmParams& P, int px, int py, bool active,
                                            float4 h, int nc, float* out, int out_stride)
{
    if (!active) h = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    const float3 dp = disparity_plane(px, py, h);
    const float d0 = to_disparity(px, py, dp);
    uint32_t okmask = 0;
    for (int k = 0; k < nc; ++k) {
        const float2 a = geo_anchor(T.geo[k], px, py, d0);
        const bool ok = active && T.nb_ok[k] && (__float_as_uint(a.x) < P.W_bits) && (__float_as_uint(a.y) < P.H_bits);
        okmask |= ok ? (1u << k) : 0u;
    }
    uint32_t todo = __reduce_or_sync(kFullMask, okmask);
    unsigned ntaps = 0;
    for (int k = 0; k < nc; ++k)
        if (!((todo >> k) & 1u)) out[k * out_stride] = kCostMax;
    while (todo) {
        int ks[16];
        int nks = 0;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            ks[c] = todo ? (__ffs(todo) - 1) : 0;
            if (todo) { ++nks; todo &= todo - 1; }
        }
        if (nks > 4) {
            float c6[6];
            ncc_chunk<6, BLUR, COUNT>(T, P, px, py, dp, ks, nks, okmask, c6, ntaps);
#pragma unroll
            for (int c = 0; c < 6; ++c) if (c < nks) out[ks[c] * out_stride] = c6[c];
        } else {
            float c4[4];
            ncc_chunk<4, BLUR, COUNT>(T, P, px, py, dp, ks, nks, okmask, c4, ntaps);
#pragma unroll
            for (int c = 0; c < 4; ++c) if (c < nks) out[ks[c] * out_stride] = c4[c];
        }
    }
    if (COUNT) {
        const unsigned tot = __reduce_add_sync(kFullMask, ntaps);
        if ((threadIdx.x & 31) == 0 && tot) atomicAdd(P.tap_counter, (unsigned long long)tot);
    }
}

// ComputeWeightedCost_Frame (AdaptMIPMFrame.cu:284-317), streamed: call add(k,
// c) for k = 0..nc-1 in order, then result().
struct WeightedCost {
    float norm, total, min_cost;
    int min_idx;
    __device__ __forceinline__ WeightedCost() : norm(0.0f), total(0.0f), min_cost(2.0f), min_idx(-1) {}
    __device__ __forceinline__ void add(int k, float c, float w)
    {
        if (w > 0.0f) { norm = __fadd_rn(norm, w); total = __fmaf_rn(w, c, total); }
        if (c < min_cost) { min_cost = c; min_idx = k; }
    }
    __device__ __forceinline__ float result() const { return (norm <= 1e-6f) ? 2.0f : __fdiv_rn(total, norm); }
};

}  // namespace pfd
