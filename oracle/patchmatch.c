/*
 * oracle/patchmatch.c -- CPU restatement of the reference's whole-frame
 * plane-hypothesis PatchMatch (AdaptMIPMFrame).  TEST INFRASTRUCTURE ONLY;
 * see pfd_oracle.h for who may call it and how it is pinned to the
 * reference's own kernels.
 *
 * Structure and order of operations follow the reference line by line:
 *   MIStereo/AdaptMIPMFrame.cu:24-947, MIStereo/CudaUtil.cu:13-170,341-361,491-507,
 *   MIStereo/AdaptMIPMUtil.cu:463-501,625-649.
 * Arithmetic follows oracle/canon.h.  Deliberate, documented deviations from
 * the reference (each marked DEVIATION below):
 *   - NaN coordinates make a tap / anchor / proxy invalid (the reference passes
 *     NaN through tex2D, whose result is unspecified);
 *   - the perturbed-normal candidate keeps the current disparity in .w
 *     (GeneratePerturbedNormalLF leaves .w uninitialised, CudaUtil.cu:132-141);
 *   - the Marsaglia rejection loop gives up after 64 rejected pairs (probability
 *     ~1e-43) and returns the +z normal;
 *   - random numbers come from Philox4x32-10 streams instead of cuRAND seeded
 *     from clock64() (AdaptMIPMFrame.cu:501).
 */
#include "pfd_oracle.h"
#include "canon.h"

#include <float.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float x, y, z, w; } f4;
typedef struct { float x, y, z; } f3;

#define COST_MAX 2.0f
#define MAX_NB 32

static inline f4 mk4(float x, float y, float z, float w) { f4 r = { x, y, z, w }; return r; }
static inline f4 ld4(const float* a, long i) { return mk4(a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]); }
static inline void st4(float* a, long i, f4 v) { a[4 * i] = v.x; a[4 * i + 1] = v.y; a[4 * i + 2] = v.z; a[4 * i + 3] = v.w; }

/* AdaptMIPMFrame.cu:24-27 */
static inline float clamp_cost(float v) { return fminf(2.0f, fmaxf(0.0f, v)); }

/* AdaptMIPMFrame.cu:29-34 */
static inline float safe_denom(float v)
{
    if (fabsf(v) < 1e-6f) return (v >= 0.0f) ? 1e-6f : -1e-6f;
    return v;
}

/* CudaUtil.cu:13-21 */
static inline void set_bit(uint32_t* m, int n) { *m |= (uint32_t)(1u << n); }
static inline int is_set(uint32_t m, int n) { return (int)((m >> n) & 1u); }

/* DisparityPlane, CudaUtil.cu:158-170: plane (n, d at p) -> disparity plane A x + B y + C. */
static inline f3 disparity_plane(int px, int py, f4 h)
{
    f3 d;
    d.x = -h.x / h.z;
    d.y = -h.y / h.z;
    float num = fmaf(h.y, (float)py, h.x * (float)px);
    num = fmaf(h.z, h.w, num);
    d.z = num / h.z;
    return d;
}

/* to_disparity CudaUtil.cu:152-156 and EvalDisparityAtPixel_Frame AdaptMIPMFrame.cu:55-60 */
static inline float to_disparity(int px, int py, f3 dp)
{
    return fmaf(dp.y, (float)py, dp.x * (float)px) + dp.z;
}

/* NormalizeVec3, CudaUtil.cu:49-56 */
static inline f4 normalize3(f4 v)
{
    const float n2 = fmaf(v.z, v.z, fmaf(v.y, v.y, v.x * v.x));
    const float inv = canon_rsqrtf(n2);
    v.x *= inv; v.y *= inv; v.z *= inv;
    return v;
}

/* DisparityGeometricMapOperate_Hex, AdaptMIPMUtil.cu:625-649. */
static inline void geo_map_hex(const float* c0, const float* c1, int pfx, int pfy, f4 h, int p0x, int p0y,
                               float base, float* p1x, float* p1y, f4* disp)
{
    const f3 dp = disparity_plane(pfx, pfy, h);
    const float d = to_disparity(p0x, p0y, dp);
    const float ey = c1[1] - c0[1], ex = c1[0] - c0[0];
    const float baseline = sqrtf(fmaf(ex, ex, ey * ey));
    const float bx = c0[0] - c1[0], by = c0[1] - c1[1];
    const float dxn = bx / baseline, dyn = by / baseline;
    const float scale = baseline / base;
    *p1x = fmaf(dxn * d, scale, (float)p0x);
    *p1y = fmaf(dyn * d, scale, (float)p0y);
    const float dr2 = fmaf(by, (float)p0y - *p1y, bx * ((float)p0x - *p1x));
    const float d_real = sqrtf(dr2);
    disp->x = d;
    disp->y = d_real;
    disp->z = baseline;
    disp->w = (float)((double)baseline / ((double)d_real + 1e-7));
}

/* ComputeBilateralNCC_Frame, AdaptMIPMFrame.cu:73-179, with ComputeBilateralWeight
 * CudaUtil.cu:145-150.  Loop order: i = x offset outer, j = y offset inner. */
static float ncc_frame(const orc_frame* f, const orc_params* p, int vid, int nvid, int px, int py, f4 h,
                       float* blur_x, float* blur_y, f4* disp, long long* taps)
{
    const int W = f->mi_w, H = f->mi_h;
    const long ppv = (long)W * H;
    const float* R = f->gray + (long)vid * ppv;
    const float* S = f->gray + (long)nvid * ppv;
    const float* RB = f->blur ? f->blur + (long)vid * ppv : NULL;
    const float* SB = f->blur ? f->blur + (long)nvid * ppv : NULL;
    const float* c0 = f->centers + 2 * vid;
    const float* c1 = f->centers + 2 * nvid;
    const int radius = p->patch_size / 2;

    *blur_x = 0.0f; *blur_y = 0.0f;
    float ax, ay;
    geo_map_hex(c0, c1, px, py, h, px, py, p->base, &ax, &ay, disp);
    /* DEVIATION: a NaN anchor is out of bounds */
    if (!(ax >= 0.0f && ax < (float)W && ay >= 0.0f && ay < (float)H)) return COST_MAX;

    const f3 dp = disparity_plane(px, py, h);
    const float inv_base = 1.0f / fmaxf(p->base, 1e-6f);
    const float stx = (c0[0] - c1[0]) * inv_base;
    const float sty = (c0[1] - c1[1]) * inv_base;

    float s_r = 0.0f, s_rr = 0.0f, s_s = 0.0f, s_ss = 0.0f, s_rs = 0.0f, s_w = 0.0f;
    const float rc = R[py * W + px];
    /* shifted moments (not in the reference): texels and samples minus the
     * centre texel, exact subtractions; shift 0 is the reference's sums */
    const float sh = p->shifted ? rc : 0.0f;
    const float ss2 = (2.0f * p->sigma_spatial) * p->sigma_spatial;
    const float cc2 = (2.0f * p->sigma_color) * p->sigma_color;

    for (int i = -radius; i <= radius; i += p->radius_increment) {
        for (int j = -radius; j <= radius; j += p->radius_increment) {
            const int xr = px + i, yr = py + j;
            if (xr < 0 || xr >= W || yr < 0 || yr >= H) continue;
            const float d = fmaf(dp.y, (float)yr, dp.x * (float)xr) + dp.z;
            const float sx = fmaf(stx, d, (float)xr);
            const float sy = fmaf(sty, d, (float)yr);
            /* DEVIATION: NaN source coordinates are out of bounds */
            if (!(sx >= 0.0f && sx < (float)W && sy >= 0.0f && sy < (float)H)) continue;
            if (taps) ++*taps;
            const float r = R[yr * W + xr];
            const float s = canon_tex_fetch(S, W, H, sx, sy) - sh;
            if (RB) {
                *blur_x += RB[yr * W + xr] / 255.0f;
                *blur_y += canon_tex_fetch(SB, W, H, sx, sy) / 255.0f;
            }
            const float fi = (float)i, fj = (float)j;
            const float sd = sqrtf(fmaf(fj, fj, fi * fi));
            const float cd = fabsf(r - rc);
            const float w = canon_expf((-sd) / ss2 - cd / cc2);
            const float rs = r - sh;
            const float wr = w * rs;
            const float ws = w * s;
            s_r  = fmaf(w, rs, s_r);
            s_rr = fmaf(wr, rs, s_rr);
            s_s  = fmaf(w, s, s_s);
            s_ss = fmaf(ws, s, s_ss);
            s_rs = fmaf(wr, s, s_rs);
            s_w  = s_w + w;
        }
    }
    if (s_w <= 1e-6f) return COST_MAX;
    const float inv = 1.0f / s_w;
    const float m_r = s_r * inv, m_rr = s_rr * inv, m_s = s_s * inv, m_ss = s_ss * inv, m_rs = s_rs * inv;
    const float var_r = fmaf(-m_r, m_r, m_rr);
    const float var_s = fmaf(-m_s, m_s, m_ss);
    if (var_r < 1e-5f || var_s < 1e-5f) return COST_MAX;
    const float cov = fmaf(-m_r, m_s, m_rs);
    const float vv = sqrtf(var_r * var_s);
    return clamp_cost(1.0f - cov / vv);
}

/* ComputeMultiViewCostVector_Frame, AdaptMIPMFrame.cu:181-225 (blur_vector is
 * never read downstream and is not kept). */
static void cost_vector(const orc_frame* f, const orc_params* p, int vid, int px, int py, f4 h,
                        float* cv, f4* dv, long long* taps)
{
    for (int i = 0; i < MAX_NB; ++i) { cv[i] = 2.0f; dv[i] = mk4(0, 0, 0, 0); }
    const int nc = f->nb_counts[vid];
    for (int k = 0; k < nc && k < f->max_nb; ++k) {
        const int nvid = f->nb_ids[vid * f->max_nb + k];
        if (nvid < 0) continue;
        float bx, by;
        f4 db = mk4(0, 0, 0, 0);
        float c = ncc_frame(f, p, vid, nvid, px, py, h, &bx, &by, &db, taps);
        const float t = bx - by;
        const float bw = canon_expf((-0.007368f * t) * t);
        /* blur penalty gain: 2 in the Frame matcher, 0.8 in the ACMM one
         * (AdaptMIPMFrameACMM.cu:99) */
        c = clamp_cost(fmaf(p->acmm ? 0.8f : 2.0f, 1.0f - bw, c));
        cv[k] = c;
        dv[k] = db;
    }
}

/* ComputeSelectedViewsTopK_Frame, AdaptMIPMFrame.cu:227-282 */
static uint32_t topk_views(const float* cv, int nc, int top_k, float* mean_cost, int* best_idx)
{
    *best_idx = -1;
    int valid = 0;
    for (int i = 0; i < nc; ++i) {
        if (cv[i] < 2.0f) {
            ++valid;
            if (*best_idx < 0 || cv[i] < cv[*best_idx]) *best_idx = i;
        }
    }
    if (valid <= 0) { *mean_cost = 2.0f; return 0; }
    const int k = valid < top_k ? valid : top_k;
    float tmp[MAX_NB];
    for (int i = 0; i < nc; ++i) tmp[i] = cv[i];
    for (int i = nc; i < MAX_NB; ++i) tmp[i] = 2.0f;
    for (int i = 0; i < k; ++i)
        for (int j = i + 1; j < nc; ++j)
            if (tmp[j] < tmp[i]) { const float t = tmp[i]; tmp[i] = tmp[j]; tmp[j] = t; }
    float m = 0.0f;
    for (int i = 0; i < k; ++i) m += tmp[i];
    m /= (float)k;
    *mean_cost = m;
    const float thr = tmp[k - 1];
    uint32_t mask = 0;
    for (int i = 0; i < nc && i < 32; ++i)
        if (cv[i] <= thr) set_bit(&mask, i);
    return mask;
}

/* ComputeWeightedCost_Frame, AdaptMIPMFrame.cu:284-317 */
static float weighted_cost(const float* cv, const float* vw, int nc, const f4* dv, f4* best_disp)
{
    float norm = 0.0f, total = 0.0f, min_cost = 2.0f;
    int min_idx = -1;
    for (int i = 0; i < nc; ++i) {
        if (vw[i] > 0.0f) {
            norm += vw[i];
            total = fmaf(vw[i], cv[i], total);
        }
        if (cv[i] < min_cost) { min_cost = cv[i]; min_idx = i; }
    }
    *best_disp = (min_idx >= 0) ? dv[min_idx] : mk4(0, 0, 0, 0);
    if (norm <= 1e-6f) return 2.0f;
    return total / norm;
}

/* GenerateRandomNormal_MIPM AdaptMIPMUtil.cu:463-492 == GenerateRandomNormalLF CudaUtil.cu:341-361 */
static f4 random_normal(canon_rng* g)
{
    float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
    int attempts = 0;
    while (s >= 1.0f) {
        if (attempts++ == 64) { q1 = 0.0f; q2 = 0.0f; s = 0.0f; break; }   /* DEVIATION: bounded */
        q1 = fmaf(2.0f, canon_uniform(g), -1.0f);
        q2 = fmaf(2.0f, canon_uniform(g), -1.0f);
        s = fmaf(q2, q2, q1 * q1);
    }
    const float sq = sqrtf(1.0f - s);
    f4 n = mk4((2.0f * q1) * sq, (2.0f * q2) * sq, fmaf(-2.0f, s, 1.0f), 0.0f);
    return normalize3(n);
}

/* GenerateRandomPlaneHypothesis_MIPM, AdaptMIPMUtil.cu:494-501 */
static f4 random_plane(canon_rng* g, float dmin, float dmax)
{
    const float depth = fmaf(canon_uniform(g), dmax - dmin, dmin);
    f4 h = random_normal(g);
    h.w = depth;
    return h;
}

/* GeneratePerturbedNormalLF, CudaUtil.cu:105-142 with GetViewDirectionLF :58-72 */
static f4 perturbed_normal(int px, int py, f4 n, canon_rng* g, float pert)
{
    const float X0 = (float)px, X1 = (float)py, X2 = 1.0f;
    const float norm = sqrtf(fmaf(X2, X2, fmaf(X1, X1, X0 * X0)));
    const float vx = X0 / norm, vy = X1 / norm, vz = X2 / norm;

    const float a1 = (canon_uniform(g) - 0.5f) * pert;
    const float a2 = (canon_uniform(g) - 0.5f) * pert;
    const float a3 = (canon_uniform(g) - 0.5f) * pert;
    const float s1 = canon_sin_small(a1), s2 = canon_sin_small(a2), s3 = canon_sin_small(a3);
    const float c1 = canon_cos_small(a1), c2 = canon_cos_small(a2), c3 = canon_cos_small(a3);
    float R[9];
    R[0] = c2 * c3;
    R[1] = fmaf(-c1, s3, (c3 * s1) * s2);
    R[2] = fmaf(c1 * c3, s2, s1 * s3);
    R[3] = c2 * s3;
    R[4] = fmaf(s1 * s2, s3, c1 * c3);
    R[5] = fmaf(-c3, s1, (c1 * s2) * s3);
    R[6] = -s2;
    R[7] = c2 * s1;
    R[8] = c1 * c2;
    f4 q;
    q.x = fmaf(R[2], n.z, fmaf(R[1], n.y, R[0] * n.x));
    q.y = fmaf(R[5], n.z, fmaf(R[4], n.y, R[3] * n.x));
    q.z = fmaf(R[8], n.z, fmaf(R[7], n.y, R[6] * n.x));
    q.w = n.w;                                            /* DEVIATION: keeps .w */
    const float dot = fmaf(q.z, vz, fmaf(q.y, vy, q.x * vx));
    if (dot >= 0.0f) q = n;
    return normalize3(q);
}

/* EncodePlaneHypothesisFromDispPlaneDevice, AdaptMIPMFrame.cu:36-53 */
static f4 encode_plane(int ax, int ay, float alpha, float beta, float gamma)
{
    float nx = -alpha, ny = -beta, nz = 1.0f;
    const float inv = canon_rsqrtf(fmaf(nz, nz, fmaf(ny, ny, nx * nx)) + 1e-12f);
    nx *= inv; ny *= inv; nz *= inv;
    const float d = fmaf(beta, (float)ay, alpha * (float)ax) + gamma;
    return mk4(nx, ny, nz, d);
}

/* BuildCrossViewPlaneProposal, AdaptMIPMFrame.cu:350-398 */
static int cross_view_proposal(const orc_frame* f, const orc_params* p, const float* plane_prev,
                               int vid, int nvid, int px, int py, f4 cur, f4* out)
{
    const int W = f->mi_w, H = f->mi_h;
    const long ppv = (long)W * H;
    const float* cr = f->centers + 2 * vid;
    const float* cn = f->centers + 2 * nvid;
    float qfx, qfy;
    f4 tmp;
    geo_map_hex(cr, cn, px, py, cur, px, py, p->base, &qfx, &qfy, &tmp);
    const float fx = floorf(qfx + 0.5f), fy = floorf(qfy + 0.5f);
    /* DEVIATION: NaN is out of bounds (the float test equals the reference's
     * integer test for every finite value) */
    if (!(fx >= 0.0f && fx < (float)W && fy >= 0.0f && fy < (float)H)) return 0;
    const int qx = (int)fx, qy = (int)fy;
    const f4 hn = ld4(plane_prev, (long)nvid * ppv + qy * W + qx);
    const f3 dp = disparity_plane(qx, qy, hn);
    const float du = cr[0] - cn[0], dv = cr[1] - cn[1];
    float denom = fmaf(dp.y, dv, fmaf(dp.x, du, 1.0f));
    denom = safe_denom(denom);
    *out = encode_plane(px, py, dp.x / denom, dp.y / denom, dp.z / denom);
    return 1;
}

/* PlaneHypothesisRefinement_Frame, AdaptMIPMFrame.cu:400-471 */
static void refine(const orc_frame* f, const orc_params* p, int vid, int px, int py, canon_rng* g,
                   const float* vw, f4* best_plane, float* best_cost, f4* best_disp, long long* taps)
{
    const int nc = f->nb_counts[vid];
    if (nc <= 0) return;
    const float pert = 0.02f;
    const float depth_now = best_plane->w;
    float depth_rand;
    if (*best_cost < 0.1f) depth_rand = fmaf(canon_uniform(g) - 0.5f, 2.0f, depth_now);
    else depth_rand = fmaf(canon_uniform(g), p->depth_max - p->depth_min, p->depth_min);
    (void)depth_rand;                               /* drawn but unused, as in the reference */
    const f4 rn = random_normal(g);
    const float pert_pi = (float)((double)pert * 3.14159265358979323846);
    const f4 pn = perturbed_normal(px, py, *best_plane, g, pert_pi);
    const float dmin_p = (1.0f - pert) * depth_now;
    const float dmax_p = (1.0f + pert) * depth_now;
    const float depth_perturbed = fmaf(canon_uniform(g), dmax_p - dmin_p, dmin_p);

    f4 cand[5];
    cand[0] = random_plane(g, p->depth_min, p->depth_max);
    cand[1] = rn;
    cand[2] = pn;
    cand[3] = *best_plane;
    cand[4] = *best_plane;
    cand[4].w = depth_perturbed;
    for (int i = 1; i < 5; ++i) {
        const f3 dp = disparity_plane(px, py, cand[i]);
        cand[i].w = to_disparity(px, py, dp);
    }
    for (int i = 0; i < 5; ++i) {
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vid, px, py, cand[i], cv, dv, taps);
        f4 td;
        const float c = weighted_cost(cv, vw, nc, dv, &td);
        if (c < *best_cost) { *best_cost = c; *best_plane = cand[i]; *best_disp = td; }
    }
}

static void init_pixel(const orc_frame* f, const orc_params* p, uint64_t seed, int vid, int x, int y,
                       orc_state* out)
{
    const int W = f->mi_w;
    const long ppv = (long)W * f->mi_h;
    const long idx = (long)vid * ppv + (long)y * W + x;
    canon_rng g;
    canon_rng_init(&g, seed, 0u, (uint32_t)idx);
    const f4 h = random_plane(&g, p->depth_min, p->depth_max);
    float cv[MAX_NB];
    f4 dv[MAX_NB];
    cost_vector(f, p, vid, x, y, h, cv, dv, NULL);
    float mean = 2.0f;
    int bi = -1;
    const uint32_t sel = topk_views(cv, f->nb_counts[vid], p->top_k, &mean, &bi);
    st4(out->plane, idx, h);
    out->cost[idx] = mean;
    st4(out->disp, idx, bi >= 0 ? dv[bi] : mk4(0, 0, 0, 0));
    out->sel[idx] = sel;
}

static void copy_pixel(const orc_state* a, orc_state* b, long idx)
{
    memcpy(b->plane + 4 * idx, a->plane + 4 * idx, 16);
    b->cost[idx] = a->cost[idx];
    memcpy(b->disp + 4 * idx, a->disp + 4 * idx, 16);
    b->sel[idx] = a->sel[idx];
}

/* Scan for the lowest-cost sample along one direction (AdaptMIPMFrame.cu:604-795). */
#define PREV_COST(pos) (prev->cost[(long)vid * ppv + (pos)])

/* CheckerboardUpdateFrame, AdaptMIPMFrame.cu:520-947, for one pixel. */
static void update_pixel(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                         int vid, int x, int y, const orc_state* prev, orc_state* next, long long* taps)
{
    const int width = f->mi_w, height = f->mi_h;
    const long ppv = (long)width * height;
    const long idx = (long)vid * ppv + (long)y * width + x;

    if (((x + y) & 1) != phase) { copy_pixel(prev, next, idx); return; }
    const int nc = f->nb_counts[vid];
    if (nc <= 0) { copy_pixel(prev, next, idx); return; }

    canon_rng g;
    canon_rng_init(&g, seed, (uint32_t)(1 + 2 * iter + phase), (uint32_t)idx);

    static const f4 zero4 = { 0, 0, 0, 0 };
    float cost_array[8][MAX_NB];
    f4 disp_array[8][MAX_NB];
    int flag[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
    int positions[8];
    for (int a = 0; a < 8; ++a) {
        positions[a] = (int)idx;
        for (int b = 0; b < MAX_NB; ++b) { cost_array[a][b] = 2.0f; disp_array[a][b] = zero4; }
    }
    const int farDis = 2, nerDis = 2;
    const int center = y * width + x;
    int left_near = center - 1, left_far = center - 3;
    int right_near = center + 1, right_far = center + 3;
    int up_near = center - width, up_far = center - 3 * width;
    int down_near = center + width, down_far = center + 3 * width;
    float costMin;
    int costMinPoint;
    const float* PP = prev->plane;
#define CAND(slot, pos) cost_vector(f, p, vid, x, y, ld4(PP, (long)vid * ppv + (pos)), cost_array[slot], disp_array[slot], taps)

    if (y > 2) {
        flag[1] = 1;
        costMin = PREV_COST(up_far); costMinPoint = up_far;
        for (int i = 1; i < farDis; ++i)
            if (y > 2 + i) {
                const int pt = up_far - i * width;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        up_far = costMinPoint; positions[1] = up_far;
        CAND(1, up_far);
    }
    if (y < height - 3) {
        flag[3] = 1;
        costMin = PREV_COST(down_far); costMinPoint = down_far;
        for (int i = 1; i < farDis; ++i)
            if (y < height - 3 - i) {
                const int pt = down_far + i * width;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        down_far = costMinPoint; positions[3] = down_far;
        CAND(3, down_far);
    }
    if (x > 2) {
        flag[5] = 1;
        costMin = PREV_COST(left_far); costMinPoint = left_far;
        for (int i = 1; i < farDis; ++i)
            if (x > 2 + i) {
                const int pt = left_far - i;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        left_far = costMinPoint; positions[5] = left_far;
        CAND(5, left_far);
    }
    if (x < width - 3) {
        flag[7] = 1;
        costMin = PREV_COST(right_far); costMinPoint = right_far;
        for (int i = 1; i < farDis; ++i)
            if (x < width - 3 - i) {
                const int pt = right_far + i;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        right_far = costMinPoint; positions[7] = right_far;
        CAND(7, right_far);
    }
    if (y > 0) {
        flag[0] = 1;
        costMin = PREV_COST(up_near); costMinPoint = up_near;
        for (int i = 0; i < nerDis; ++i) {
            if (y > 1 + i && x > i) {
                const int pt = up_near - (1 + i) * width - i;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
            if (y > 1 + i && x < width - 1 - i) {
                const int pt = up_near - (1 + i) * width + i;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        }
        up_near = costMinPoint; positions[0] = up_near;
        CAND(0, up_near);
    }
    if (y <= 2 && y > 0) {
        flag[1] = 1; positions[1] = up_near;
        for (int j = 0; j < MAX_NB; ++j) { cost_array[1][j] = cost_array[0][j]; disp_array[1][j] = disp_array[0][j]; }
    }
    if (y < height - 1) {
        flag[2] = 1;
        costMin = PREV_COST(down_near); costMinPoint = down_near;
        for (int i = 0; i < nerDis; ++i) {
            if (y < height - 2 - i && x > i) {
                const int pt = down_near + (1 + i) * width - i;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
            if (y < height - 2 - i && x < width - 1 - i) {
                const int pt = down_near + (1 + i) * width + i;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        }
        down_near = costMinPoint; positions[2] = down_near;
        CAND(2, down_near);
    }
    if (y >= height - 3 && y < height - 1) {
        flag[3] = 1; positions[3] = down_near;
        for (int j = 0; j < MAX_NB; ++j) { cost_array[3][j] = cost_array[2][j]; disp_array[3][j] = disp_array[2][j]; }
    }
    if (x > 0) {
        flag[4] = 1;
        costMin = PREV_COST(left_near); costMinPoint = left_near;
        for (int i = 0; i < nerDis; ++i) {
            if (x > 1 + i && y > i) {
                const int pt = left_near - (1 + i) - i * width;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
            if (x > 1 + i && y < height - 1 - i) {
                const int pt = left_near - (1 + i) + i * width;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        }
        left_near = costMinPoint; positions[4] = left_near;
        CAND(4, left_near);
    }
    if (x <= 2 && x > 0) {
        flag[5] = 1; positions[5] = left_near;
        for (int j = 0; j < MAX_NB; ++j) { cost_array[5][j] = cost_array[4][j]; disp_array[5][j] = disp_array[4][j]; }
    }
    if (x < width - 1) {
        flag[6] = 1;
        costMin = PREV_COST(right_near); costMinPoint = right_near;
        for (int i = 0; i < nerDis; ++i) {
            if (x < width - 2 - i && y > i) {
                const int pt = right_near + (1 + i) - i * width;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
            if (x < width - 2 - i && y < height - 1 - i) {
                const int pt = right_near + (1 + i) + i * width;
                if (PREV_COST(pt) < costMin) { costMin = PREV_COST(pt); costMinPoint = pt; }
            }
        }
        right_near = costMinPoint; positions[6] = right_near;
        CAND(6, right_near);
    }
    if (x >= width - 3 && x < width - 1) {
        flag[7] = 1; positions[7] = right_near;
        for (int j = 0; j < MAX_NB; ++j) { cost_array[7][j] = cost_array[6][j]; disp_array[7][j] = disp_array[6][j]; }
    }
#undef CAND

    /* view-selection priors from the four direct neighbours (AdaptMIPMFrame.cu:797-815) */
    float priors[MAX_NB];
    for (int j = 0; j < MAX_NB; ++j) priors[j] = 0.0f;
    const int direct_pos[4] = {
        (y > 0) ? (center - width) : -1,
        (y < height - 1) ? (center + width) : -1,
        (x > 0) ? (center - 1) : -1,
        (x < width - 1) ? (center + 1) : -1 };
    const int same_flags[4] = { 0, 2, 4, 6 };
    for (int ii = 0; ii < 4; ++ii) {
        if (direct_pos[ii] < 0 || !flag[same_flags[ii]]) continue;
        const uint32_t sm = prev->sel[(long)vid * ppv + direct_pos[ii]];
        for (int j = 0; j < nc; ++j) priors[j] += is_set(sm, j) == 1 ? 0.9f : 0.1f;
    }

    /* sampling probabilities (AdaptMIPMFrame.cu:817-839) */
    float probs[MAX_NB];
    for (int j = 0; j < MAX_NB; ++j) probs[j] = 0.0f;
    const float thr = 0.8f * canon_expf((float)(iter * iter) / (-90.0f));
    for (int i = 0; i < nc; ++i) {
        float count = 0.0f, tmpw = 0.0f;
        int count_false = 0;
        for (int j = 0; j < 8; ++j) {
            if (!flag[j]) continue;
            const float c = cost_array[j][i];
            if (c < thr) { tmpw += canon_expf((c * c) / (-0.18f)); count += 1.0f; }
            if (c > 1.2f) count_false++;
        }
        if (count > 2.0f && count_false < 3) probs[i] = tmpw / count;
        else if (count_false < 3) probs[i] = canon_expf((thr * thr) / (-0.32f));
        probs[i] *= priors[i];
    }
    /* TransformPDFToCDF, CudaUtil.cu:491-507 */
    {
        float sum = 0.0f;
        for (int i = 0; i < nc; ++i) sum += probs[i];
        const float inv = 1.0f / sum;
        float cum = 0.0f;
        for (int i = 0; i < nc; ++i) { cum = fmaf(probs[i], inv, cum); probs[i] = cum; }
    }
    float vw[MAX_NB];
    for (int j = 0; j < MAX_NB; ++j) vw[j] = 0.0f;
    for (int sample = 0; sample < 15; ++sample) {
        const float rp = canon_uniform(&g) - FLT_EPSILON;
        for (int id = 0; id < nc; ++id)
            if (probs[id] > rp) { vw[id] += 1.0f; break; }
    }
    uint32_t tsel = 0;
    float wn = 0.0f;
    for (int i = 0; i < nc; ++i)
        if (vw[i] > 0.0f) { set_bit(&tsel, i); wn += vw[i]; }
    if (wn <= 0.0f) {
        for (int i = 0; i < nc; ++i) { vw[i] = 1.0f; set_bit(&tsel, i); }
        wn = (float)nc;
    }

    f4 best_plane = ld4(prev->plane, idx);
    float best_cost;
    f4 best_disp;
    {
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vid, x, y, best_plane, cv, dv, taps);
        best_cost = weighted_cost(cv, vw, nc, dv, &best_disp);
    }
    for (int i = 0; i < 8; ++i) {
        if (!flag[i]) continue;
        f4 cd;
        const float c = weighted_cost(cost_array[i], vw, nc, disp_array[i], &cd);
        if (c < best_cost) {
            best_cost = c;
            best_plane = ld4(prev->plane, (long)vid * ppv + positions[i]);
            best_disp = cd;
        }
    }
    for (int k = 0; k < nc && k < f->max_nb; ++k) {
        if (is_set(tsel, k) == 0) continue;
        const int nvid = f->nb_ids[vid * f->max_nb + k];
        if (nvid < 0) continue;
        f4 proxy;
        if (!cross_view_proposal(f, p, prev->plane, vid, nvid, x, y, best_plane, &proxy)) continue;
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vid, x, y, proxy, cv, dv, taps);
        f4 pd;
        const float c = weighted_cost(cv, vw, nc, dv, &pd);
        if (c < best_cost) { best_cost = c; best_plane = proxy; best_disp = pd; }
    }
    refine(f, p, vid, x, y, &g, vw, &best_plane, &best_cost, &best_disp, taps);

    if (p->acmm) {
        /* ACMM write-back (AdaptMIPMFrameACMM.cu:880-900): DetailRestorer_FrameACMM
         * returns at once without a warm start; RecomputeSupportCostDisp_Frame
         * (:259-280) evaluates the final plane on every view and stores the
         * top-k mean, the top-k view mask and the lowest-cost view's disp */
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vid, x, y, best_plane, cv, dv, taps);
        int bi = -1;
        tsel = topk_views(cv, nc, p->top_k, &best_cost, &bi);
        best_disp = bi >= 0 ? dv[bi] : mk4(0, 0, 0, 0);
    }
    st4(next->plane, idx, best_plane);
    next->cost[idx] = best_cost;
    st4(next->disp, idx, best_disp);
    next->sel[idx] = tsel;
}
#undef PREV_COST

/* ------------------------------------------------------------------------ */

int orc_cost_vectors(const orc_frame* f, const orc_params* p, const int* vids, const int* pxy,
                     const float* planes, int n, float* costs, float* disps)
{
    if (!f || !p || f->max_nb > MAX_NB) return -1;
    for (int i = 0; i < n; ++i) {
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vids[i], pxy[2 * i], pxy[2 * i + 1], ld4(planes, i), cv, dv, NULL);
        for (int k = 0; k < f->max_nb; ++k) {
            costs[(long)i * f->max_nb + k] = cv[k];
            if (disps) st4(disps, (long)i * f->max_nb + k, dv[k]);
        }
    }
    return 0;
}

long long orc_count_taps(const orc_frame* f, const orc_params* p, const int* vids, const int* pxy,
                         const float* planes, int n)
{
    long long taps = 0;
    for (int i = 0; i < n; ++i) {
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vids[i], pxy[2 * i], pxy[2 * i + 1], ld4(planes, i), cv, dv, &taps);
    }
    return taps;
}

int orc_pm_init_views(const orc_frame* f, const orc_params* p, uint64_t seed, orc_state* out, int v0, int v1,
                      int nthreads)
{
    if (!f || !p || f->max_nb > MAX_NB) return -1;
    const int W = f->mi_w, H = f->mi_h;
    const long t0 = (long)v0 * W * H, t1 = (long)v1 * W * H;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long t = t0; t < t1; ++t) {
        const int vid = (int)(t / ((long)W * H));
        const int rem = (int)(t % ((long)W * H));
        init_pixel(f, p, seed, vid, rem % W, rem / W, out);
    }
    (void)nthreads;
    return 0;
}

int orc_pm_init(const orc_frame* f, const orc_params* p, uint64_t seed, orc_state* out, int nthreads)
{
    return orc_pm_init_views(f, p, seed, out, 0, f->n_views, nthreads);
}

int orc_pm_sweep_views(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                       const orc_state* prev, orc_state* next, int v0, int v1, int nthreads)
{
    if (!f || !p || f->max_nb > MAX_NB) return -1;
    const int W = f->mi_w, H = f->mi_h;
    const long ppv = (long)W * H;
    const long t0 = (long)v0 * ppv, t1 = (long)v1 * ppv;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (long t = t0; t < t1; ++t) {
        const int vid = (int)(t / ppv);
        const int rem = (int)(t % ppv);
        update_pixel(f, p, seed, iter, phase, vid, rem % W, rem / W, prev, next, NULL);
    }
    (void)nthreads;
    return 0;
}

long long orc_pm_sweep_views_taps(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                                  const orc_state* prev, orc_state* next, int v0, int v1, int nthreads)
{
    if (!f || !p || f->max_nb > MAX_NB) return -1;
    const long ppv = (long)f->mi_w * f->mi_h;
    const long t0 = (long)v0 * ppv, t1 = (long)v1 * ppv;
    long long taps = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) reduction(+ : taps)
#endif
    for (long t = t0; t < t1; ++t) {
        long long mine = 0;
        const int vid = (int)(t / ppv);
        const int rem = (int)(t % ppv);
        update_pixel(f, p, seed, iter, phase, vid, rem % f->mi_w, rem / f->mi_w, prev, next, &mine);
        taps += mine;
    }
    (void)nthreads;
    return taps;
}

long long orc_pm_sweep_taps(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                            const orc_state* prev, orc_state* next, int nthreads)
{
    return orc_pm_sweep_views_taps(f, p, seed, iter, phase, prev, next, 0, f->n_views, nthreads);
}

int orc_pm_sweep(const orc_frame* f, const orc_params* p, uint64_t seed, int iter, int phase,
                 const orc_state* prev, orc_state* next, int nthreads)
{
    return orc_pm_sweep_views(f, p, seed, iter, phase, prev, next, 0, f->n_views, nthreads);
}

int orc_patchmatch(const orc_frame* f, const orc_params* p, uint64_t seed, orc_state* out, int nthreads)
{
    const long total = (long)f->n_views * f->mi_w * f->mi_h;
    orc_state tmp;
    tmp.plane = (float*)malloc(sizeof(float) * 4 * total);
    tmp.cost = (float*)malloc(sizeof(float) * total);
    tmp.disp = (float*)malloc(sizeof(float) * 4 * total);
    tmp.sel = (uint32_t*)malloc(sizeof(uint32_t) * total);
    if (!tmp.plane || !tmp.cost || !tmp.disp || !tmp.sel) {
        free(tmp.plane); free(tmp.cost); free(tmp.disp); free(tmp.sel);
        return -2;
    }
    int rc = orc_pm_init(f, p, seed, out, nthreads);
    orc_state* a = out;
    orc_state* b = &tmp;
    for (int it = 0; rc == 0 && it < p->max_iterations; ++it) {
        for (int ph = 0; ph < 2 && rc == 0; ++ph) {
            rc = orc_pm_sweep(f, p, seed, it, ph, a, b, nthreads);
            orc_state* s = a; a = b; b = s;
        }
    }
    /* an even number of half-sweeps leaves the result in out */
    free(tmp.plane); free(tmp.cost); free(tmp.disp); free(tmp.sel);
    if (rc == 0 && p->acmm) rc = orc_acmm_post_refine(f, p, out, nthreads);
    return rc;
}

/* PostRefineMetadataFrame (AdaptMIPMFrameACMM.cu:903-929): cost, selected views
 * and disp of every pixel recomputed from its plane (RecomputeSupportCostDisp_Frame). */
int orc_acmm_post_refine(const orc_frame* f, const orc_params* p, orc_state* st, int nthreads)
{
    if (!f || !p || f->max_nb > MAX_NB) return -1;
    const int W = f->mi_w;
    const long ppv = (long)W * f->mi_h, total = ppv * f->n_views;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long t = 0; t < total; ++t) {
        const int vid = (int)(t / ppv), rem = (int)(t % ppv);
        float cv[MAX_NB];
        f4 dv[MAX_NB];
        cost_vector(f, p, vid, rem % W, rem / W, ld4(st->plane, t), cv, dv, NULL);
        float mean = 2.0f;
        int bi = -1;
        st->sel[t] = topk_views(cv, f->nb_counts[vid], p->top_k, &mean, &bi);
        st->cost[t] = mean;
        st4(st->disp, t, bi >= 0 ? dv[bi] : mk4(0, 0, 0, 0));
    }
    (void)nthreads;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FP64 NCC with exact bilinear sampling (the precision oracle). */
static double tex_exact(const float* img, int W, int H, double sx, double sy)
{
    const double fx0 = floor(sx), fy0 = floor(sy);
    int ix = (int)fx0, iy = (int)fy0;
    const double ax = sx - fx0, ay = sy - fy0;
    int ix1 = ix + 1, iy1 = iy + 1;
    if (ix < 0) ix = 0; if (ix > W - 1) ix = W - 1;
    if (iy < 0) iy = 0; if (iy > H - 1) iy = H - 1;
    if (ix1 > W - 1) ix1 = W - 1;
    if (iy1 > H - 1) iy1 = H - 1;
    const double t00 = img[iy * W + ix], t10 = img[iy * W + ix1], t01 = img[iy1 * W + ix], t11 = img[iy1 * W + ix1];
    return (1 - ax) * (1 - ay) * t00 + ax * (1 - ay) * t10 + (1 - ax) * ay * t01 + ax * ay * t11;
}

/* The texture's own sampling in double: the sample point rounded to 1/256 of a
 * texel and the 8-bit bilinear weights of canon_tex_fetch, so the only
 * difference from the device is the arithmetic. */
static double tex_quantised(const float* img, int W, int H, double sx, double sy)
{
    const int qx = (int)floor((sx + 0.5) * 256.0 - 127.5);
    const int qy = (int)floor((sy + 0.5) * 256.0 - 127.5);
    int ix = qx >> 8, iy = qy >> 8;
    const int a = qx & 255, b = qy & 255;
    int ix1 = ix + 1, iy1 = iy + 1;
    if (ix < 0) ix = 0; if (ix > W - 1) ix = W - 1;
    if (iy < 0) iy = 0; if (iy > H - 1) iy = H - 1;
    if (ix1 < 0) ix1 = 0; if (ix1 > W - 1) ix1 = W - 1;
    if (iy1 < 0) iy1 = 0; if (iy1 > H - 1) iy1 = H - 1;
    const int w11 = (a * b + 128) >> 8;
    const int w10 = a - w11, w01 = b - w11, w00 = 256 - a - b + w11;
    return (w00 * (double)img[iy * W + ix] + w10 * (double)img[iy * W + ix1] + w01 * (double)img[iy1 * W + ix] +
            w11 * (double)img[iy1 * W + ix1]) / 256.0;
}

static double ncc_fp64(const orc_frame* f, const orc_params* p, int vid, int k, int px, int py, const float* plane,
                       int sampling)
{
    const int W = f->mi_w, H = f->mi_h;
    const long ppv = (long)W * H;
    const int nvid = f->nb_ids[vid * f->max_nb + k];
    if (nvid < 0) return 2.0;
    const float* R = f->gray + (long)vid * ppv;
    const float* S = f->gray + (long)nvid * ppv;
    const double c0x = f->centers[2 * vid], c0y = f->centers[2 * vid + 1];
    const double c1x = f->centers[2 * nvid], c1y = f->centers[2 * nvid + 1];
    const double nx = plane[0], ny = plane[1], nz = plane[2], w = plane[3];
    const double A = -nx / nz, B = -ny / nz, C = (nx * px + ny * py + nz * w) / nz;
    const double d0 = A * px + B * py + C;
    const double stx = (c0x - c1x) / p->base, sty = (c0y - c1y) / p->base;
    const double ax = px + stx * d0, ay = py + sty * d0;
    /* sampling 2: the FP32 path's anchor, tap disparities and sample points */
    const f4 h = mk4(plane[0], plane[1], plane[2], plane[3]);
    const f3 dpf = disparity_plane(px, py, h);
    const float stxf = (f->centers[2 * vid] - f->centers[2 * nvid]) * (1.0f / fmaxf(p->base, 1e-6f));
    const float styf = (f->centers[2 * vid + 1] - f->centers[2 * nvid + 1]) * (1.0f / fmaxf(p->base, 1e-6f));
    if (sampling == 2) {
        float axf, ayf;
        f4 db;
        geo_map_hex(f->centers + 2 * vid, f->centers + 2 * nvid, px, py, h, px, py, p->base, &axf, &ayf, &db);
        if (!(axf >= 0.0f && axf < (float)W && ayf >= 0.0f && ayf < (float)H)) return 2.0;
    } else if (!(ax >= 0 && ax < W && ay >= 0 && ay < H)) {
        return 2.0;
    }
    const int radius = p->patch_size / 2;
    const double rc = R[py * W + px];
    const double ss2 = 2.0 * p->sigma_spatial * p->sigma_spatial, cc2 = 2.0 * p->sigma_color * p->sigma_color;
    double s_r = 0, s_rr = 0, s_s = 0, s_ss = 0, s_rs = 0, s_w = 0;
    for (int i = -radius; i <= radius; i += p->radius_increment)
        for (int j = -radius; j <= radius; j += p->radius_increment) {
            const int xr = px + i, yr = py + j;
            if (xr < 0 || xr >= W || yr < 0 || yr >= H) continue;
            double sx, sy;
            if (sampling == 2) {
                const float d = fmaf(dpf.y, (float)yr, dpf.x * (float)xr) + dpf.z;
                const float fx = fmaf(stxf, d, (float)xr), fy = fmaf(styf, d, (float)yr);
                if (!(fx >= 0.0f && fx < (float)W && fy >= 0.0f && fy < (float)H)) continue;
                sx = fx; sy = fy;
            } else {
                const double d = A * xr + B * yr + C;
                sx = xr + stx * d; sy = yr + sty * d;
                if (!(sx >= 0 && sx < W && sy >= 0 && sy < H)) continue;
            }
            const double r = R[yr * W + xr];
            const double s = sampling ? tex_quantised(S, W, H, sx, sy) : tex_exact(S, W, H, sx, sy);
            const double wgt = exp(-sqrt((double)(i * i + j * j)) / ss2 - fabs(r - rc) / cc2);
            s_r += wgt * r; s_rr += wgt * r * r; s_s += wgt * s; s_ss += wgt * s * s; s_rs += wgt * r * s; s_w += wgt;
        }
    if (s_w <= 1e-6) return 2.0;
    const double mr = s_r / s_w, ms = s_s / s_w;
    const double vr = s_rr / s_w - mr * mr, vs = s_ss / s_w - ms * ms;
    if (vr < 1e-5 || vs < 1e-5) return 2.0;
    const double c = 1.0 - (s_rs / s_w - mr * ms) / sqrt(vr * vs);
    return c < 0 ? 0 : (c > 2 ? 2 : c);
}

double orc_ncc_fp64(const orc_frame* f, const orc_params* p, int vid, int k, int px, int py, const float* plane)
{
    return ncc_fp64(f, p, vid, k, px, py, plane, 0);
}

void orc_ncc_fp64_batch(const orc_frame* f, const orc_params* p, const int* vids, const int* pxy,
                        const float* planes, int n, int sampling, int nthreads, double* out)
{
    const int K = f->max_nb;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int h = 0; h < n; ++h)
        for (int k = 0; k < K; ++k)
            out[(long)h * K + k] = k < f->nb_counts[vids[h]]
                                       ? ncc_fp64(f, p, vids[h], k, pxy[2 * h], pxy[2 * h + 1], planes + 4 * (long)h,
                                                  sampling)
                                       : 2.0;
}

/* ------------------------------------------------------------------------ */
float orc_expf(float x) { return canon_expf(x); }

float orc_uniform(uint64_t seed, uint32_t sweep, uint32_t pixel, uint32_t n)
{
    canon_rng g;
    canon_rng_init(&g, seed, sweep, pixel);
    float u = 0.0f;
    for (uint32_t i = 0; i <= n; ++i) u = canon_uniform(&g);
    return u;
}

float orc_tex_fetch(const float* img, int w, int h, float sx, float sy) { return canon_tex_fetch(img, w, h, sx, sy); }

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { canon_philox4x32_10(ctr, key, out); }
