/*
 * oracle/checks.c -- CPU restatement of the consistency pass that follows the
 * PatchMatch: MIDisparityFilterCPU (CheckModule/MIDisparityFilter.cpp) and
 * MICycleCheckerCPU (CheckModule/MICycleCheck.cpp).  TEST INFRASTRUCTURE
 * ONLY; parity unpinned (see pfd_oracle.h).
 *
 * Arithmetic: the reference is host C++ built with -O3 -ffast-math
 * -march=native (CMakeLists.txt:66), whose bits depend on the compiler's
 * choices.  This restatement evaluates every expression as written, left to
 * right, one rounding per operation and no fused operations, and the CUDA
 * kernels do the same.  std::hypot(float, float) is taken as the correctly
 * rounded (float)sqrt((double)x*x + (double)y*y); cv::meanStdDev as OpenCV's
 * scalar path: double sums in row-major order, mean = s * (1/n),
 * std = sqrt(max(sq * (1/n) - mean*mean, 0)).
 *
 * Neighbour indices: the reference reads bit b of selected_views as the b-th
 * entry of m_NeighsSortVecForMatch, while the matcher set it for the b-th
 * entry of its own compacted list (AdaptMIPMFrame.cpp:207-218); the two agree
 * when every listed neighbour is a matched view.  Both passes here use the
 * matcher's list, the one the bits were set for.
 */
#include "pfd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline float hypot_canon(float x, float y)
{
    const double dx = (double)x, dy = (double)y;
    return (float)sqrt(dx * dx + dy * dy);
}

/* EnumerateSetBits, MIDisparityFilter.cpp:25-34 */
static int set_bits(uint32_t mask, int* out, int max_needed)
{
    int n = 0;
    for (int b = 0; mask && n < max_needed; ++b) {
        if (mask & 1u) out[n++] = b;
        mask >>= 1u;
    }
    return n;
}

/* BilinearSampleF32, MIDisparityFilter.cpp:53-78 (MICycleCheck.cpp:55-66 is the same) */
static int bilinear_f32(const float* img, int W, int H, float x, float y, float* v)
{
    if (x < 0 || y < 0 || x > W - 1 || y > H - 1) return 0;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = x0 + 1 < W - 1 ? x0 + 1 : W - 1;
    const int y1 = y0 + 1 < H - 1 ? y0 + 1 : H - 1;
    const float ax = x - (float)x0, ay = y - (float)y0;
    const float v00 = img[y0 * W + x0], v01 = img[y1 * W + x0], v10 = img[y0 * W + x1], v11 = img[y1 * W + x1];
    float s = ((1.0f - ax) * (1.0f - ay)) * v00;
    s = s + ((1.0f - ax) * ay) * v01;
    s = s + (ax * (1.0f - ay)) * v10;
    s = s + (ax * ay) * v11;
    *v = s;
    return 1;
}

/* cv::meanStdDev over a 3x3 window with top-left (x0, y0). */
static void mean_std_3x3(const float* img, int W, int x0, int y0, float* mean, float* stdv)
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
    *mean = (float)s;
    *stdv = (float)sqrt(var);
}

/* std::round (half away from zero) to int */
static inline int round_half_away(float f) { return (int)roundf(f); }

/* PatchMeanStd3x3, MIDisparityFilter.cpp:120-136: centred window */
static int patch_mean_std_centred(const float* img, int W, int H, float fx, float fy, float* m, float* s)
{
    const int cx = round_half_away(fx), cy = round_half_away(fy);
    if (cx < 1 || cy < 1 || cx >= W - 1 || cy >= H - 1) return 0;
    mean_std_3x3(img, W, cx - 1, cy - 1, m, s);
    return isfinite(*m) && isfinite(*s) && *s > 1.0e-3f;
}

/* ComputePhotoResidual, MIDisparityFilter.cpp:138-156 */
static float photo_residual_filter(const float* ref, const float* nei, int W, int H, float px, float py, float qx, float qy)
{
    float Ir = 0.0f, In = 0.0f;
    if (!bilinear_f32(ref, W, H, px, py, &Ir)) return NAN;
    if (!bilinear_f32(nei, W, H, qx, qy, &In)) return NAN;
    float mr, sr, mn, sn;
    if (patch_mean_std_centred(ref, W, H, px, py, &mr, &sr) && patch_mean_std_centred(nei, W, H, qx, qy, &mn, &sn)) {
        const float Irn = (Ir - mr) / sr;
        const float Inn = (In - mn) / sn;
        return fabsf(Irn - Inn);
    }
    return fabsf(In - Ir);
}

/* Disparity of a pixel as FilterTile reads it: ph.w, falling back to d_cuda,
 * which WriteBackResults sets to the same value (AdaptMIPMFrame.cpp:376-377). */
static inline float read_disp(const orc_state* s, long i) { return s->plane[4 * i + 3]; }

/* BilinearDisparity, MIDisparityFilter.cpp:80-118 */
static float bilinear_disp(const orc_state* s, long base, int W, int H, float x, float y, float min_valid)
{
    if (x < 0 || y < 0 || x > W - 1 || y > H - 1) return NAN;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = x0 + 1 < W - 1 ? x0 + 1 : W - 1;
    const int y1 = y0 + 1 < H - 1 ? y0 + 1 : H - 1;
    const float ax = x - (float)x0, ay = y - (float)y0;
    float d[4];
    const long id[4] = { base + y0 * W + x0, base + y1 * W + x0, base + y0 * W + x1, base + y1 * W + x1 };
    for (int k = 0; k < 4; ++k) {
        d[k] = read_disp(s, id[k]);
        if (!isfinite(d[k]) || d[k] <= min_valid) return NAN;
    }
    float r = ((1.0f - ax) * (1.0f - ay)) * d[0];
    r = r + ((1.0f - ax) * ay) * d[1];
    r = r + (ax * (1.0f - ay)) * d[2];
    r = r + (ax * ay) * d[3];
    return r;
}

/* bilinear_cost lambda, MIDisparityFilter.cpp:455-476 */
static float bilinear_cost(const orc_state* s, long base, int W, int H, float x, float y)
{
    if (x < 0 || y < 0 || x > W - 1 || y > H - 1) return NAN;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const int x1 = x0 + 1 < W - 1 ? x0 + 1 : W - 1;
    const int y1 = y0 + 1 < H - 1 ? y0 + 1 : H - 1;
    const float ax = x - (float)x0, ay = y - (float)y0;
    const float c00 = s->cost[base + y0 * W + x0], c01 = s->cost[base + y1 * W + x0];
    const float c10 = s->cost[base + y0 * W + x1], c11 = s->cost[base + y1 * W + x1];
    if (!isfinite(c00) || !isfinite(c01) || !isfinite(c10) || !isfinite(c11)) return NAN;
    float r = ((1.0f - ax) * (1.0f - ay)) * c00;
    r = r + ((1.0f - ax) * ay) * c01;
    r = r + (ax * (1.0f - ay)) * c10;
    r = r + (ax * ay) * c11;
    return r;
}

/* Projection of p into neighbour k and back (the geometric cycle of
 * FilterTile :562-571 and ComputeTileReprojectionErrorMap :803-838). */
typedef struct { float dx, dy, scale; int ok; } nb_dir;

static nb_dir neighbour_dir(const orc_frame* f, int v, int nv, float baseline_unit)
{
    nb_dir r = { 0, 0, 0, 0 };
    const float Bx = f->centers[2 * v] - f->centers[2 * nv];          /* c_ref - c_nb (cv::Point2f) */
    const float By = f->centers[2 * v + 1] - f->centers[2 * nv + 1];
    const float baseline = hypot_canon(Bx, By);
    if (baseline < 1.0e-6f) return r;
    r.dx = Bx / baseline;
    r.dy = By / baseline;
    r.scale = baseline / baseline_unit;
    r.ok = 1;
    return r;
}

/* FilterTile (MIDisparityFilter.cpp:423-693) for one view, in place. */
static void filter_tile(const orc_frame* f, const orc_filter_cfg* cfg, float baseline_unit, int v, orc_state* st,
                        uint8_t* reason, long long* stats)
{
    const int W = f->mi_w, H = f->mi_h, N = W * H;
    const long base = (long)v * N;
    const float* ref = f->gray + base;
    unsigned char keep1[32 * 32], keepf[32 * 32];
    memset(keep1, 0, (size_t)N);
    memset(keepf, 0, (size_t)N);
    for (int i = 0; i < N; ++i) reason[base + i] = ORC_PR_KEEP;

    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int idx = y * W + x;
            stats[ORC_FS_TOTAL]++;
            const float d = read_disp(st, base + idx);
            if (!isfinite(d) || d <= cfg->min_valid_disp) continue;
            stats[ORC_FS_VALID_IN]++;
            const float cost = st->cost[base + idx];
            if (cfg->enable_cost_filter) {
                const int invalid_cost = (!isfinite(cost) || cost < 0.0f);
                const int high_cost = (isfinite(cost) && cost > cfg->max_cost);
                if (invalid_cost || high_cost) { reason[base + idx] = ORC_PR_COST; stats[ORC_FS_COST]++; continue; }
            }
            int vids[32];
            int nv;
            if (cfg->use_selected_views_only) nv = set_bits(st->sel[base + idx], vids, cfg->max_triplet);
            else {
                nv = f->nb_counts[v] < cfg->max_triplet ? f->nb_counts[v] : cfg->max_triplet;
                for (int i = 0; i < nv; ++i) vids[i] = i;
            }
            if (nv == 0) { reason[base + idx] = ORC_PR_NOSUPPORT; stats[ORC_FS_NOSUPPORT]++; continue; }
            const float px = (float)x, py = (float)y;
            int support = 0, good = 0;
            for (int vi = 0; vi < nv; ++vi) {
                const int b = vids[vi];
                if (b < 0 || b >= f->nb_counts[v]) continue;
                const int nvid = f->nb_ids[v * f->max_nb + b];
                if (nvid < 0) continue;
                const nb_dir g = neighbour_dir(f, v, nvid, baseline_unit);
                if (!g.ok) continue;
                const float qx = px + (g.dx * d) * g.scale;
                const float qy = py + (g.dy * d) * g.scale;
                if (qx < 0 || qy < 0 || qx > W - 1 || qy > H - 1) continue;
                const long nbase = (long)nvid * N;
                const float d_nei = bilinear_disp(st, nbase, W, H, qx, qy, cfg->min_valid_disp);
                if (!isfinite(d_nei)) continue;
                if (cfg->enable_cost_filter) {
                    const float nc = bilinear_cost(st, nbase, W, H, qx, qy);
                    const int inv = (!isfinite(nc) || nc < 0.0f);
                    const int high = (isfinite(nc) && nc > cfg->max_cost);
                    if (inv || high) continue;
                }
                ++support;
                int pass_geo = 1, pass_photo = 1;
                if (cfg->enable_cycle_geo_filter) {
                    const float phx = qx - (g.dx * d_nei) * g.scale;
                    const float phy = qy - (g.dy * d_nei) * g.scale;
                    const float ge = hypot_canon(phx - px, phy - py);
                    pass_geo = isfinite(ge) && ge <= cfg->max_geo_err_px;
                }
                if (cfg->enable_cycle_photo_filter) {
                    const float pe = photo_residual_filter(ref, f->gray + nbase, W, H, px, py, qx, qy);
                    pass_photo = isfinite(pe) && pe <= cfg->max_photo_err_u;
                }
                if (pass_geo && pass_photo) ++good;
            }
            if (support < cfg->min_good_neighbors) { reason[base + idx] = ORC_PR_NOSUPPORT; stats[ORC_FS_NOSUPPORT]++; continue; }
            if (good < cfg->min_good_neighbors) { reason[base + idx] = ORC_PR_CYCLE; stats[ORC_FS_CYCLE]++; continue; }
            keep1[idx] = 1;
            keepf[idx] = 1;
            reason[base + idx] = ORC_PR_KEEP;
        }

    if (cfg->enable_spike_filter) {
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int idx = y * W + x;
                if (!keep1[idx]) continue;
                float nvals[8];
                int n = 0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0) continue;
                        const int xn = x + dx, yn = y + dy;
                        if (xn < 0 || yn < 0 || xn >= W || yn >= H) continue;
                        const int ni = yn * W + xn;
                        if (!keep1[ni]) continue;
                        const float dv = read_disp(st, base + ni);
                        if (!isfinite(dv) || dv <= cfg->min_valid_disp) continue;
                        nvals[n++] = dv;
                    }
                if (n < cfg->spike_min_neighbors) continue;
                /* the element std::nth_element puts at n/2: the (n/2)-th smallest */
                for (int a = 1; a < n; ++a) {
                    const float t = nvals[a];
                    int b = a - 1;
                    while (b >= 0 && nvals[b] > t) { nvals[b + 1] = nvals[b]; --b; }
                    nvals[b + 1] = t;
                }
                const float med = nvals[n / 2];
                const float cur = read_disp(st, base + idx);
                if (!isfinite(cur)) continue;
                if (fabsf(cur - med) > cfg->spike_abs_diff) {
                    keepf[idx] = 0;
                    reason[base + idx] = ORC_PR_SPIKE;
                    stats[ORC_FS_SPIKE]++;
                }
            }
    }

    for (int idx = 0; idx < N; ++idx) {
        const float d = read_disp(st, base + idx);
        if (!isfinite(d) || d <= cfg->min_valid_disp) continue;
        if (keepf[idx]) { stats[ORC_FS_KEPT]++; continue; }
        stats[ORC_FS_REMOVED]++;
        /* InvalidatePixel, MIDisparityFilter.cpp:158-174 */
        float* pl = st->plane + 4 * (base + idx);
        pl[0] = 0.0f; pl[1] = 0.0f; pl[2] = 0.0f; pl[3] = -1.0f;
        st->cost[base + idx] = 2.0f;
        float* dp = st->disp + 4 * (base + idx);
        dp[0] = -1.0f; dp[1] = -1.0f; dp[2] = 0.0f; dp[3] = 0.0f;
        if (cfg->clear_selected_views_when_invalid) st->sel[base + idx] = 0u;
    }
}

int orc_filter_global(const orc_frame* f, const orc_filter_cfg* cfg, float baseline_unit, orc_state* st,
                      uint8_t* reason, long long* stats)
{
    if (!f || !cfg || !st || !reason || !stats || f->mi_w > 32 || f->mi_h > 32) return -1;
    for (int i = 0; i < ORC_FS_COUNT; ++i) stats[i] = 0;
    /* FilterGlobal (MIDisparityFilter.cpp:962-986): tiles in problem-map order */
    for (int v = 0; v < f->n_views; ++v) filter_tile(f, cfg, baseline_unit, v, st, reason, stats);
    return 0;
}

/* QuantileFromSorted, MIDisparityFilter.cpp:36-51 */
static float quantile_sorted(const float* v, int n, float q)
{
    if (n == 0) return 0.0f;
    if (n == 1) return v[0];
    const float qq = q < 0.0f ? 0.0f : (q > 1.0f ? 1.0f : q);
    const float pos = qq * (float)(n - 1);
    const int lo = (int)floorf(pos), hi = (int)ceilf(pos);
    const float t = pos - (float)lo;
    if (lo == hi) return v[lo];
    return v[lo] * (1.0f - t) + v[hi] * t;
}

/* ComputeTileReprojectionErrorMap (MIDisparityFilter.cpp:695-842) over all views. */
int orc_reprojection_error(const orc_frame* f, const orc_filter_cfg* cfg, float baseline_unit, const orc_state* st,
                           float* err)
{
    if (!f || !cfg || !st || !err) return -1;
    const int W = f->mi_w, H = f->mi_h, N = W * H;
    for (int v = 0; v < f->n_views; ++v) {
        const long base = (long)v * N;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int idx = y * W + x;
                err[base + idx] = -1.0f;
                const float d = read_disp(st, base + idx);
                if (!isfinite(d) || d <= cfg->min_valid_disp) continue;
                if (cfg->enable_cost_filter) {
                    const float c = st->cost[base + idx];
                    if ((!isfinite(c) || c < 0.0f) || (isfinite(c) && c > cfg->max_cost)) continue;
                }
                int vids[32];
                int nv;
                if (cfg->use_selected_views_only) nv = set_bits(st->sel[base + idx], vids, cfg->max_triplet);
                else {
                    nv = f->nb_counts[v] < cfg->max_triplet ? f->nb_counts[v] : cfg->max_triplet;
                    for (int i = 0; i < nv; ++i) vids[i] = i;
                }
                if (nv == 0) continue;
                const float px = (float)x, py = (float)y;
                float ge[32];
                int ng = 0;
                for (int vi = 0; vi < nv; ++vi) {
                    const int b = vids[vi];
                    if (b < 0 || b >= f->nb_counts[v]) continue;
                    const int nvid = f->nb_ids[v * f->max_nb + b];
                    if (nvid < 0) continue;
                    const nb_dir g = neighbour_dir(f, v, nvid, baseline_unit);
                    if (!g.ok) continue;
                    const float qx = px + (g.dx * d) * g.scale;
                    const float qy = py + (g.dy * d) * g.scale;
                    if (qx < 0 || qy < 0 || qx > W - 1 || qy > H - 1) continue;
                    const long nbase = (long)nvid * N;
                    const float d_nei = bilinear_disp(st, nbase, W, H, qx, qy, cfg->min_valid_disp);
                    if (!isfinite(d_nei)) continue;
                    if (cfg->enable_cost_filter) {
                        const float nc = bilinear_cost(st, nbase, W, H, qx, qy);
                        if ((!isfinite(nc) || nc < 0.0f) || (isfinite(nc) && nc > cfg->max_cost)) continue;
                    }
                    const float phx = qx - (g.dx * d_nei) * g.scale;
                    const float phy = qy - (g.dy * d_nei) * g.scale;
                    const float e = hypot_canon(phx - px, phy - py);
                    if (isfinite(e)) ge[ng++] = e;
                }
                if (ng >= cfg->min_good_neighbors) {
                    for (int a = 1; a < ng; ++a) {
                        const float t = ge[a];
                        int b = a - 1;
                        while (b >= 0 && ge[b] > t) { ge[b + 1] = ge[b]; --b; }
                        ge[b + 1] = t;
                    }
                    err[base + idx] = quantile_sorted(ge, ng, 0.5f);
                }
            }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* MICycleCheckerCPU (CheckModule/MICycleCheck.cpp)                          */
/* ------------------------------------------------------------------------- */

void orc_mean_std_3x3(const float* img, int W, int x0, int y0, float* mean, float* stdv)
{
    mean_std_3x3(img, W, x0, y0, mean, stdv);
}

/* cv::BORDER_REFLECT_101 index (borderInterpolate) */
static int reflect101(int i, int n)
{
    if (n == 1) return 0;
    while (i < 0 || i >= n) {
        if (i < 0) i = -i;
        else i = 2 * n - 2 - i;
    }
    return i;
}

/* BuildTextureMaskAndViz, MICycleCheck.cpp:186-213.  Gray values are integers
 * 0..255, so the Sobel sums and the 7x7 box sums are exact in any order; the
 * box mean is OpenCV's (float)(double_sum * (1.0 / 49)). */
int orc_texture_mask(const float* g, int W, int H, const orc_cycle_cfg* cfg, float* grad, float* var, uint8_t* mask)
{
    if (!g || !cfg || W < 1 || H < 1) return -1;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int xm = reflect101(x - 1, W), xp = reflect101(x + 1, W);
            const int ym = reflect101(y - 1, H), yp = reflect101(y + 1, H);
            /* cv::Sobel(dx=1): [-1 0 1] along x, [1 2 1] along y; dy=1 transposed */
            const float gx = (g[ym * W + xp] - g[ym * W + xm]) + 2.0f * (g[y * W + xp] - g[y * W + xm]) +
                             (g[yp * W + xp] - g[yp * W + xm]);
            const float gy = (g[yp * W + xm] - g[ym * W + xm]) + 2.0f * (g[yp * W + x] - g[ym * W + x]) +
                             (g[yp * W + xp] - g[ym * W + xp]);
            const float mag = sqrtf(gx * gx + gy * gy);          /* cv::magnitude */
            double s = 0.0, s2 = 0.0;
            for (int dy = -3; dy <= 3; ++dy)
                for (int dx = -3; dx <= 3; ++dx) {
                    const float v = g[reflect101(y + dy, H) * W + reflect101(x + dx, W)];
                    s += (double)v;
                    s2 += (double)(v * v);                          /* gray.mul(gray) is float */
                }
            const double scale = 1.0 / 49.0;
            const float mean = (float)(s * scale), mean2 = (float)(s2 * scale);
            const float vr = mean2 - mean * mean;                    /* mean2 - mean.mul(mean) */
            const int m1 = mag > cfg->sobel_thresh, m2 = vr > cfg->var_thresh;
            if (grad) grad[y * W + x] = mag;
            if (var) var[y * W + x] = vr;
            if (mask) mask[y * W + x] = (uint8_t)((cfg->use_and ? (m1 && m2) : (m1 || m2)) ? 255 : 0);
        }
    return 0;
}

/* patch_mean_std lambda, MICycleCheck.cpp:327-339: 3x3 window with top-left
 * (round(x) - 2, round(y) - 2) */
static int patch_mean_std_cycle(const float* img, int W, int H, float fx, float fy, float* m, float* s)
{
    const int cx = round_half_away(fx), cy = round_half_away(fy);
    if (cx < 2 || cy < 2 || cx >= W - 2 || cy >= H - 2) return 0;
    mean_std_3x3(img, W, cx - 2, cy - 2, m, s);
    return isfinite(*m) && isfinite(*s) && *s > 1e-3f;
}

/* bilinear_disp lambda, MICycleCheck.cpp:306-325: non-finite corners are
 * replaced (d00 by 0, the others by d00) instead of failing. */
static float bilinear_disp_cycle(const orc_state* s, long base, int W, int H, float fx, float fy)
{
    if (fx < 0 || fy < 0 || fx > W - 1 || fy > H - 1) return NAN;
    const int x0 = (int)floorf(fx), y0 = (int)floorf(fy);
    const int x1 = x0 + 1 < W - 1 ? x0 + 1 : W - 1;
    const int y1 = y0 + 1 < H - 1 ? y0 + 1 : H - 1;
    const float ax = fx - (float)x0, ay = fy - (float)y0;
    float d00 = read_disp(s, base + y0 * W + x0), d01 = read_disp(s, base + y1 * W + x0);
    float d10 = read_disp(s, base + y0 * W + x1), d11 = read_disp(s, base + y1 * W + x1);
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

static inline float min_std(float a, float b) { return (b < a) ? b : a; }   /* std::min */
static inline float max_std(float a, float b) { return (a < b) ? b : a; }   /* std::max */

int orc_cycle_check(const orc_frame* f, const orc_cycle_cfg* cfg, float baseline_unit, const orc_state* st,
                    orc_cycle_stats* out, float* geo_err, float* pho_err, uint8_t* texmask)
{
    if (!f || !cfg || !st || !out || f->mi_w > 32 || f->mi_h > 32) return -1;
    const int W = f->mi_w, H = f->mi_h, N = W * H;
    memset(out, 0, sizeof(*out));
    /* global accumulators of CheckGlobal (MICycleCheck.cpp:742-756) */
    double mask_geo_sq = 0.0, mask_photo_sq = 0.0, mask_geo_sum = 0.0, mask_photo_sum = 0.0;
    long long mask_count = 0, all_count = 0, comp_total = 0, comp_good = 0, comp_good_geo = 0, comp_good_photo = 0;
    long long hist[256];
    int hist_n = 0;
    memset(hist, 0, sizeof(hist));
    double geo_min = INFINITY, geo_max = 0.0;
    double io_mean_geo = 0.0, io_mean_photo = 0.0, io_rmse_geo = 0.0, io_rmse_photo = 0.0;
    long long io_num = 0;

    float g_avg[32 * 32], p_avg[32 * 32];
    uint8_t masked[32 * 32], tm[32 * 32];

    for (int v = 0; v < f->n_views; ++v) {
        const long base = (long)v * N;
        const float* ref = f->gray + base;
        orc_texture_mask(ref, W, H, cfg, NULL, NULL, tm);
        if (texmask) memcpy(texmask + base, tm, (size_t)N);
        int n = 0, n_m = 0;
        long long lc_total = 0, lc_good = 0, lc_geo = 0, lc_photo = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int idx = y * W + x;
                float gcell = 0.0f, pcell = 0.0f;
                const float d = read_disp(st, base + idx);
                if (isfinite(d)) {
                    int vids[32];
                    const int nv = set_bits(st->sel[base + idx], vids, cfg->max_triplet);
                    if (nv > 0) {
                        const float px = (float)x, py = (float)y;
                        float gsum = 0.0f, psum = 0.0f;
                        int cnt = 0;
                        float m_ref, s_ref;
                        const int ref_mask_ok = patch_mean_std_cycle(ref, W, H, px, py, &m_ref, &s_ref);
                        if (ref_mask_ok) ++lc_total;
                        int gate = 0, gate_geo = 0, gate_photo = 0;
                        for (int vi = 0; vi < nv; ++vi) {
                            const int b = vids[vi];
                            if (b < 0 || b >= f->nb_counts[v]) continue;
                            const int nvid = f->nb_ids[v * f->max_nb + b];
                            /* a missing neighbour has an empty gray image, so its sample
                             * fails (MICycleCheck.cpp:396-399) after nothing was counted */
                            if (nvid < 0) continue;
                            const int dn_vid = nvid;
                            const nb_dir g = neighbour_dir(f, v, nvid, baseline_unit);
                            if (!g.ok) continue;
                            const float qx = px + (g.dx * d) * g.scale;
                            const float qy = py + (g.dy * d) * g.scale;
                            if (qx < 0 || qy < 0 || qx > W - 1 || qy > H - 1) continue;
                            const float d_nei = bilinear_disp_cycle(st, (long)dn_vid * N, W, H, qx, qy);
                            const float phx = qx - (g.dx * d_nei) * g.scale;
                            const float phy = qy - (g.dy * d_nei) * g.scale;
                            const float geo_e = hypot_canon(phx - px, phy - py);
                            if (!(geo_e < (float)(W * 2))) continue;
                            float Ir, In;
                            if (!bilinear_f32(ref, W, H, px, py, &Ir)) continue;
                            const float* nei = f->gray + (long)nvid * N;
                            if (!bilinear_f32(nei, W, H, qx, qy, &In)) continue;
                            float mr, sr, mn, sn, phe;
                            if (patch_mean_std_cycle(ref, W, H, px, py, &mr, &sr) &&
                                patch_mean_std_cycle(nei, W, H, qx, qy, &mn, &sn)) {
                                const float Irn = (Ir - mr) / sr, Inn = (In - mn) / sn;
                                phe = fabsf(Irn - Inn);
                            } else {
                                phe = fabsf(In - Ir);
                            }
                            const float phe_raw = phe;
                            if (isfinite(phe)) phe = min_std(phe, 3.0f);
                            const float geo_used = cfg->clamp_geo ? min_std(geo_e, cfg->geo_u_px) : geo_e;
                            const float phe_used = cfg->clamp_photo ? min_std(phe, cfg->photo_u) : phe;
                            const int pg = cfg->gate_use_clamped ? (geo_used <= cfg->gate_geo_px) : (geo_e <= cfg->gate_geo_px);
                            const int pp = cfg->gate_use_clamped ? (phe_used <= cfg->gate_photo_u) : (phe_raw <= cfg->gate_photo_u);
                            if (pg && pp) ++gate;
                            if (pg) ++gate_geo;
                            if (pp) ++gate_photo;
                            int pixel_ok = 1;
                            if (cfg->pixel_gate_enabled) pixel_ok = pg && pp;
                            if (pixel_ok) { gsum = gsum + geo_used; psum = psum + phe_used; ++cnt; }
                            if (cnt > 0) { gcell = max_std(gcell, geo_used); pcell = max_std(pcell, phe_used); }
                        }
                        if (ref_mask_ok && gate >= cfg->gate_min_good_neighbors) ++lc_good;
                        if (ref_mask_ok && gate_geo >= cfg->gate_min_good_neighbors) ++lc_geo;
                        if (ref_mask_ok && gate_photo >= cfg->gate_min_good_neighbors) ++lc_photo;
                        if ((!cfg->pixel_gate_enabled && cnt > 0) ||
                            (cfg->pixel_gate_enabled && cnt >= cfg->gate_min_good_neighbors)) {
                            g_avg[n] = cnt > 0 ? gsum / (float)cnt : 0.0f;
                            p_avg[n] = cnt > 0 ? psum / (float)cnt : 0.0f;
                            masked[n] = tm[idx] != 0;
                            n_m += masked[n];
                            ++n;
                        }
                    }
                }
                if (geo_err) geo_err[base + idx] = gcell;
                if (pho_err) pho_err[base + idx] = pcell;
            }

        /* tile statistics and their merge (MICycleCheck.cpp:541-600) */
        double sg = 0.0, sp = 0.0, sqg = 0.0, sqp = 0.0;
        double sgm = 0.0, spm = 0.0, sqgm = 0.0, sqpm = 0.0;
        for (int i = 0; i < n; ++i) { sg += g_avg[i]; sqg += (double)(g_avg[i] * g_avg[i]); }
        for (int i = 0; i < n; ++i) { sp += p_avg[i]; sqp += (double)(p_avg[i] * p_avg[i]); }
        for (int i = 0; i < n; ++i) if (masked[i]) { sgm += g_avg[i]; sqgm += (double)(g_avg[i] * g_avg[i]); }
        for (int i = 0; i < n; ++i) if (masked[i]) { spm += p_avg[i]; sqpm += (double)(p_avg[i] * p_avg[i]); }
        if (n > 0) {
            const double mg = sg / (double)n, mp = sp / (double)n;
            const long long N0 = io_num + n;
            const double den = (double)(N0 > 1 ? N0 : 1);
            io_mean_geo = (io_mean_geo * (double)io_num + mg * (double)n) / den;
            io_mean_photo = (io_mean_photo * (double)io_num + mp * (double)n) / den;
            io_num = N0;
            io_rmse_geo += sqg;
            io_rmse_photo += sqp;
        }
        mask_geo_sq += sqgm;
        mask_photo_sq += sqpm;
        mask_geo_sum += sgm;
        mask_photo_sum += spm;
        comp_total += lc_total;
        comp_good += lc_good;
        comp_good_geo += lc_geo;
        comp_good_photo += lc_photo;
        for (int i = 0; i < n; ++i) {
            if (!masked[i]) continue;
            const float gv = g_avg[i];
            if (!isfinite(gv) || gv < 0.0f) continue;
            int bi = (int)floor((double)gv / 0.5);
            if (bi < 0) bi = 0;
            if (bi > 255) bi = 255;
            hist[bi] += 1;
            if (bi + 1 > hist_n) hist_n = bi + 1;
            if (gv < geo_min) geo_min = gv;
            if (gv > geo_max) geo_max = gv;
        }
        mask_count += n_m;
        all_count += n;
    }

    out->num_samples = io_num;
    out->mean_geo_err_px = io_mean_geo;
    out->mean_photo_err = io_mean_photo;
    out->completeness = comp_total > 0 ? (double)comp_good / (double)comp_total : 0.0;
    out->completeness_geo = comp_total > 0 ? (double)comp_good_geo / (double)comp_total : 0.0;
    out->completeness_photo = comp_total > 0 ? (double)comp_good_photo / (double)comp_total : 0.0;
    out->completeness_masked_pixels = comp_total;
    out->completeness_good_pixels = comp_good;
    out->completeness_good_pixels_geo = comp_good_geo;
    out->completeness_good_pixels_photo = comp_good_photo;
    if (io_num > 0) {
        out->rmse_geo_err_px = sqrt(io_rmse_geo / (double)io_num);
        out->rmse_photo_err = sqrt(io_rmse_photo / (double)io_num);
    }
    out->median_geo_err_px = out->mean_geo_err_px;     /* MICycleCheck.cpp:831-832 */
    out->p90_geo_err_px = out->mean_geo_err_px;
    out->masked_count = mask_count;
    out->all_count = all_count;
    out->masked_geo_mean = mask_count > 0 ? mask_geo_sum / (double)mask_count : 0.0;
    out->masked_photo_mean = mask_count > 0 ? mask_photo_sum / (double)mask_count : 0.0;
    out->masked_geo_rmse = mask_count > 0 ? sqrt(mask_geo_sq / (double)mask_count) : 0.0;
    out->masked_photo_rmse = mask_count > 0 ? sqrt(mask_photo_sq / (double)mask_count) : 0.0;
    out->coverage = all_count > 0 ? (double)mask_count / (double)all_count : 0.0;
    if (mask_count > 0 && hist_n > 0) {
        long long cum = 0;
        int med = 0, p90 = 0;
        for (int i = 0; i < hist_n; ++i) {
            cum += hist[i];
            if (!med && cum >= (long long)ceil(0.5 * (double)mask_count)) { out->masked_geo_median_approx = (i + 0.5) * 0.5; med = 1; }
            if (!p90 && cum >= (long long)ceil(0.9 * (double)mask_count)) { out->masked_geo_p90_approx = (i + 0.5) * 0.5; p90 = 1; }
            if (med && p90) break;
        }
    }
    out->masked_geo_min = isfinite(geo_min) ? geo_min : 0.0;
    out->masked_geo_max = geo_max;
    return 0;
}
