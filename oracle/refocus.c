/*
 * oracle/refocus.c -- CPU restatement of the focal-stack render.  TEST
 * INFRASTRUCTURE ONLY; parity unpinned (see pfd_oracle.h).
 *
 * The reference has no multi-slice render; the definition here is built from
 * its back-projection LFRefocus::BackProject2MI (FocalStack/LFRefocus.cpp:
 * 2119-2125): a virtual point X at virtual depth v maps into micro-image i at
 * u = (X - c_i) / v + center_mi, with center_mi = ((m-1)/2 + 1) as in
 * FuseVirtualDepth_BackProject (:1635-1636).  Arithmetic is IEEE single
 * precision as written, the three bilinear steps fused (fmaf).
 */
#include "pfd_oracle.h"

#include <math.h>
#include <stdlib.h>

/* Views whose centre lies in [cx_lo, cx_hi] x [cy_lo, cy_hi], ascending. */
static int views_in_box(const orc_frame* f, float cx_lo, float cx_hi, float cy_lo, float cy_hi, int* ids)
{
    int n = 0;
    for (int i = 0; i < f->n_views; ++i) {
        const float cx = f->centers[2 * i], cy = f->centers[2 * i + 1];
        if (cx >= cx_lo && cx <= cx_hi && cy >= cy_lo && cy <= cy_hi) ids[n++] = i;
    }
    return n;
}

static long long render(const orc_frame* f, int raw_w, int raw_h, const float* slice_vd, int n_slices, int out_w,
                        int out_h, float* out)
{
    const int m = f->mi_w, mh = f->mi_h;
    const float cmx = (float)(m - 1) * 0.5f + 1.0f, cmy = (float)(mh - 1) * 0.5f + 1.0f;
    const float sx = (float)raw_w / (float)out_w, sy = (float)raw_h / (float)out_h;
    const float umax = (float)(m - 1), wmax = (float)(mh - 1);
    const int TB = 16;                     /* output blocks, for culling only */
    const int nbx = (out_w + TB - 1) / TB, nby = (out_h + TB - 1) / TB;
    const long long nblocks = (long long)n_slices * nbx * nby;
    long long samples = 0;
#pragma omp parallel reduction(+ : samples)
    {
        int* ids = (int*)malloc(sizeof(int) * (size_t)(f->n_views > 0 ? f->n_views : 1));
#pragma omp for schedule(dynamic, 4)
        for (long long blk = 0; blk < nblocks; ++blk) {
            const int s = (int)(blk / ((long long)nbx * nby));
            const int by = (int)((blk / nbx) % nby) * TB, bx = (int)(blk % nbx) * TB;
            const float v = slice_vd[s];
            const int ex = bx + TB < out_w ? bx + TB : out_w, ey = by + TB < out_h ? by + TB : out_h;
            const float X0 = ((float)bx + 0.5f) * sx - 0.5f, X1 = ((float)(ex - 1) + 0.5f) * sx - 0.5f;
            const float Y0 = ((float)by + 0.5f) * sy - 0.5f, Y1 = ((float)(ey - 1) + 0.5f) * sy - 0.5f;
            /* u in [0, m-1]  <=>  c in [X - (m-1-cm) v, X + cm v]; 1 px of slack */
            const int n = views_in_box(f, X0 - (umax - cmx) * v - 1.0f, X1 + cmx * v + 1.0f,
                                       Y0 - (wmax - cmy) * v - 1.0f, Y1 + cmy * v + 1.0f, ids);
            for (int oy = by; oy < ey; ++oy)
                for (int ox = bx; ox < ex; ++ox) {
                    const float X = ((float)ox + 0.5f) * sx - 0.5f, Y = ((float)oy + 0.5f) * sy - 0.5f;
                    float sum = 0.0f;
                    int cnt = 0;
                    for (int k = 0; k < n; ++k) {
                        const int i = ids[k];
                        const float u = (X - f->centers[2 * i]) / v + cmx;
                        const float w = (Y - f->centers[2 * i + 1]) / v + cmy;
                        if (!(u >= 0.0f && u <= umax && w >= 0.0f && w <= wmax)) continue;
                        const int x0 = (int)floorf(u), y0 = (int)floorf(w);
                        const int x1 = x0 + 1 < m - 1 ? x0 + 1 : m - 1;
                        const int y1 = y0 + 1 < mh - 1 ? y0 + 1 : mh - 1;
                        const float ax = u - (float)x0, ay = w - (float)y0;
                        const float* T = f->gray + (size_t)i * m * mh;
                        const float t00 = T[y0 * m + x0], t01 = T[y0 * m + x1];
                        const float t10 = T[y1 * m + x0], t11 = T[y1 * m + x1];
                        const float top = fmaf(ax, t01 - t00, t00);
                        const float bot = fmaf(ax, t11 - t10, t10);
                        sum = sum + fmaf(ay, bot - top, top);
                        ++cnt;
                    }
                    samples += cnt;
                    if (out) out[((size_t)s * out_h + oy) * out_w + ox] = cnt ? sum / (float)cnt : 0.0f;
                }
        }
        free(ids);
    }
    return samples;
}

int orc_refocus(const orc_frame* f, int raw_w, int raw_h, const float* slice_vd, int n_slices, int out_w, int out_h,
                float* out)
{
    if (!f || !slice_vd || !out || n_slices < 1 || out_w < 1 || out_h < 1 || raw_w < 1 || raw_h < 1) return -1;
    for (int s = 0; s < n_slices; ++s)
        if (!(slice_vd[s] > 0.0f)) return -1;
    render(f, raw_w, raw_h, slice_vd, n_slices, out_w, out_h, out);
    return 0;
}

long long orc_refocus_samples(const orc_frame* f, int raw_w, int raw_h, const float* slice_vd, int n_slices,
                              int out_w, int out_h)
{
    if (!f || !slice_vd || n_slices < 1 || out_w < 1 || out_h < 1) return -1;
    return render(f, raw_w, raw_h, slice_vd, n_slices, out_w, out_h, NULL);
}
