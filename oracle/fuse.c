/*
 * oracle/fuse.c -- CPU restatement of the virtual-depth fusion and all-in-focus
 * splat LFRefocus::FuseVirtualDepth_BackProject (FocalStack/LFRefocus.cpp:
 * 1553-1794) with ComputeVirtualDepth (:2087-2098), ComputeVirtual3D
 * (:2100-2117) and BackProject2MI (:2119-2125).  TEST INFRASTRUCTURE ONLY;
 * parity unpinned (see pfd_oracle.h).
 *
 * Sequential, in the reference's order: reference micro-images in map order,
 * pixels row by row, neighbours in list order.  The masks a consistent pixel
 * sets on the neighbour pixels it used are read by everything processed after
 * it, and a later point overwrites an earlier one at the same output pixel.
 * Arithmetic is IEEE single precision as written (no contraction), except
 * ComputeVirtualDepth, whose double argument makes its division double.
 * Integer conversions follow x86: (int) truncates and cvRound rounds to
 * nearest even, both giving INT_MIN for NaN and out-of-range values.
 */
#include "pfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define INVALID_IMAGE (-9999.0f)            /* g_Invalid_image, Common/Common.cpp:53 */

static int trunc_x86(float x) { return (fabsf(x) < 2147483648.0f) ? (int)x : (int)0x80000000; }
static int round_x86(float x) { return (fabsf(x) < 2147483648.0f) ? (int)lrintf(x) : (int)0x80000000; }
static uint8_t sat_u8(float v)              /* saturate_cast<uchar>(float) */
{
    const int i = round_x86(v);
    return (uint8_t)(i < 0 ? 0 : (i > 255 ? 255 : i));
}

/* ComputeVirtualDepth: float mla_base over a double disparity. */
static float virtual_depth(float mla_base, float disp)
{
    const double d = (double)disp;
    if (d <= 0) return INVALID_IMAGE;
    return (float)((double)mla_base / d);
}

/* ComputeVirtual3D */
static void virtual_3d(float vd, int col, int row, int cols, int rows, const float* c_mla, float* out)
{
    const float cmx = (float)(cols - 1) * 0.5f + 1.0f, cmy = (float)(rows - 1) * 0.5f + 1.0f;
    const float ox = (float)col - cmx, oy = (float)row - cmy;
    out[0] = ox * vd + c_mla[0];
    out[1] = oy * vd + c_mla[1];
    out[2] = vd;
}

/* BackProject2MI */
static void back_project(const float* P, const float* c_mla, float cmx, float cmy, float* q)
{
    q[0] = ((P[0] - c_mla[0]) / P[2]) + cmx;
    q[1] = ((P[1] - c_mla[1]) / P[2]) + cmy;
}

static void colour_at(const orc_frame* f, const uint8_t* bgr, int v, int idx, float* c)
{
    const size_t ppv = (size_t)f->mi_w * f->mi_h;
    if (bgr) {
        const uint8_t* p = bgr + ((size_t)v * ppv + idx) * 3;
        c[0] = (float)p[0]; c[1] = (float)p[1]; c[2] = (float)p[2];
    } else {
        c[0] = c[1] = c[2] = f->gray[(size_t)v * ppv + idx];
    }
}

long long orc_fuse_virtual_depth(const orc_frame* f, const float* plane, const uint8_t* bgr, const int* lists,
                                 const int* list_counts, int max_list, const uint8_t* is_ref, const orc_fuse_params* p,
                                 int raw_w, int raw_h, float* vd_map, uint8_t* conf, uint8_t* aif, float* points)
{
    if (!f || !plane || !lists || !list_counts || !is_ref || !p || !vd_map || !conf || !aif) return -1;
    const int V = f->n_views, cols = f->mi_w, rows = f->mi_h, ppv = cols * rows;
    memset(vd_map, 0, sizeof(float) * (size_t)raw_w * raw_h);
    memset(conf, 0, (size_t)raw_w * raw_h);
    memset(aif, 0, (size_t)raw_w * raw_h * 3);
    uint8_t* mask = (uint8_t*)calloc((size_t)V * ppv, 1);
    int* used = (int*)malloc(sizeof(int) * (max_list > 0 ? max_list : 1));
    if (!mask || !used) { free(mask); free(used); return -1; }
    const float cmx = (float)(cols - 1) * 0.5f + 1.0f, cmy = (float)(rows - 1) * 0.5f + 1.0f;
    long long np = 0;
    for (int v = 0; v < V; ++v) {
        if (!is_ref[v]) continue;
        const float* c_ref = f->centers + 2 * v;
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) {
                const int index = r * cols + c;
                if (mask[(size_t)v * ppv + index] == 1) continue;
                const float* pl = plane + ((size_t)v * ppv + index) * 4;
                const float disp_ref = pl[3];
                if (disp_ref < p->min_ref_disp) continue;
                const float vd_ref = virtual_depth(p->mla_base, disp_ref);
                if (fabsf(vd_ref - INVALID_IMAGE) < 1.0e-6f || !isfinite(vd_ref)) continue;
                float normal[3] = { pl[0], pl[1], pl[2] };
                float P[3];
                virtual_3d(vd_ref, c, r, cols, rows, c_ref, P);
                float point[3] = { P[0], P[1], P[2] };
                float color[3];
                colour_at(f, bgr, v, index, color);
                const int nl = list_counts[v] < max_list ? list_counts[v] : max_list;
                for (int j = 0; j < nl; ++j) used[j] = -1;
                int num = 0;
                for (int j = 0; j < nl; ++j) {
                    const int u = lists[(size_t)v * max_list + j];
                    if (u < 0) continue;
                    const float* c_src = f->centers + 2 * u;
                    float q[2];
                    back_project(P, c_src, cmx, cmy, q);
                    const int src_r = trunc_x86(q[1] + 0.5f), src_c = trunc_x86(q[0] + 0.5f);
                    if (src_c < 0 || src_c >= cols || src_r < 0 || src_r >= rows) continue;
                    const int index_src = src_r * cols + src_c;
                    if (mask[(size_t)u * ppv + index_src] == 1) continue;
                    const float* ps = plane + ((size_t)u * ppv + index_src) * 4;
                    const float disp_src = ps[3];
                    if (disp_src <= 0.0f) continue;
                    const float vd_src = virtual_depth(p->mla_base, disp_src);
                    if (fabsf(vd_src - INVALID_IMAGE) < 1.0e-6f || !isfinite(vd_src)) continue;
                    float Ps[3];
                    virtual_3d(vd_src, src_c, src_r, cols, rows, c_src, Ps);
                    float rq[2];
                    back_project(Ps, c_ref, cmx, cmy, rq);
                    const float ex = (float)c - rq[0], ey = (float)r - rq[1];
                    const float reproj = sqrtf(ex * ex + ey * ey);
                    const float den = vd_ref < 1.0e-6f ? 1.0e-6f : vd_ref;     /* std::max(vd_ref, 1e-6f) */
                    const float rel = fabsf(vd_src - vd_ref) / den;
                    if (reproj < p->max_reproj_px && rel < p->max_rel_vd) {
                        for (int i = 0; i < 3; ++i) point[i] = point[i] + Ps[i];
                        normal[0] = normal[0] + ps[0];
                        normal[1] = normal[1] + ps[1];
                        normal[2] = normal[2] + ps[2];
                        float cs[3];
                        colour_at(f, bgr, u, index_src, cs);
                        for (int i = 0; i < 3; ++i) color[i] = color[i] + cs[i];
                        used[j] = index_src;
                        ++num;
                    }
                }
                if (num < p->min_consistent) continue;
                /* cv::Vec3f /= float: multiply by the float reciprocal */
                const float ia = 1.0f / ((float)num + 1.0f);
                for (int i = 0; i < 3; ++i) {
                    point[i] = point[i] * ia;
                    normal[i] = normal[i] * ia;
                    color[i] = color[i] * ia;
                }
                const int vx = round_x86(point[0]), vy = round_x86(point[1]);
                if (vy >= 0 && vy < raw_h && vx >= 0 && vx < raw_w) {
                    const size_t o = (size_t)vy * raw_w + vx;
                    vd_map[o] = point[2];
                    const int cf = (num + 1) * 60;
                    conf[o] = (uint8_t)(cf < 255 ? cf : 255);
                    aif[3 * o + 0] = sat_u8(color[0]);
                    aif[3 * o + 1] = sat_u8(color[1]);
                    aif[3 * o + 2] = sat_u8(color[2]);
                    if (points) {
                        float* pt = points + (size_t)np * 9;
                        pt[0] = point[0]; pt[1] = point[1]; pt[2] = point[2];
                        pt[3] = normal[0]; pt[4] = normal[1]; pt[5] = normal[2];
                        pt[6] = color[0]; pt[7] = color[1]; pt[8] = color[2];
                    }
                    ++np;
                }
                for (int j = 0; j < nl; ++j)
                    if (used[j] >= 0) mask[(size_t)lists[(size_t)v * max_list + j] * ppv + used[j]] = 1;
            }
    }
    free(mask);
    free(used);
    return np;
}
