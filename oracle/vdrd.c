/*
 * oracle/vdrd.c -- CPU restatement of the virtual-to-real depth conversion and
 * the behavioural-model fit.  TEST INFRASTRUCTURE ONLY; parity unpinned (see
 * pfd_oracle.h).  FP64 throughout, every expression as written, no fused
 * operations (built with -ffp-contract=off).
 */
#include "pfd_oracle.h"

#include <math.h>

/* LFRefocus::ConvertVdToRd, FocalStack/LFRefocus.cpp:2515-2534 */
float orc_vd_to_rd(float v_depth, const double c[3])
{
    const double v = (double)v_depth;
    const double denom = 1.0 - v * c[0];
    if (fabs(denom) < 1.0e-12) return 0.0f;
    const double z = (v * c[1] + c[2]) / denom;
    if (!isfinite(z) || z < 0.0) return 0.0f;
    return (float)z;
}

/* LFRefocus::ConvertVdToRdSegment, LFRefocus.cpp:2536-2593, with the segments
 * (depth_min, depth_max, c0, c1, c2) passed in instead of read from XML. */
float orc_vd_to_rd_segment(float v_depth, const double* segs, int nseg)
{
    double z = 0.0;
    for (int s = 0; s < nseg; ++s) {
        const double* g = segs + 5 * s;
        if ((double)v_depth >= g[0] && (double)v_depth < g[1]) {
            const double v = (double)v_depth;
            const double denom = 1.0 - v * g[2];
            if (fabs(denom) < 1.0e-12) return 0.0f;
            z = (v * g[3] + g[4]) / denom;
            break;
        }
    }
    if (!isfinite(z) || z < 0.0) return 0.0f;
    return (float)z;
}

/* VirtualToRealDepthFunc::convertVirtualToRealDepth, VirtualToRealDepthFunc.cpp:
 * 3421-3450: z = (v c1 + c2) / (1 - v c0) per pixel in double (IEEE division),
 * NaN, infinite and negative values set to 0. */
void orc_vd_to_rd_map(const float* vd, long n, const double c[3], double* rd)
{
    for (long i = 0; i < n; ++i) {
        const double v = (double)vd[i];
        const double num = v * c[1] + c[2];
        const double den = 1.0 - v * c[0];
        double z = num / den;
        if (isnan(z) || isinf(z) || z < 0.0) z = 0.0;
        rd[i] = z;
    }
}

/* VirtualToRealDepthFunc::BehavioralModel (VirtualToRealDepthFunc.cpp:3390-3418):
 * least squares of [a_L v, v, 1] c = a_L over the pairs (a_L = real depth).  The
 * reference solves with cv::solve(DECOMP_SVD); this restatement solves the
 * normal equations in long double (a different but well-conditioned route, so
 * parity here is to a stated relative tolerance).  Returns -1 when n < 3 or
 * the system is singular. */
int orc_behavioral_fit(const float* real_depth, const float* vd, long n, double c[3])
{
    if (n < 3) return -1;
    long double A[3][3] = { { 0 } }, b[3] = { 0 };
    for (long i = 0; i < n; ++i) {
        const long double aL = real_depth[i], v = vd[i];
        const long double x[3] = { aL * v, v, 1.0L };
        for (int r = 0; r < 3; ++r) {
            for (int q = 0; q < 3; ++q) A[r][q] += x[r] * x[q];
            b[r] += x[r] * aL;
        }
    }
    /* Gaussian elimination with partial pivoting */
    long double M[3][4];
    for (int r = 0; r < 3; ++r) { for (int q = 0; q < 3; ++q) M[r][q] = A[r][q]; M[r][3] = b[r]; }
    for (int col = 0; col < 3; ++col) {
        int piv = col;
        for (int r = col + 1; r < 3; ++r) if (fabsl(M[r][col]) > fabsl(M[piv][col])) piv = r;
        if (fabsl(M[piv][col]) < 1e-300L) return -1;
        if (piv != col) for (int q = 0; q < 4; ++q) { long double t = M[col][q]; M[col][q] = M[piv][q]; M[piv][q] = t; }
        for (int r = 0; r < 3; ++r) {
            if (r == col) continue;
            const long double f = M[r][col] / M[col][col];
            for (int q = col; q < 4; ++q) M[r][q] -= f * M[col][q];
        }
    }
    for (int r = 0; r < 3; ++r) c[r] = (double)(M[r][3] / M[r][r]);
    return 0;
}
