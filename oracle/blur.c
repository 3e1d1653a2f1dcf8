/*
 * oracle/blur.c -- CPU restatement of the blur channel of the frame path.
 * TEST INFRASTRUCTURE ONLY; pinned to OpenCV's cv::Laplacian, cv::threshold and
 * saturating 8-bit conversion by the committed fixture tests/golden/blur_cv.npz
 * (tests/golden/make_blur_golden.py).
 *
 * ImageQualityEstimate::QuantizeBlurByLaplacian (Util/ImageQualityEstimate.cpp:
 * 211-230): score = cv::Laplacian(gray, CV_32F) with ksize 1, i.e. the 3x3
 * aperture 0 1 0 / 1 -4 1 / 0 1 0, scale 1, delta 0, default border (reflect
 * without repeating the edge).  DepthSolver::SliceAndIndicatlizeForMI
 * (DepthSolver.cpp:2709-2754): binary = cv::threshold(score, 10, 255,
 * THRESH_BINARY) (a float map), and for every micro-image the window at its
 * left-down corner of both maps is copied into the problem's cv::Mat_<uint8>
 * images; a copy into a fixed 8-bit type converts with saturate_cast (round to
 * nearest even, clamp to [0, 255]).  MLA_Problem::ComputeBlurenessValue
 * (MVStereo/LFDepthInfo.cpp:65-83) counts the 255s of the binary window.
 */
#include "pfd_oracle.h"

#include <math.h>
#include <stdlib.h>

static int reflect101(int p, int n)
{
    if (n == 1) return 0;
    while (p < 0 || p >= n) p = p < 0 ? -p : 2 * n - 2 - p;
    return p;
}

void orc_laplacian(const uint8_t* gray, int W, int H, int pitch, float* score)
{
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const float c = gray[(size_t)y * pitch + x];
            const float l = gray[(size_t)y * pitch + reflect101(x - 1, W)];
            const float r = gray[(size_t)y * pitch + reflect101(x + 1, W)];
            const float u = gray[(size_t)reflect101(y - 1, H) * pitch + x];
            const float d = gray[(size_t)reflect101(y + 1, H) * pitch + x];
            score[(size_t)y * W + x] = u + l + -4.0f * c + r + d;
        }
}

static uint8_t saturate_u8(float v)
{
    const long r = lrintf(v);            /* round to nearest even (default rounding mode) */
    return (uint8_t)(r < 0 ? 0 : (r > 255 ? 255 : r));
}

int orc_blur_tiles(const uint8_t* gray, int W, int H, int pitch, const int* origin, int V, int mi_w, int mi_h,
                   uint8_t* tiles, uint32_t* counts)
{
    float* score = (float*)malloc(sizeof(float) * (size_t)W * H);
    float* binary = (float*)malloc(sizeof(float) * (size_t)W * H);
    if (!score || !binary) { free(score); free(binary); return -1; }
    orc_laplacian(gray, W, H, pitch, score);
    for (size_t i = 0; i < (size_t)W * H; ++i) binary[i] = score[i] > 10.0f ? 255.0f : 0.0f;
    for (int v = 0; v < V; ++v) {
        const int x0 = origin[2 * v], y0 = origin[2 * v + 1];
        if (x0 < 0 || y0 < 0 || x0 + mi_w > W || y0 + mi_h > H) { free(score); free(binary); return -1; }
        uint32_t n = 0;
        for (int y = 0; y < mi_h; ++y)
            for (int x = 0; x < mi_w; ++x) {
                const size_t s = (size_t)(y0 + y) * W + (x0 + x);
                tiles[((size_t)v * mi_h + y) * mi_w + x] = saturate_u8(score[s]);
                if (saturate_u8(binary[s]) == 255) ++n;
            }
        if (counts) counts[v] = n;
    }
    free(score);
    free(binary);
    return 0;
}
