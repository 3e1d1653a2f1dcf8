/*
 * oracle/blur.c -- CPU restatement of the blur and richness channels of the
 * frame path.  TEST INFRASTRUCTURE ONLY; pinned to OpenCV's cv::Laplacian,
 * cv::threshold and saturating 8-bit conversion by the committed fixture
 * tests/golden/blur_cv.npz (tests/golden/make_blur_golden.py), and to
 * cv::normalize (NORM_MINMAX) by tests/golden/richness_cv.npz
 * (tests/golden/make_richness_golden.py).
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

#include <float.h>
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

/*
 * Richness channel.  ImageQualityEstimate::QuantizeRichnessByGLCM
 * (Util/ImageQualityEstimate.cpp:310-340): a float map, zero where no window
 * fits, and for every pixel with 4 <= row < H - 4 and 4 <= col < W - 4 the
 * value calculate_matrix (:659-682) gives for the 8x8 window whose top-left
 * corner is (col - 4, row - 4): an 8x8 float GLCM counting the pairs
 * (m(r, c) / 32, m(r + 1, c + 1) / 32) for r, c in 0..6 (integer division of the
 * 8-bit gray), and its contrast, the sum over i then j of glcm(i, j) * (i - j)^2
 * in float.  Then cv::normalize(map, map, 0, 255, NORM_MINMAX): min and max of
 * the map in double, scale = (float)((255 - 0) * (1 / (max - min))) (0 when
 * max - min <= DBL_EPSILON), shift = (float)0 - (float)(min * scale), every
 * value v -> v * scale + shift in float.
 */
void orc_glcm_contrast(const uint8_t* gray, int W, int H, int pitch, float* score)
{
    for (size_t i = 0; i < (size_t)W * H; ++i) score[i] = 0.0f;
    for (int row = 4; row < H - 4; ++row)
        for (int col = 4; col < W - 4; ++col) {
            const uint8_t* m = gray + (size_t)(row - 4) * pitch + (col - 4);
            float glcm[8][8];
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) glcm[i][j] = 0.0f;
            for (int r = 0; r < 7; ++r)
                for (int c = 0; c < 7; ++c) {
                    const int i = m[(size_t)r * pitch + c] / 32;
                    const int j = m[(size_t)(r + 1) * pitch + c + 1] / 32;
                    glcm[i][j] += 1.0f;
                }
            float contrast = 0.0f;
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) contrast += glcm[i][j] * (float)((i - j) * (i - j));
            score[(size_t)row * W + col] = contrast;
        }
}

void orc_normalize_minmax(float* map, size_t n, double lo, double hi)
{
    if (n == 0) return;
    double smin = map[0], smax = map[0];
    for (size_t i = 1; i < n; ++i) {
        if (map[i] < smin) smin = map[i];
        if (map[i] > smax) smax = map[i];
    }
    const double dmin = lo < hi ? lo : hi, dmax = lo < hi ? hi : lo;
    const double s = (dmax - dmin) * (smax - smin > DBL_EPSILON ? 1.0 / (smax - smin) : 0.0);
    const float scale = (float)s;
    const float shift = (float)dmin - (float)(smin * scale);
    for (size_t i = 0; i < n; ++i) {
        const float p = map[i] * scale;
        map[i] = p + shift;
    }
}

/*
 * DepthSolver::SliceAndIndicatlizeForMI (DepthSolver.cpp:2709-2754) on the
 * normalised map: cv::threshold(map, 10, 255, THRESH_BINARY), every view's
 * window of it copied into the 8-bit MLA_Problem::m_Image_Richness (saturating
 * conversion: 0 or 255), and MLA_Problem::ComputeRichnessValue
 * (MVStereo/LFDepthInfo.cpp:86-104) counts its 255s.  DepthSolver::
 * GetRichnessScoreMI (:2307-2326) gives the window of the normalised map.
 * score_tiles [V][mi_h][mi_w], binary [V][mi_h][mi_w] and counts [V] may each
 * be NULL.  Returns 0, or -1 for a window outside the frame or no memory.
 */
int orc_richness_tiles(const uint8_t* gray, int W, int H, int pitch, const int* origin, int V, int mi_w, int mi_h,
                       float* score_tiles, uint8_t* binary, uint32_t* counts)
{
    float* score = (float*)malloc(sizeof(float) * ((size_t)W * H + 1));
    if (!score) return -1;
    orc_glcm_contrast(gray, W, H, pitch, score);
    orc_normalize_minmax(score, (size_t)W * H, 0.0, 255.0);
    for (int v = 0; v < V; ++v) {
        const int x0 = origin[2 * v], y0 = origin[2 * v + 1];
        if (x0 < 0 || y0 < 0 || x0 + mi_w > W || y0 + mi_h > H) { free(score); return -1; }
        uint32_t n = 0;
        for (int y = 0; y < mi_h; ++y)
            for (int x = 0; x < mi_w; ++x) {
                const float s = score[(size_t)(y0 + y) * W + (x0 + x)];
                const uint8_t b = saturate_u8(s > 10.0f ? 255.0f : 0.0f);
                const size_t t = ((size_t)v * mi_h + y) * mi_w + x;
                if (score_tiles) score_tiles[t] = s;
                if (binary) binary[t] = b;
                if (b == 255) ++n;
            }
        if (counts) counts[v] = n;
    }
    free(score);
    return 0;
}
