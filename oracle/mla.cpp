/*
 * oracle/mla.cpp -- CPU restatement of the micro-lens centre detection
 * DepthSolver::ComputeMLACentersFromWhiteImage (DepthSolver.cpp:710-870) with
 * its Otsu threshold (DepthSolver::Otsu, :486-546).  TEST INFRASTRUCTURE ONLY.
 *
 * The OpenCV 4.2 steps it calls are restated from their published
 * definitions and pinned against the Python cv2 present here (4.13) by
 * tests/test_mla_cpu.py:
 *   cvtColor(BGR2GRAY) on 8 bits: (3735 B + 19235 G + 9798 R + 16384) >> 15, the
 *   15-bit fixed point of OpenCV 4's 8-bit path (cv2 4.13 agrees on every value);
 *   threshold(THRESH_BINARY): 255 where gray > t;
 *   findContours(RETR_EXTERNAL, CHAIN_APPROX_SIMPLE): the outer border of
 *   each 8-connected foreground component, traced by Suzuki-Abe border
 *   following from the component's first pixel in raster order, contours
 *   listed in reverse order of discovery (components inside holes of other
 *   components are not expected in a white image and are listed too);
 *   moments(contour): polygon moments by Green's theorem, integer-exact
 *   sums in double scaled by 1/2 and 1/6 (signed by the orientation), so
 *   collinear points removed by CHAIN_APPROX_SIMPLE change nothing;
 *   contourArea: |shoelace sum| / 2.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <vector>

#include "pfd_oracle.h"

namespace {

struct Contour {
    double a00 = 0, a10 = 0, a01 = 0;
};

// 8 directions counter-clockwise on screen (rows grow downwards)
const int DR[8] = { 0, -1, -1, -1, 0, 1, 1, 1 };
const int DC[8] = { 1, 1, 0, -1, -1, -1, 0, 1 };

int dir_of(int dr, int dc)
{
    for (int d = 0; d < 8; ++d)
        if (DR[d] == dr && DC[d] == dc) return d;
    return -1;
}

// Suzuki-Abe outer border following from start (r0, c0), the first pixel of
// its component in raster order; accumulates the polygon sums over the
// closed vertex sequence.
Contour trace(const std::vector<uint8_t>& fg, int W, int H, int r0, int c0)
{
    auto on = [&](int r, int c) { return r >= 0 && r < H && c >= 0 && c < W && fg[(size_t)r * W + c]; };
    std::vector<std::pair<int, int>> pts;
    pts.push_back({ c0, r0 });
    // (3.1) clockwise from the left neighbour for the first foreground pixel
    int d1 = -1;
    for (int k = 0; k < 8; ++k) {
        const int d = (4 - k + 8) & 7;
        if (on(r0 + DR[d], c0 + DC[d])) { d1 = d; break; }
    }
    Contour C;
    if (d1 >= 0) {
        const int r1 = r0 + DR[d1], c1 = c0 + DC[d1];
        int r2 = r1, c2 = c1, r3 = r0, c3 = c0;
        for (long step = 0; step < 4L * W * H + 8; ++step) {
            // (3.3) counter-clockwise around (r3, c3), from the element after (r2, c2)
            const int d2 = dir_of(r2 - r3, c2 - c3);
            int r4 = r3, c4 = c3;
            for (int k = 1; k <= 8; ++k) {
                const int d = (d2 + k) & 7;
                if (on(r3 + DR[d], c3 + DC[d])) { r4 = r3 + DR[d]; c4 = c3 + DC[d]; break; }
            }
            // (3.5)
            if (r4 == r0 && c4 == c0 && r3 == r1 && c3 == c1) break;
            r2 = r3; c2 = c3; r3 = r4; c3 = c4;
            pts.push_back({ c3, r3 });
        }
    }
    const size_t n = pts.size();
    double xp = pts[n - 1].first, yp = pts[n - 1].second;
    for (size_t i = 0; i < n; ++i) {
        const double x = pts[i].first, y = pts[i].second;
        const double dxy = xp * y - x * yp;
        C.a00 += dxy;
        C.a10 += dxy * (xp + x);
        C.a01 += dxy * (yp + y);
        xp = x; yp = y;
    }
    return C;
}

}  // namespace

extern "C" int orc_mla_otsu(const uint8_t* bgr, int W, int H, int step)
{
    // DepthSolver::Otsu: the first W bytes of every row of the 3-channel image
    long count[256] = { 0 };
    for (int i = 0; i < H; ++i)
        for (int j = 0; j < W; ++j) count[bgr[(size_t)i * step + j]]++;
    const int sum = W * H;
    float pro[256];
    for (int i = 0; i < 256; ++i) pro[i] = (float)count[i] / (float)sum;
    float deltaMax = 0;
    int threshold = 0;
    for (int i = 0; i < 256; ++i) {
        float w0 = 0, w1 = 0, u0tmp = 0, u1tmp = 0;
        for (int j = 0; j < 256; ++j) {
            if (j <= i) { w0 += pro[j]; u0tmp += j * pro[j]; }
            else { w1 += pro[j]; u1tmp += j * pro[j]; }
        }
        const float u0 = u0tmp / w0, u1 = u1tmp / w1, u = u0tmp + u1tmp;
        const float deltaTmp = w0 * (u0 - u) * (u0 - u) + w1 * (u1 - u) * (u1 - u);
        if (deltaTmp > deltaMax) { deltaMax = deltaTmp; threshold = i; }
    }
    return threshold;
}

// Contours of the thresholded gray image in OpenCV's order: centroid (float,
// -1 when m00 == 0) and area.  Returns the count, or -1 when max_out is too small.
extern "C" int orc_mla_contours(const uint8_t* bgr, int W, int H, int step, int threshold, float* cx, float* cy,
                                double* area, int max_out)
{
    std::vector<uint8_t> fg((size_t)W * H);
    for (int r = 0; r < H; ++r)
        for (int c = 0; c < W; ++c) {
            const uint8_t* p = bgr + (size_t)r * step + 3 * c;
            const int g = (p[0] * 3735 + p[1] * 19235 + p[2] * 9798 + 16384) >> 15;
            fg[(size_t)r * W + c] = g > threshold;
        }
    // components in raster order of their first pixel
    std::vector<int> comp((size_t)W * H, -1);
    std::vector<std::pair<int, int>> starts;
    std::vector<int> stack;
    for (int r = 0; r < H; ++r)
        for (int c = 0; c < W; ++c) {
            const size_t i = (size_t)r * W + c;
            if (!fg[i] || comp[i] >= 0) continue;
            const int id = (int)starts.size();
            starts.push_back({ r, c });
            comp[i] = id;
            stack.assign(1, (int)i);
            while (!stack.empty()) {
                const int q = stack.back();
                stack.pop_back();
                const int qr = q / W, qc = q % W;
                for (int d = 0; d < 8; ++d) {
                    const int nr = qr + DR[d], nc = qc + DC[d];
                    if (nr < 0 || nr >= H || nc < 0 || nc >= W) continue;
                    const size_t k = (size_t)nr * W + nc;
                    if (fg[k] && comp[k] < 0) { comp[k] = id; stack.push_back((int)k); }
                }
            }
        }
    const int n = (int)starts.size();
    if (n > max_out) return -1;
    for (int k = 0; k < n; ++k) {
        const int s = n - 1 - k;                  // reverse order of discovery
        const Contour C = trace(fg, W, H, starts[s].first, starts[s].second);
        double m00 = 0, m10 = 0, m01 = 0;
        if (std::fabs(C.a00) > 1.1920928955078125e-07) {
            const double h = C.a00 > 0 ? 0.5 : -0.5;
            const double s6 = C.a00 > 0 ? 1.0 / 6.0 : -1.0 / 6.0;
            m00 = C.a00 * h;
            m10 = C.a10 * s6;
            m01 = C.a01 * s6;
        }
        float x = -1, y = -1;
        if (m00 != 0) { x = (float)(m10 / m00); y = (float)(m01 / m00); }
        cx[k] = x;
        cy[k] = y;
        area[k] = std::fabs(C.a00 * 0.5);
    }
    return n;
}

// The rest of ComputeMLACentersFromWhiteImage (:752-868): position filter,
// rows by running mean y, columns by x, small-area flag.  Outputs one entry
// per map key, in key order (row, then column): col, row, centre, area,
// abandon.  Returns the entry count, or -1.
extern "C" int orc_mla_centers(const uint8_t* bgr, int W, int H, int step, float baseline, int mla_u_size,
                               int mla_v_size, int* out_col, int* out_row, float* out_cx, float* out_cy,
                               float* out_area, int* out_abandon, int max_out, int* threshold_out)
{
    const int t = orc_mla_otsu(bgr, W, H, step);
    if (threshold_out) *threshold_out = t;
    const int cap = W * H / 2 + 1;
    std::vector<float> cx(cap), cy(cap);
    std::vector<double> area(cap);
    const int nc = orc_mla_contours(bgr, W, H, step, t, cx.data(), cy.data(), area.data(), cap);
    if (nc < 0) return -1;
    // MLA_Info holds its area as a float (SetArea(float), Common/CommonUtil.h:48)
    struct Info { float x, y; float area; int col = 0, row = 0; bool abandon = false; };
    std::vector<Info> infos;
    double average_area = 0.0;
    for (int k = 0; k < nc; ++k) {
        const float x = cx[k], y = cy[k];
        if (y >= baseline * 0.5 && y <= baseline * mla_v_size && x >= baseline * 0.5 && x <= baseline * mla_u_size) {
            average_area += area[k];
            infos.push_back({ x, y, (float)area[k] });
        }
    }
    average_area /= nc;
    std::map<int, std::vector<int>> rows;
    float y_ideal_next = 0.0f;
    int y_ideal_next_count = 0;
    for (int row = 0; row < mla_v_size; ++row) {
        std::vector<int> members;
        float y_ideal = 0.0f;
        if (row == 0) {
            y_ideal = baseline * 0.5;
        } else {
            y_ideal = y_ideal_next / y_ideal_next_count;
            y_ideal += baseline;
            y_ideal_next = 0.0f;
            y_ideal_next_count = 0;
        }
        for (int i = 0; i < (int)infos.size(); ++i) {
            if (std::fabs(infos[i].y - y_ideal) < baseline * 0.5) {
                members.push_back(i);
                y_ideal_next += infos[i].y;
                y_ideal_next_count++;
            }
        }
        std::map<float, int> by_x;
        for (int i = 0; i < (int)members.size(); ++i) by_x[infos[members[i]].x] = i;
        std::vector<int> sorted;
        for (auto& kv : by_x) sorted.push_back(members[kv.second]);
        rows[row] = sorted;
    }
    std::map<std::pair<int, int>, int> keyed;           // (row, col) -> info
    for (auto& kv : rows)
        for (int col = 0; col < (int)kv.second.size(); ++col) {
            Info& I = infos[kv.second[col]];
            I.col = col;
            I.row = kv.first;
            I.abandon = I.area < average_area * 0.8;
            keyed[{ kv.first, col }] = kv.second[col];
        }
    if ((int)keyed.size() > max_out) return -1;
    int n = 0;
    for (auto& kv : keyed) {
        const Info& I = infos[kv.second];
        out_col[n] = kv.first.second;
        out_row[n] = kv.first.first;
        out_cx[n] = I.x;
        out_cy[n] = I.y;
        out_area[n] = I.area;
        out_abandon[n] = I.abandon;
        ++n;
    }
    return n;
}
