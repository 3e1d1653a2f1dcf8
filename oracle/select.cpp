/*
 * oracle/select.cpp -- CPU restatement of the matching-neighbour selection
 * SelectNeighbors::CollectMIANeighImagesForMatch (MINeighbor/SelectNeighbors.cpp:
 * 113-193) with its ring search (ComputeNearestCircleKeys :195-365,
 * CollectCircleNeighborsKey :367-385, ConfirmNearestNeighKeys :387-417,
 * ConfirmNearestNeighKeysByHorizontal :925-978), candidate scoring
 * (ComputeCandidateNeighborScoresForMatch :558-641, ComputeNeighborScoresForMatch
 * :770-832), MISimilarityMeasure::MeasureSimilarity (Util/MISimilarityMeasure.cpp:
 * 173-284) and MLA_Problem's RANSAC line, outlier test, normalisation and sort
 * (MVStereo/LFDepthInfo.cpp:136-241,404-429).  TEST INFRASTRUCTURE ONLY.
 *
 * Arithmetic follows the reference's types: float where it declares float,
 * double where std::pow / std::sqrt of promoted values or double literals make
 * it double.  The unqualified abs() of the reference resolves to the float
 * overload (CUDA's crt/math_functions.h, pulled in through CommonCUDA.h, puts
 * std::abs into the global namespace).  The similarity's shift loop is an
 * OpenMP loop nested inside the per-micro-image parallel loop, so it runs on
 * one thread, in order; step k is evaluated at the shift step k - 1 left
 * behind (0 for steps 0 and 1).  cv::warpAffine(INTER_NEAREST) with a pure
 * translation (sx, sy) reads source pixel (x + floor((rnd(-1024 sx) + 512) /
 * 1024), floor((rnd(1024 (y - sy)) + 512) / 1024)), rnd rounding half to even,
 * 0 outside: OpenCV's 10-bit fixed point, pinned against cv2 by
 * tests/test_select_cpu.py.  Ties of std::sort fall as libstdc++ orders them.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <utility>
#include <vector>

#include "pfd_oracle.h"

namespace {

int to_int_x86(float x) { return std::fabs(x) < 2147483648.0f ? (int)x : (int)0x80000000; }
int round_x86(double x) { return std::fabs(x) < 2147483648.0 ? (int)std::lrint(x) : (int)0x80000000; }

// MeasureSimilarity on binary (0 / 255) images; dx, dy = c_neigh - c_src.
int similarity(const uint8_t* src, const uint8_t* nb, int W, int H, float dx, float dy)
{
    if (std::fabs(dx) < 5) dx = 0;
    if (std::fabs(dy) < 5) dy = 0;
    const float norm = std::sqrt(dx * dx + dy * dy);
    const float dxs = (dx / norm) * 2.0f, dys = (dy / norm) * 2.0f;
    int dxc = to_int_x86((float)W / std::fabs(dxs));
    int dyc = to_int_x86((float)H / std::fabs(dys));
    if (dxs == 0) dxc = 0;
    else if (dys == 0) dyc = 0;
    const int max_steps = (int)std::ceil((double)std::max(dxc, dyc));
    if (max_steps <= 0) return 0;
    std::vector<int> counts(max_steps, 0);
    float sx = 0.0f, sy = 0.0f;
    for (int step = 0; step < max_steps; ++step) {
        if (std::fabs(sx) >= W || std::fabs(sy) >= H) continue;
        const int X0 = round_x86((double)(-sx) * 1024.0) + 512;
        const int x1 = (int)std::max(0.0f, sx), y1 = (int)std::max(0.0f, sy);
        const int x2 = (int)std::floor(std::min((float)(W - 1), sx + W - 1));
        const int y2 = (int)std::floor(std::min((float)(H - 1), sy + H - 1));
        int c = 0;
        if (x2 >= x1 && y2 >= y1)
            for (int y = y1; y <= y2; ++y) {
                const int Y = (round_x86(((double)y + (double)(-sy)) * 1024.0) + 512) >> 10;
                for (int x = x1; x <= x2; ++x) {
                    const int X = (X0 + x * 1024) >> 10;
                    const uint8_t v = (X >= 0 && X < W && Y >= 0 && Y < H) ? nb[Y * W + X] : 0;
                    c += src[y * W + x] == v;
                }
            }
        counts[step] = c;
        sx = step * dxs;
        sy = step * dys;
    }
    return *std::max_element(counts.begin(), counts.end());
}

struct Lens {
    float cx, cy;
};

struct Grid {
    int u, v;
    std::vector<int> id;                      // [row][col] -> view or -1
    int at(int col, int row) const { return (col >= 0 && col < u && row >= 0 && row < v) ? id[(size_t)row * u + col] : -1; }
};

struct RingSearch {
    const Grid& G;
    const std::vector<Lens>& L;
    float pitch, delt;
    std::vector<char> seen;
    std::vector<int> touched;

    // ConfirmNearestNeighKeys
    bool confirm(const Lens& c, int col, int row, std::vector<int>& out)
    {
        const int n = G.at(col, row);
        if (n < 0) return false;
        const float dist = (float)std::sqrt(std::pow((double)(c.cx - L[n].cx), 2) + std::pow((double)(c.cy - L[n].cy), 2));
        if (std::fabs(dist - pitch) < delt) {
            if (!seen[n]) { seen[n] = 1; touched.push_back(n); out.push_back(n); }
            return true;
        }
        return false;
    }
    void horizontal(const Lens& c, int col, int row, std::vector<int>& out)
    {
        for (int x = col - 1; x > -1; --x)
            if (!confirm(c, x, row, out)) break;
        for (int x = col + 1; x < G.u; ++x)
            if (!confirm(c, x, row, out)) break;
    }
    void adjacent_row(const Lens& c, int col, int row, std::vector<int>& out)
    {
        if (confirm(c, col, row, out)) horizontal(c, col, row, out);
        else if (confirm(c, col - 1, row, out)) horizontal(c, col - 1, row, out);
        else if (confirm(c, col + 1, row, out)) horizontal(c, col + 1, row, out);
    }
    // ComputeNearestCircleKeys over the centre keys
    void ring(const std::vector<int>& centres, const std::vector<int>& cols, const std::vector<int>& rows,
              std::vector<int>& out)
    {
        for (int k : centres) {
            const Lens& c = L[k];
            const int col = cols[k], row = rows[k];
            if (row - 1 > -1) adjacent_row(c, col, row - 1, out);
            for (int x = col - 1; x > -1; --x)
                if (!confirm(c, x, row, out)) break;
            for (int x = col + 1; x < G.u; ++x)
                if (!confirm(c, x, row, out)) break;
            if (row + 1 < G.v) adjacent_row(c, col, row + 1, out);
        }
    }
};

struct Entry {
    float similarity, baseline;
};

}  // namespace

extern "C" int orc_similarity(const uint8_t* src_bin, const uint8_t* nb_bin, int W, int H, float dx, float dy)
{
    return similarity(src_bin, nb_bin, W, H, dx, dy);
}

/* m_NeighsSortVecForMatch of every view (views = micro-images with a problem and
 * lens information; tilekeys (column, row) inside u_size x v_size).  images [V][mi_h][mi_w]
 * gray, or NULL for similarity 0 everywhere (no candidate is then rejected).
 * nb_ids [V][max_out] (-1 padded), nb_counts [V] the full list lengths, nb_sim
 * (may be NULL) the similarity of each listed neighbour.  Returns 0, or -1. */
extern "C" int orc_select_neighbors(int n_views, const float* centers, const int* tilekeys, int u_size, int v_size,
                                    float pitch, const uint8_t* images, int mi_w, int mi_h, int max_out,
                                    int* nb_ids, int* nb_counts, float* nb_sim)
{
    const int V = n_views;
    Grid G;
    G.u = u_size;
    G.v = v_size;
    G.id.assign((size_t)u_size * v_size, -1);
    std::vector<Lens> L(V);
    std::vector<int> cols(V), rows(V);
    for (int i = 0; i < V; ++i) {
        L[i] = { centers[2 * i], centers[2 * i + 1] };
        cols[i] = tilekeys[2 * i];
        rows[i] = tilekeys[2 * i + 1];
        if (cols[i] < 0 || cols[i] >= u_size || rows[i] < 0 || rows[i] >= v_size) return -1;
        G.id[(size_t)rows[i] * u_size + cols[i]] = i;
    }
    const size_t ppv = (size_t)mi_w * mi_h;
    std::vector<uint8_t> bin(images ? (size_t)V * ppv : 0);
    for (size_t i = 0; i < bin.size(); ++i) bin[i] = images[i] > 128 ? 255 : 0;   // threshold(128, BINARY)
    float delt = 0.15f;
    delt *= pitch;
    // views in parallel, as the reference's loop (SelectNeighbors.cpp:123, omp
    // parallel for, schedule(dynamic)); each thread has its own ring marks
#pragma omp parallel
    {
    RingSearch R{ G, L, pitch, delt, std::vector<char>(V, 0), {} };
#pragma omp for schedule(dynamic, 16)
    for (int v = 0; v < V; ++v) {
        for (int t : R.touched) R.seen[t] = 0;
        R.touched.clear();
        R.seen[v] = 1;
        R.touched.push_back(v);
        // the neighbour-score map, ordered by key (row, column)
        std::map<std::pair<int, int>, std::pair<int, Entry>> scores;
        float bmax = 0.0f;                            // m_NeigDistance_range_forMatch.y (x stays 0)
        bool ransac = false;
        float slope = 0, icpt = 0;
        std::vector<int> prev;
        int circle = 0;
        bool stop = false;
        while (!stop && circle < 5) {
            if (circle == 2 && scores.size() >= 2) {  // RansacNeighborKeyForMatch
                const float bthr = 2 * (pitch * 1.05);       // baselineThreshold is a float
                float sx = 0, sy = 0, sxx = 0, sxy = 0;
                int N = 0;
                for (auto& kv : scores) {
                    const Entry& e = kv.second.second;
                    if (e.baseline < bthr) {
                        sx += e.baseline; sy += e.similarity;
                        sxx += e.baseline * e.baseline; sxy += e.baseline * e.similarity;
                        ++N;
                    }
                }
                const float den = N * sxx - sx * sx;
                if (!(std::fabs(den) < 1e-6)) {
                    slope = (N * sxy - sx * sy) / den;
                    icpt = (sy - slope * sx) / N;
                    ransac = true;
                }
            }
            std::vector<int> ring;
            if (circle == 0) R.ring({ v }, cols, rows, ring);
            else R.ring(prev, cols, rows, ring);
            int outliers = 0;
            for (int n : ring) {
                float sim = 0.0f;
                if (images) {
                    const float dx = L[n].cx - L[v].cx, dy = L[n].cy - L[v].cy;
                    sim = (float)(double)similarity(&bin[(size_t)v * ppv], &bin[(size_t)n * ppv], mi_w, mi_h, dx, dy);
                }
                const float baseline =
                    (float)std::sqrt(std::pow((double)(L[n].cx - L[v].cx), 2) + std::pow((double)(L[n].cy - L[v].cy), 2));
                bool outlier = false;
                if (ransac) {                         // OutlierImpByRANSAC
                    const float pred = slope * baseline + icpt;
                    float err = std::fabs(sim - pred);
                    err /= sim;
                    const float bcrit = 1 * (pitch * 1.05);  // baselineCritical is a float
                    outlier = baseline > bcrit && err > 0.1f;
                }
                if (outlier) { ++outliers; continue; }
                scores[{ rows[n], cols[n] }] = { n, { sim, baseline } };
                if (bmax < baseline) bmax = baseline;
            }
            prev = ring;
            stop = outliers >= 2;
            if (circle > 1 && stop) break;
            ++circle;
        }
        // ItemsNormalization + ComputeNeighborScoresForMatch (a = 1, b = c = 0) + SortNeighScoreForMatch
        std::vector<std::pair<int, float>> sv;
        for (auto& kv : scores) {
            const float b = kv.second.second.baseline;
            const float range = bmax - 0.0f;
            const float ratio = range == 0.0f ? 0.0f : std::fabs(b - 0.0f) / range;
            const float a = 1.00f, bw = 0.0f, cw = 0.0f;
            const float score = a * (1.0 - ratio) + bw * 0.0f + cw * 1.0f;
            sv.push_back({ kv.second.first, score });
        }
        std::sort(sv.begin(), sv.end(), [](const std::pair<int, float>& x, const std::pair<int, float>& y) {
            return x.second > y.second;
        });
        const int n = (int)sv.size();
        nb_counts[v] = n;
        for (int k = 0; k < max_out; ++k) {
            nb_ids[(size_t)v * max_out + k] = k < n ? sv[k].first : -1;
            if (nb_sim) nb_sim[(size_t)v * max_out + k] = k < n ? scores[{ rows[sv[k].first], cols[sv[k].first] }].second.similarity : 0.0f;
        }
    }
    }
    return 0;
}
