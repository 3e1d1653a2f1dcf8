// neighbors_impl.h -- the per-view selection of neighbors.h (a template over
// the similarity source).
//
// Types follow the reference's: baselines are floats computed through double
// std::pow / std::sqrt; the RANSAC sums are floats; the thresholds 2 (or 1) x
// pitch x 1.05 are stored in floats; the score a (1.0 - ratio) + ... is formed
// in double and stored in a float; the sort is std::sort over the key-ordered
// candidates, so ties fall as libstdc++ orders them.
#pragma once
#include <algorithm>
#include <cmath>
#include <map>
#include <utility>

namespace pfd {

inline float lens_baseline(const LensGrid& G, int a, int b)
{
    return (float)std::sqrt(std::pow((double)(G.cx[b] - G.cx[a]), 2) + std::pow((double)(G.cy[b] - G.cy[a]), 2));
}

template <class Sim>
void select_for_view(const LensGrid& G, float pitch, int v, const std::vector<std::vector<int>>& rings, Sim sim,
                     std::vector<int>& out)
{
    struct Entry { int view; float similarity, baseline; };
    std::map<std::pair<int, int>, Entry> scores;          // m_NeighScoreMapForMatch, key (row, column)
    float bmax = 0.0f;                                     // m_NeigDistance_range_forMatch (.x stays 0)
    bool ransac = false;
    float slope = 0.0f, icpt = 0.0f;
    int circle = 0;
    bool stop = false;
    while (!stop && circle < (int)rings.size()) {
        if (circle == 2 && scores.size() >= 2) {           // MLA_Problem::RansacNeighborKeyForMatch (LFDepthInfo.cpp:136-189)
            const float bthr = 2 * (pitch * 1.05);
            float sx = 0, sy = 0, sxx = 0, sxy = 0;
            int N = 0;
            for (auto& kv : scores)
                if (kv.second.baseline < bthr) {
                    const float x = kv.second.baseline, y = kv.second.similarity;
                    sx += x; sy += y; sxx += x * x; sxy += x * y;
                    ++N;
                }
            const float den = N * sxx - sx * sx;
            if (!(std::fabs(den) < 1e-6)) {
                slope = (N * sxy - sx * sy) / den;
                icpt = (sy - slope * sx) / N;
                ransac = true;
            }
        }
        // ComputeCandidateNeighborScoresForMatch (SelectNeighbors.cpp:558-641)
        const std::vector<int>& ring = rings[circle];
        int outliers = 0;
        for (size_t i = 0; i < ring.size(); ++i) {
            const int n = ring[i];
            const float s = sim(circle, (int)i);
            const float b = lens_baseline(G, v, n);
            if (ransac) {                                  // MLA_Problem::OutlierImpByRANSAC (LFDepthInfo.cpp:191-211)
                const float pred = slope * b + icpt;
                float err = std::fabs(s - pred);
                err /= s;
                const float bcrit = 1 * (pitch * 1.05);
                if (b > bcrit && err > 0.1f) { ++outliers; continue; }
            }
            scores[{ G.row[n], G.col[n] }] = { n, s, b };
            if (bmax < b) bmax = b;
        }
        stop = outliers >= 2;
        if (circle > 1 && stop) break;
        ++circle;
    }
    // ItemsNormalization + ComputeNeighborScoresForMatch (a = 1, b = c = 0) + SortNeighScoreForMatch
    std::vector<std::pair<int, float>> sv;
    sv.reserve(scores.size());
    for (auto& kv : scores) {
        const float range = bmax - 0.0f;
        const float ratio = (range == 0.0f) ? 0.0f : std::fabs(kv.second.baseline - 0.0f) / range;
        const float a = 1.00f, bw = 0.0f, cw = 0.0f;
        const float score = a * (1.0 - ratio) + bw * 0.0f + cw * 1.0f;
        sv.push_back({ kv.second.view, score });
    }
    std::sort(sv.begin(), sv.end(), [](const std::pair<int, float>& x, const std::pair<int, float>& y) {
        return x.second > y.second;
    });
    out.clear();
    for (auto& e : sv) out.push_back(e.first);
}

}  // namespace pfd
