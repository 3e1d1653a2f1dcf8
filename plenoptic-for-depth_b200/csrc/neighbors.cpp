// neighbors.cpp -- ordered neighbour lists for matching, host side.
//
// Restates the parts of SelectNeighbors::CollectMIANeighImagesForMatch
// (MINeighbor/SelectNeighbors.cpp:113-193) that fix the matching order when no
// candidate is rejected as an outlier:
//   * rings grown breadth-first from the lens: a lens joins ring r+1 when its
//     centre lies within |dist - pitch| < 0.15 pitch of a ring-r lens
//     (ComputeNearestCircleKeys / ConfirmNearestNeighKeys, :195-420);
//   * score = 1 - (b - b_min) / (b_max - b_min) over all collected candidates
//     (ComputeNeighborScoresForMatch with a = 1, b = c = 0, :770-832, and
//     MLA_Problem::ItemsNormalization / ComputeBaselineRatio,
//     MVStereo/LFDepthInfo.cpp:395-429);
//   * std::sort by descending score of the candidates listed in key order
//     (MLA_Problem::SortNeighScoreForMatch, LFDepthInfo.cpp:214-241), so ties
//     fall exactly as libstdc++ orders them in the reference.
// The similarity-driven RANSAC stop (MISimilarityMeasure::MeasureSimilarity,
// OutlierImpByRANSAC) is not applied here: all `rings` rings are collected.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <utility>
#include <vector>

#include "../../include/pfd_abi.h"
#include "../../include/pfd_host.h"

extern "C" pfd_status pfd_neighbors_by_baseline(const float* centers, const int* tilekeys, int n_views, float pitch,
                                                int rings, int max_nb, int* nb_ids, int* nb_counts)
{
    if (!centers || !tilekeys || !nb_ids || !nb_counts || n_views <= 0 || !(pitch > 0.0f) || rings < 1 ||
        max_nb < 1 || max_nb > 32)
        return PFD_EINVAL;
    // key (row, col) -> view, ordered like QuadTreeTileKey (LOD, Y, X)
    std::map<std::pair<int, int>, int> by_key;
    for (int v = 0; v < n_views; ++v) by_key[{ tilekeys[2 * v + 1], tilekeys[2 * v] }] = v;
    const float delt = 0.15f * pitch;

    for (int v = 0; v < n_views; ++v) {
        std::map<std::pair<int, int>, int> seen;     // key -> ring
        seen[{ tilekeys[2 * v + 1], tilekeys[2 * v] }] = 0;
        std::vector<int> frontier{ v };
        std::map<std::pair<int, int>, float> cand;   // key-ordered candidates -> baseline
        for (int r = 1; r <= rings && !frontier.empty(); ++r) {
            std::vector<int> next;
            for (int c : frontier) {
                const float cx = centers[2 * c], cy = centers[2 * c + 1];
                const int col = tilekeys[2 * c], row = tilekeys[2 * c + 1];
                for (int drow = -1; drow <= 1; ++drow)
                    for (int dcol = -2; dcol <= 2; ++dcol) {
                        auto it = by_key.find({ row + drow, col + dcol });
                        if (it == by_key.end()) continue;
                        const int u = it->second;
                        const float ex = cx - centers[2 * u], ey = cy - centers[2 * u + 1];
                        const float dist = std::sqrt(ex * ex + ey * ey);
                        if (!(std::fabs(dist - pitch) < delt)) continue;
                        const std::pair<int, int> key{ tilekeys[2 * u + 1], tilekeys[2 * u] };
                        if (seen.count(key)) continue;
                        seen[key] = r;
                        next.push_back(u);
                        const float bx = centers[2 * u] - centers[2 * v], by = centers[2 * u + 1] - centers[2 * v + 1];
                        cand[key] = std::sqrt(bx * bx + by * by);
                    }
            }
            frontier.swap(next);
        }
        float bmin = 1e30f, bmax = -1e30f;
        for (auto& kv : cand) { bmin = std::min(bmin, kv.second); bmax = std::max(bmax, kv.second); }
        std::vector<std::pair<std::pair<int, int>, float>> score;
        for (auto& kv : cand) {
            const float range = bmax - bmin;
            const float ratio = (range == 0.0f) ? 0.0f : std::fabs(kv.second - bmin) / range;
            const float s = 1.00f * (float)(1.0 - ratio);
            score.push_back({ kv.first, s });
        }
        std::sort(score.begin(), score.end(), [](const auto& a, const auto& b) { return a.second > b.second; });
        int cnt = 0;
        for (int k = 0; k < max_nb; ++k) nb_ids[v * max_nb + k] = -1;
        for (auto& s : score) {
            if (cnt >= max_nb) break;
            nb_ids[v * max_nb + cnt++] = by_key[{ s.first.first, s.first.second }];
        }
        nb_counts[v] = cnt;
    }
    return PFD_OK;
}
