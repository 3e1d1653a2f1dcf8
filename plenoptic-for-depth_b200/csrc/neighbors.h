// neighbors.h -- matching-neighbour selection, host side (neighbors.cpp).
#pragma once
#include <cstdint>
#include <functional>
#include <vector>

namespace pfd {

// The lens layout SelectNeighbors searches: centres, (column, row) keys on a
// u_size x v_size grid.
struct LensGrid {
    int V = 0, u = 0, v = 0;
    std::vector<float> cx, cy;
    std::vector<int> col, row;
    std::vector<int> id;                          // [row][col] -> view, -1
    bool build(const float* centers, const int* tilekeys, int n_views, int u_size, int v_size);
};

// body(a, b) over [0, n) split into contiguous ranges, one host thread each
// (up to 32; one range for small n).
void parallel_views(int n, const std::function<void(int, int)>& body);

// The five rings of every view (ComputeNearestCircleKeys, SelectNeighbors.cpp:
// 195-365): rings[v][k] in the reference's push order.
void collect_rings(const LensGrid& G, float pitch, int n_rings, std::vector<std::vector<std::vector<int>>>& rings);

// CollectMIANeighImagesForMatch's per-view loop (SelectNeighbors.cpp:145-172)
// given the similarity of every ring candidate (sim(v, ring, index), in the
// order of collect_rings), then ComputeNeighborScoresForMatch and
// SortNeighScoreForMatch: the view's m_NeighsSortVecForMatch.
template <class Sim>
void select_for_view(const LensGrid& G, float pitch, int view, const std::vector<std::vector<int>>& rings, Sim sim,
                     std::vector<int>& out);

}  // namespace pfd

#include "neighbors_impl.h"
