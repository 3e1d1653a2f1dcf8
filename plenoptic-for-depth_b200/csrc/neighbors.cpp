// neighbors.cpp -- matching-neighbour selection, host side.
//
// SelectNeighbors::CollectMIANeighImagesForMatch (MINeighbor/SelectNeighbors.cpp:
// 113-193) for every micro-image: rings of lenses at one pitch from the
// previous ring, found by the reference's walk over the key grid
// (ComputeNearestCircleKeys :195-365 with ConfirmNearestNeighKeys :387-417 and
// ConfirmNearestNeighKeysByHorizontal :925-978: the row above, tried at the
// same column, then one to the left, then one to the right, then walked
// sideways while lenses keep confirming; the own row walked both ways; the
// row below like the row above), then the per-view scoring of neighbors_impl.h.
// A lens confirms when |dist - pitch| < 0.15 pitch, dist computed in double
// and stored in a float; the unqualified abs of the reference is the float one
// (CUDA's math headers, included through its CommonCUDA.h, put std::abs into
// the global namespace).
//
// pfd_neighbors_by_baseline is the selection without similarities (every
// similarity 0, so no candidate is ever an outlier): the lists depend on the
// geometry only.  pfd_select_neighbors (pfd_abi.cu) adds the similarities,
// computed on the device.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <thread>
#include <vector>

#include "../../include/pfd_abi.h"
#include "../../include/pfd_host.h"
#include "neighbors.h"

namespace pfd {

bool LensGrid::build(const float* centers, const int* tilekeys, int n_views, int u_size, int v_size)
{
    V = n_views;
    u = u_size;
    v = v_size;
    cx.resize(V); cy.resize(V); col.resize(V); row.resize(V);
    id.assign((size_t)u * v, -1);
    for (int i = 0; i < V; ++i) {
        cx[i] = centers[2 * i];
        cy[i] = centers[2 * i + 1];
        col[i] = tilekeys[2 * i];
        row[i] = tilekeys[2 * i + 1];
        if (col[i] < 0 || col[i] >= u || row[i] < 0 || row[i] >= v) return false;
        if (id[(size_t)row[i] * u + col[i]] >= 0) return false;        // one lens per key
        id[(size_t)row[i] * u + col[i]] = i;
    }
    return true;
}

namespace {

struct Walk {
    const LensGrid& G;
    float pitch, delt;
    std::vector<char>& seen;
    std::vector<int>& touched;

    int at(int c, int r) const { return (c >= 0 && c < G.u && r >= 0 && r < G.v) ? G.id[(size_t)r * G.u + c] : -1; }
    bool confirm(int centre, int c, int r, std::vector<int>& out)
    {
        const int n = at(c, r);
        if (n < 0) return false;
        const float dist = lens_baseline(G, n, centre);
        if (std::fabs(dist - pitch) < delt) {
            if (!seen[n]) { seen[n] = 1; touched.push_back(n); out.push_back(n); }
            return true;
        }
        return false;
    }
    void sideways(int centre, int c, int r, std::vector<int>& out)
    {
        for (int x = c - 1; x > -1; --x)
            if (!confirm(centre, x, r, out)) break;
        for (int x = c + 1; x < G.u; ++x)
            if (!confirm(centre, x, r, out)) break;
    }
    void other_row(int centre, int c, int r, std::vector<int>& out)
    {
        if (confirm(centre, c, r, out)) sideways(centre, c, r, out);
        else if (confirm(centre, c - 1, r, out)) sideways(centre, c - 1, r, out);
        else if (confirm(centre, c + 1, r, out)) sideways(centre, c + 1, r, out);
    }
    void ring(const std::vector<int>& centres, std::vector<int>& out)
    {
        for (int k : centres) {
            const int c = G.col[k], r = G.row[k];
            if (r - 1 > -1) other_row(k, c, r - 1, out);
            for (int x = c - 1; x > -1; --x)
                if (!confirm(k, x, r, out)) break;
            for (int x = c + 1; x < G.u; ++x)
                if (!confirm(k, x, r, out)) break;
            if (r + 1 < G.v) other_row(k, c, r + 1, out);
        }
    }
};

}  // namespace

void parallel_views(int n, const std::function<void(int, int)>& body)
{
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<unsigned>(std::min(hw, 32u), (unsigned)std::max(1, n / 256));
    if (nt <= 1) { body(0, n); return; }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; ++t) {
        const int a = (int)((long long)n * t / nt), b = (int)((long long)n * (t + 1) / nt);
        th.emplace_back(body, a, b);
    }
    for (auto& x : th) x.join();
}

void collect_rings(const LensGrid& G, float pitch, int n_rings, std::vector<std::vector<std::vector<int>>>& rings)
{
    float delt = 0.15f;
    delt *= pitch;
    rings.assign(G.V, {});
    // views are independent: each thread walks its own range with its own marks
    parallel_views(G.V, [&](int a, int b) {
        std::vector<char> seen(G.V, 0);
        std::vector<int> touched;
        Walk W{ G, pitch, delt, seen, touched };
        for (int v = a; v < b; ++v) {
            for (int t : touched) seen[t] = 0;
            touched.clear();
            seen[v] = 1;
            touched.push_back(v);
            rings[v].assign(n_rings, {});
            for (int k = 0; k < n_rings; ++k) W.ring(k == 0 ? std::vector<int>{ v } : rings[v][k - 1], rings[v][k]);
        }
    });
}

}  // namespace pfd

extern "C" pfd_status pfd_neighbors_by_baseline(const float* centers, const int* tilekeys, int n_views, float pitch,
                                                int rings, int max_nb, int* nb_ids, int* nb_counts)
{
    if (!centers || !tilekeys || !nb_ids || !nb_counts || n_views <= 0 || !(pitch > 0.0f) || rings < 1 || rings > 5 ||
        max_nb < 1 || max_nb > 128)
        return PFD_EINVAL;
    int u = 0, v = 0;
    for (int i = 0; i < n_views; ++i) {
        if (tilekeys[2 * i] < 0 || tilekeys[2 * i + 1] < 0) return PFD_EINVAL;
        u = std::max(u, tilekeys[2 * i] + 1);
        v = std::max(v, tilekeys[2 * i + 1] + 1);
    }
    if ((long long)u * v > (1LL << 28)) return PFD_EINVAL;
    pfd::LensGrid G;
    if (!G.build(centers, tilekeys, n_views, u, v)) return PFD_EINVAL;
    std::vector<std::vector<std::vector<int>>> R;
    pfd::collect_rings(G, pitch, rings, R);
    pfd::parallel_views(n_views, [&](int a, int b) {
        std::vector<int> list;
        for (int i = a; i < b; ++i) {
            pfd::select_for_view(G, pitch, i, R[i], [](int, int) { return 0.0f; }, list);
            const int n = std::min((int)list.size(), max_nb);
            for (int k = 0; k < max_nb; ++k) nb_ids[(size_t)i * max_nb + k] = k < n ? list[k] : -1;
            nb_counts[i] = n;
        }
    });
    return PFD_OK;
}
