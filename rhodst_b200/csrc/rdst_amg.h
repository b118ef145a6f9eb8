// rdst_amg.h -- the coarsening plan of the block AMG preconditioner and
// solver (host code shared by the B200 library and the CPU oracle).
//
// foam-extend registers BlockAMGPrecon and BlockAMGSolver for the 5x5 block
// matrix (libraries/vector5/Vector5typedefs/Vector5typedefs.C:1601-1708)
// with coefficient-based coarsening (BlockMatrixClustering/Selection); its
// sources are not vendored.  This path coarsens by plain aggregation of the
// cell graph (Vanek, Mandel and Brezina 1996), once per mesh: a pass that
// makes every cell whose neighbours are all free the root of an aggregate
// with them, then a pass that puts each remaining cell into the aggregate of
// its first aggregated neighbour.  Prolongation is piecewise constant, so a
// coarse block is the sum of the fine blocks between two aggregates
// (Galerkin P^T A P), rebuilt on the device every step from the step's
// matrix.  Coarsening stops at n_coarsest nodes, max_levels levels, or when
// a pass removes fewer than a tenth of the nodes.
#pragma once

#include <algorithm>
#include <vector>

namespace rdst {

struct AmgPlan {
    std::vector<int> n;                          // nodes per level, n[0] = cells
    std::vector<std::vector<int>> agg;           // agg[l][i]: node of level l+1 holding node i of level l
    std::vector<std::vector<std::vector<int>>> adj;   // adj[l][i]: neighbours of node i of level l, ascending
};

// one pass of plain aggregation; returns the number of aggregates
inline int amg_aggregate(const std::vector<std::vector<int>>& adj, std::vector<int>& agg) {
    const int n = (int)adj.size();
    agg.assign(n, -1);
    int na = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        bool all_free = true;
        for (int j : adj[i])
            if (agg[j] >= 0) { all_free = false; break; }
        if (!all_free) continue;
        agg[i] = na;
        for (int j : adj[i]) agg[j] = na;
        ++na;
    }
    const std::vector<int> first(agg);
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        for (int j : adj[i])
            if (first[j] >= 0) { agg[i] = first[j]; break; }
        if (agg[i] < 0) agg[i] = na++;           // no aggregated neighbour (not reached: a free cell is a root)
    }
    return na;
}

// cell graph (adjacency of the mesh's internal faces, original numbering)
// -> aggregation hierarchy
inline AmgPlan amg_plan(std::vector<std::vector<int>> adj0, int n_coarsest, int max_levels) {
    AmgPlan P;
    for (auto& v : adj0) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    P.n.push_back((int)adj0.size());
    P.adj.push_back(std::move(adj0));
    while ((int)P.n.size() < max_levels && P.n.back() > n_coarsest) {
        const auto& adj = P.adj.back();
        std::vector<int> agg;
        const int nc = amg_aggregate(adj, agg);
        if (nc * 10 > P.n.back() * 9) break;    // a pass that coarsens too little ends the hierarchy
        std::vector<std::vector<int>> cadj(nc);
        for (int i = 0; i < (int)adj.size(); ++i)
            for (int j : adj[i])
                if (agg[i] != agg[j]) cadj[agg[i]].push_back(agg[j]);
        for (auto& v : cadj) {
            std::sort(v.begin(), v.end());
            v.erase(std::unique(v.begin(), v.end()), v.end());
        }
        P.agg.push_back(std::move(agg));
        P.n.push_back(nc);
        P.adj.push_back(std::move(cadj));
    }
    return P;
}

}  // namespace rdst
