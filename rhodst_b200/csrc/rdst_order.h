// rdst_order.h -- the row order of the subdomain factorisations (host code
// shared by the B200 library and the CPU oracle).
//
// With "ilu.order bfs" (the default once the cells are split into more
// than one subdomain) the rows of each subdomain are factorised in
// breadth-first order of the subdomain's cell graph, the Cuthill-McKee
// family of orders that foam's renumberMesh gives a mesh before a run:
// the start is a pseudo-peripheral cell (two breadth-first sweeps from the
// component's lowest-numbered cell, each restarting from the lowest-numbered
// cell of the deepest level; George and Liu 1979), and cells of one level
// follow in ascending number.  Every coupling of a bipartite cell graph
// (hexahedra) joins consecutive levels, so the wavefront levels of the
// factorisation are the breadth-first levels and each row depends only on
// the level before it.  In mesh order ("natural") a subdomain cut out of a
// curvilinear mesh keeps couplings between its first and last wavefront
// levels (across an O-mesh seam, along the cut), which a factorisation
// applied level by level must read back from far behind.
//
// A subdomain whose cells form several components orders them one after
// the other, by their lowest-numbered cell.
#pragma once

#include <algorithm>
#include <vector>

namespace rdst {

// rank[i] = position of cell i in its subdomain's factorisation order.
// adj[i]: the cells sharing an internal face with i (any order, repeats
// allowed); part[i]: subdomain of cell i.  Couplings between subdomains are
// ignored.
inline std::vector<int> subdomain_bfs_rank(const std::vector<std::vector<int>>& adj, const std::vector<int>& part) {
    const int n = (int)adj.size();
    int np = 0;
    for (int i = 0; i < n; ++i) np = std::max(np, part[i] + 1);
    std::vector<std::vector<int>> members(np);
    for (int i = 0; i < n; ++i) members[part[i]].push_back(i);
    std::vector<int> rank(n, -1), dist(n, -1), seen(n, 0), q;
    q.reserve(n);
    // breadth-first levels from s over s's component (cells of comp); the
    // lowest-numbered cell of the deepest level
    auto sweep = [&](int s, const std::vector<int>& comp) {
        for (int i : comp) dist[i] = -1;
        q.clear();
        q.push_back(s);
        dist[s] = 0;
        for (size_t h = 0; h < q.size(); ++h) {
            const int u = q[h];
            for (int v : adj[u])
                if (part[v] == part[s] && dist[v] < 0) { dist[v] = dist[u] + 1; q.push_back(v); }
        }
        int far = s;
        for (int i : comp)
            if (dist[i] > dist[far] || (dist[i] == dist[far] && i < far)) far = i;
        return far;
    };
    for (int p = 0; p < np; ++p) {
        int next_rank = 0;
        for (int s0 : members[p]) {          // ascending: each component from its lowest cell
            if (seen[s0]) continue;
            // the component of s0
            std::vector<int> comp;
            q.clear();
            q.push_back(s0);
            seen[s0] = 1;
            for (size_t h = 0; h < q.size(); ++h) {
                const int u = q[h];
                comp.push_back(u);
                for (int v : adj[u])
                    if (part[v] == p && !seen[v]) { seen[v] = 1; q.push_back(v); }
            }
            std::sort(comp.begin(), comp.end());
            const int start = sweep(sweep(comp.front(), comp), comp);
            sweep(start, comp);
            std::sort(comp.begin(), comp.end(), [&](int a, int b) {
                return dist[a] != dist[b] ? dist[a] < dist[b] : a < b;
            });
            for (int i : comp) rank[i] = next_rank++;
        }
    }
    return rank;
}

}  // namespace rdst
