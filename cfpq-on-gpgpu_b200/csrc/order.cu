// Vertex-order heuristic (host code): cfpq_order_suggest.
//
// Tile skipping only pays off when the bits of the nonterminal matrices fall
// into few 64x64 tiles.  Graphs whose vertex ids carry no locality (RDF-like
// data with arbitrary numbering) spread even a small result over almost every
// tile.  The heuristic:
//   1. If at least half of the edges join vertices whose ids are in the same
//      or a neighbouring 64-block, the ids already have locality: identity.
//   2. Otherwise group vertices by their label signature (which labels occur
//      on their outgoing and on their incoming edges), and order every group
//      by breadth-first discovery over the undirected graph, BFS seeds taken
//      by decreasing degree.  Vertices with the same role (classes vs.
//      instances in an ontology) become contiguous, and BFS keeps neighbours
//      close within a role.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "cfpq_b200.h"

extern "C" int cfpq_order_suggest(uint32_t n, const uint32_t *from, const uint32_t *label, const uint32_t *to,
                                  size_t nedges, uint32_t *perm_out) {
    if (!perm_out || (nedges && (!from || !to || !label))) return CFPQ_ERR_INVALID;
    for (uint32_t v = 0; v < n; ++v) perm_out[v] = v;
    if (n == 0 || nedges == 0) return CFPQ_OK;
    size_t local = 0;
    for (size_t e = 0; e < nedges; ++e) {
        if (from[e] >= n || to[e] >= n) return CFPQ_ERR_INVALID;
        const int64_t d = (int64_t)(from[e] / 64) - (int64_t)(to[e] / 64);
        if (d >= -1 && d <= 1) ++local;
    }
    if (2 * local >= nedges) return CFPQ_OK;

    // signatures
    std::vector<uint64_t> sig(n, 0);
    std::vector<uint32_t> deg(n, 0);
    for (size_t e = 0; e < nedges; ++e) {
        const uint32_t l = label[e] % 31;
        sig[from[e]] |= 1ULL << (2 * l);
        sig[to[e]] |= 1ULL << (2 * l + 1);
        ++deg[from[e]];
        ++deg[to[e]];
    }
    // undirected CSR
    std::vector<uint32_t> start(n + 1, 0);
    for (size_t e = 0; e < nedges; ++e) {
        if (from[e] == to[e]) continue;
        ++start[from[e] + 1];
        ++start[to[e] + 1];
    }
    for (uint32_t v = 0; v < n; ++v) start[v + 1] += start[v];
    std::vector<uint32_t> adj(start[n]);
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (size_t e = 0; e < nedges; ++e) {
        if (from[e] == to[e]) continue;
        adj[fill[from[e]]++] = to[e];
        adj[fill[to[e]]++] = from[e];
    }
    // BFS discovery index, seeds by decreasing degree
    std::vector<uint32_t> seeds(n);
    std::iota(seeds.begin(), seeds.end(), 0u);
    std::stable_sort(seeds.begin(), seeds.end(), [&](uint32_t a, uint32_t b) { return deg[a] > deg[b]; });
    const uint32_t kUnseen = 0xffffffffu;
    std::vector<uint32_t> bfs(n, kUnseen), queue;
    queue.reserve(n);
    uint32_t next = 0;
    for (uint32_t s : seeds) {
        if (bfs[s] != kUnseen) continue;
        bfs[s] = next++;
        queue.clear();
        queue.push_back(s);
        for (size_t h = 0; h < queue.size(); ++h) {
            const uint32_t v = queue[h];
            for (uint32_t i = start[v]; i < start[v + 1]; ++i) {
                const uint32_t w = adj[i];
                if (bfs[w] == kUnseen) {
                    bfs[w] = next++;
                    queue.push_back(w);
                }
            }
        }
    }
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return sig[a] != sig[b] ? sig[a] < sig[b] : bfs[a] < bfs[b];
    });
    for (uint32_t i = 0; i < n; ++i) perm_out[order[i]] = i;
    return CFPQ_OK;
}
