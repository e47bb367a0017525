// vbd_coloring.cpp -- vertex coloring of the particle conflict graph (host code).
//
// The reference colors the graph built by construct_particle_graph (graph_coloring.py:200-240)
// with Warp's native graph_coloring_assign / graph_coloring_balance (graph_coloring.py:287-294),
// whose source is not part of the reference tree.  This file restates the published algorithms
// the reference cites:
//   * MCS: maximum cardinality search ordering (Pereira & Palsberg, "Register allocation via
//     coloring of chordal graphs", APLAS 2005) followed by greedy first-fit coloring in that
//     order.  Ties between equally-weighted vertices are broken by the most recently raised
//     vertex (a LIFO bucket), which keeps the traversal local on meshes.
//   * GREEDY: first-fit coloring in order of decreasing degree (ties by index).
//   * balance: repeatedly move vertices out of the largest color into the smallest color that
//     none of their neighbours use, until max/min color size <= target ratio or no vertex moves.
// The exact assignment is not pinned by the reference (its tests check validity and balance
// only, test_coloring.py:101-236); the solver consumes color groups as input, so parity runs
// feed both sides the same groups.
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "vbd_internal.h"

namespace {

struct Csr {
    std::vector<int64_t> off;
    std::vector<int32_t> adj;
};

Csr build_csr(int n, int64_t m, const int32_t* edges) {
    Csr g;
    g.off.assign(static_cast<size_t>(n) + 1, 0);
    for (int64_t e = 0; e < m; ++e) {
        const int a = edges[2 * e], b = edges[2 * e + 1];
        if (a == b) continue;
        g.off[a + 1]++;
        g.off[b + 1]++;
    }
    for (int i = 0; i < n; ++i) g.off[i + 1] += g.off[i];
    g.adj.assign(static_cast<size_t>(g.off[n]), 0);
    std::vector<int64_t> fill(g.off.begin(), g.off.end() - 1);
    for (int64_t e = 0; e < m; ++e) {
        const int a = edges[2 * e], b = edges[2 * e + 1];
        if (a == b) continue;
        g.adj[fill[a]++] = b;
        g.adj[fill[b]++] = a;
    }
    return g;
}

std::vector<int> mcs_order(int n, const Csr& g) {
    std::vector<int> weight(n, 0);
    std::vector<char> done(n, 0);
    std::vector<std::vector<int>> bucket(1);
    bucket[0].reserve(n);
    for (int v = n - 1; v >= 0; --v) bucket[0].push_back(v);  // pops vertex 0 first
    int top = 0;
    std::vector<int> order;
    order.reserve(n);
    while (static_cast<int>(order.size()) < n) {
        while (top > 0 && bucket[top].empty()) --top;
        if (bucket[top].empty()) break;
        const int v = bucket[top].back();
        bucket[top].pop_back();
        if (done[v] || weight[v] != top) continue;  // stale entry
        done[v] = 1;
        order.push_back(v);
        for (int64_t k = g.off[v]; k < g.off[v + 1]; ++k) {
            const int u = g.adj[k];
            if (done[u]) continue;
            const int w = ++weight[u];
            if (w >= static_cast<int>(bucket.size())) bucket.resize(w + 1);
            bucket[w].push_back(u);
            if (w > top) top = w;
        }
    }
    return order;
}

std::vector<int> greedy_order(int n, const Csr& g) {
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (g.off[a + 1] - g.off[a]) > (g.off[b + 1] - g.off[b]);
    });
    return order;
}

int first_fit(int n, const Csr& g, const std::vector<int>& order, std::vector<int>& color) {
    color.assign(n, -1);
    std::vector<int> mark;
    int ncolors = 0;
    for (int v : order) {
        const int64_t deg = g.off[v + 1] - g.off[v];
        if (static_cast<int64_t>(mark.size()) < deg + 2) mark.resize(deg + 2, -1);
        for (int64_t k = g.off[v]; k < g.off[v + 1]; ++k) {
            const int c = color[g.adj[k]];
            if (c >= 0 && c <= deg) mark[c] = v;
        }
        int c = 0;
        while (mark[c] == v) ++c;
        color[v] = c;
        ncolors = std::max(ncolors, c + 1);
    }
    return ncolors;
}

void balance(int n, const Csr& g, std::vector<int>& color, int ncolors, float target) {
    if (ncolors < 2) return;
    std::vector<int64_t> size(ncolors, 0);
    for (int v = 0; v < n; ++v) size[color[v]]++;
    std::vector<char> used(ncolors, 0);
    for (int round = 0; round < 64 * ncolors; ++round) {
        int cmax = 0, cmin = 0;
        for (int c = 1; c < ncolors; ++c) {
            if (size[c] > size[cmax]) cmax = c;
            if (size[c] < size[cmin]) cmin = c;
        }
        if (size[cmin] > 0 && static_cast<double>(size[cmax]) / static_cast<double>(size[cmin]) <= target) return;
        bool moved = false;
        for (int v = 0; v < n && size[cmax] > size[cmin] + 1; ++v) {
            if (color[v] != cmax) continue;
            bool ok = true;
            for (int64_t k = g.off[v]; k < g.off[v + 1]; ++k)
                if (color[g.adj[k]] == cmin) {
                    ok = false;
                    break;
                }
            if (!ok) continue;
            color[v] = cmin;
            size[cmax]--;
            size[cmin]++;
            moved = true;
            if (size[cmin] > 0 && static_cast<double>(size[cmax]) / static_cast<double>(size[cmin]) <= target) break;
        }
        if (!moved) return;
    }
}

}  // namespace

extern "C" int vbd_color_graph(int32_t num_nodes, int64_t num_edges, const int32_t* edges, int32_t algorithm,
                               int32_t do_balance, float target_ratio, int32_t* colors_out, int32_t* num_colors_out) {
    if (num_nodes < 0 || num_edges < 0 || (num_edges > 0 && !edges) || (num_nodes > 0 && !colors_out) ||
        !num_colors_out)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_color_graph: invalid arguments");
    if (algorithm != 0 && algorithm != 1)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_color_graph: algorithm must be 0 (MCS) or 1 (GREEDY)");
    for (int64_t e = 0; e < 2 * num_edges; ++e)
        if (edges[e] < 0 || edges[e] >= num_nodes)
            return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_color_graph: edge endpoint out of range");
    *num_colors_out = 0;
    if (num_nodes == 0) return VBD_OK;
    const Csr g = build_csr(num_nodes, num_edges, edges);
    const std::vector<int> order = algorithm == 0 ? mcs_order(num_nodes, g) : greedy_order(num_nodes, g);
    std::vector<int> color;
    const int nc = first_fit(num_nodes, g, order, color);
    if (do_balance) balance(num_nodes, g, color, nc, target_ratio);
    for (int v = 0; v < num_nodes; ++v) colors_out[v] = color[v];
    *num_colors_out = nc;
    return VBD_OK;
}

// Canonical edge list of the conflict graph (the sort-unique step of graph_coloring.py:99-197):
// the unique (min, max) pairs of the pairs `for_each(visit)` emits, self-pairs dropped, in
// lexicographic order -- the order numpy.unique(axis=0) gives -- via a counting sort by the
// smaller endpoint and a sort of each (short) row.
template <typename ForEach>
static int64_t canonical_pairs(int32_t num_nodes, ForEach&& for_each, int32_t* edges_out) {
    std::vector<int64_t> off(static_cast<size_t>(num_nodes) + 1, 0);
    for_each([&](int a, int b) {
        if (a != b) ++off[static_cast<size_t>(std::min(a, b)) + 1];
    });
    for (int v = 0; v < num_nodes; ++v) off[v + 1] += off[v];
    std::vector<int32_t> nb(static_cast<size_t>(off[num_nodes]));
    std::vector<int64_t> cur(off.begin(), off.end() - 1);
    for_each([&](int a, int b) {
        if (a != b) nb[cur[std::min(a, b)]++] = std::max(a, b);
    });
    int64_t n = 0;
    for (int v = 0; v < num_nodes; ++v) {
        auto b = nb.begin() + off[v], e = nb.begin() + off[v + 1];
        std::sort(b, e);
        e = std::unique(b, e);
        for (auto it = b; it != e; ++it) {
            edges_out[2 * n] = v;
            edges_out[2 * n + 1] = *it;
            ++n;
        }
    }
    return n;
}

// ... of an explicit pair list
extern "C" int vbd_coloring_graph_edges(int32_t num_nodes, int64_t num_pairs, const int32_t* pairs, int32_t* edges_out,
                                        int64_t* num_edges_out) {
    if (num_nodes < 0 || num_pairs < 0 || (num_pairs > 0 && (!pairs || !edges_out)) || !num_edges_out)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_coloring_graph_edges: invalid arguments");
    for (int64_t k = 0; k < 2 * num_pairs; ++k)
        if (pairs[k] < 0 || pairs[k] >= num_nodes)
            return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_coloring_graph_edges: endpoint out of range");
    *num_edges_out = canonical_pairs(
        num_nodes,
        [&](auto&& visit) {
            for (int64_t k = 0; k < num_pairs; ++k) visit(pairs[2 * k], pairs[2 * k + 1]);
        },
        edges_out);
    return VBD_OK;
}

// The whole conflict-graph construction of construct_trimesh_graph_edges
// (graph_coloring.py:99-197) from the (already mask-filtered) element arrays: each triangle adds
// (a,b) (a,c) (b,c), each bending hinge all 6 pairs of its 4 vertices, pairs with a negative id
// skipped; the result is canonicalised as vbd_coloring_graph_edges does.  edges_out needs room for
// 3 nt + 6 nb pairs.
extern "C" int vbd_trimesh_graph_edges(int32_t num_nodes, const int32_t* tris, int64_t nt, const int32_t* bend,
                                       int64_t nb, int32_t* edges_out, int64_t* num_edges_out) {
    if (num_nodes < 0 || nt < 0 || nb < 0 || (nt > 0 && !tris) || (nb > 0 && !bend) ||
        ((nt > 0 || nb > 0) && !edges_out) || !num_edges_out)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_trimesh_graph_edges: invalid arguments");
    for (int64_t k = 0; k < 3 * nt; ++k)
        if (tris[k] < 0 || tris[k] >= num_nodes)
            return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_trimesh_graph_edges: triangle vertex out of range");
    for (int64_t k = 0; k < 4 * nb; ++k)
        if (bend[k] >= num_nodes)
            return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_trimesh_graph_edges: hinge vertex out of range");
    *num_edges_out = canonical_pairs(
        num_nodes,
        [&](auto&& visit) {
            for (int64_t t = 0; t < nt; ++t) {
                const int32_t* r = tris + 3 * t;
                visit(r[0], r[1]);
                visit(r[0], r[2]);
                visit(r[1], r[2]);
            }
            for (int64_t e = 0; e < nb; ++e) {
                const int32_t* r = bend + 4 * e;
                static const int kPairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
                for (const auto& p : kPairs)
                    if (r[p[0]] >= 0 && r[p[1]] >= 0) visit(r[p[0]], r[p[1]]);
            }
        },
        edges_out);
    return VBD_OK;
}
