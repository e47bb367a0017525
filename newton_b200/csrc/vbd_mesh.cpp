// vbd_mesh.cpp -- soft-mesh connectivity on the host (model setup, no GPU).
//
// Restates the connectivity Newton's VBD cloth path builds before simulation
// (newton/_src/utils/mesh.py):
//   vbd_mesh_edge_adjacency   MeshAdjacency._compute_edge_adjacency (utils/mesh.py:465-531)
//   vbd_mesh_vertex_csr       init_vertex_adjacency + the count / fill kernels
//                             (utils/mesh.py:595-655, :675-772)
// The reference runs these as serial loops over the elements; here they are one pass over the
// element slots each (an open-addressing hash of the undirected edges, a counting sort of the
// per-vertex records), with the same ordering rules, so the tables are identical.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "vbd_internal.h"

namespace {

inline uint64_t mix64(uint64_t x) {
    // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

}  // namespace

// Edge table [o0, o1, v0, v1] of a triangle mesh.  Every triangle t contributes its local edge
// slots k = 0, 1, 2 in order: (tris[t][k], tris[t][k+1]) with opposite vertex tris[t][k+2]; an
// undirected edge is numbered when first met in that traversal.  The first triangle on an edge
// writes o0, v0, v1 and edge_tri[.,0]; the second writes o1 and edge_tri[.,1]; a third or later
// one counts as non-manifold and changes nothing.  Outputs are sized for 3 nt edges; *num_edges
// receives the count.
extern "C" int vbd_mesh_edge_adjacency(const int32_t* tris, int32_t nt, int32_t* edge_indices, int32_t* edge_tri,
                                       int32_t* tri_edge, int32_t* num_edges, int32_t* nonmanifold) {
    if (nt < 0 || (nt > 0 && (!tris || !edge_indices || !edge_tri || !tri_edge)) || !num_edges)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mesh_edge_adjacency: invalid arguments");
    *num_edges = 0;
    if (nonmanifold) *nonmanifold = 0;
    if (nt == 0) return VBD_OK;
    const size_t slots = 3 * static_cast<size_t>(nt);
    size_t cap = 1;
    while (cap < 2 * slots) cap <<= 1;
    std::vector<uint64_t> keys(cap, ~uint64_t(0));
    std::vector<int32_t> vals(cap, -1);
    std::vector<uint8_t> sides;
    sides.reserve(slots);
    int32_t ne = 0, extra = 0;
    for (int32_t t = 0; t < nt; ++t) {
        const int32_t* tri = tris + 3 * static_cast<size_t>(t);
        for (int k = 0; k < 3; ++k) {
            const int32_t a = tri[k], b = tri[(k + 1) % 3], o = tri[(k + 2) % 3];
            const uint32_t lo = static_cast<uint32_t>(a < b ? a : b), hi = static_cast<uint32_t>(a < b ? b : a);
            const uint64_t key = (static_cast<uint64_t>(lo) << 32) | hi;
            size_t h = static_cast<size_t>(mix64(key)) & (cap - 1);
            while (keys[h] != key && keys[h] != ~uint64_t(0)) h = (h + 1) & (cap - 1);
            int32_t e;
            if (keys[h] == ~uint64_t(0)) {
                keys[h] = key;
                e = ne++;
                vals[h] = e;
                sides.push_back(1);
                int32_t* row = edge_indices + 4 * static_cast<size_t>(e);
                row[0] = o;
                row[1] = -1;
                row[2] = a;
                row[3] = b;
                edge_tri[2 * static_cast<size_t>(e)] = t;
                edge_tri[2 * static_cast<size_t>(e) + 1] = -1;
            } else {
                e = vals[h];
                if (sides[e] == 1) {
                    edge_indices[4 * static_cast<size_t>(e) + 1] = o;
                    edge_tri[2 * static_cast<size_t>(e) + 1] = t;
                } else {
                    ++extra;
                }
                if (sides[e] < 255) ++sides[e];
            }
            tri_edge[3 * static_cast<size_t>(t) + k] = e;
        }
    }
    *num_edges = ne;
    if (nonmanifold) *nonmanifold = extra;
    return VBD_OK;
}

// Per-vertex CSR of (element id, local slot) pairs, records in element order.  `entries` holds
// `per_element` vertex ids per element (a vertex id of -1 is skipped) and `slot_of` the local slot
// each position stands for.  values receives 2 ints per record; offsets[v] counts ints, as the
// reference's v_adj_*_offsets do (length particle_count + 1).
extern "C" int vbd_mesh_vertex_csr(const int32_t* entries, int32_t n_elements, int32_t per_element,
                                   const int32_t* slot_of, int32_t particle_count, int32_t* values,
                                   int32_t* offsets) {
    if (n_elements < 0 || per_element < 1 || per_element > 16 || particle_count < 0 || !offsets ||
        (n_elements > 0 && (!entries || !slot_of || !values)))
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mesh_vertex_csr: invalid arguments");
    std::vector<int64_t> count(static_cast<size_t>(particle_count) + 1, 0);
    const size_t n = static_cast<size_t>(n_elements) * per_element;
    for (size_t j = 0; j < n; ++j) {
        const int32_t v = entries[j];
        if (v == -1) continue;
        if (v < 0 || v >= particle_count)
            return vbd::fail(VBD_ERR_INVALID_ARGUMENT,
                             "vbd_mesh_vertex_csr: vertex id " + std::to_string(v) + " out of range");
        ++count[static_cast<size_t>(v) + 1];
    }
    for (int32_t v = 0; v < particle_count; ++v) count[v + 1] += count[v];
    if (2 * count[particle_count] > INT32_MAX)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mesh_vertex_csr: too many records for int32 offsets");
    for (int32_t v = 0; v <= particle_count; ++v) offsets[v] = static_cast<int32_t>(2 * count[v]);
    std::vector<int64_t> cur(count.begin(), count.end() - 1);
    for (int32_t e = 0; e < n_elements; ++e) {
        for (int32_t k = 0; k < per_element; ++k) {
            const int32_t v = entries[static_cast<size_t>(e) * per_element + k];
            if (v == -1) continue;
            const int64_t r = cur[v]++;
            values[2 * r] = e;
            values[2 * r + 1] = slot_of[k];
        }
    }
    return VBD_OK;
}
