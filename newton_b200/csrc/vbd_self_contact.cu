// vbd_self_contact.cu -- cloth self-contact for the VBD step on sm_100a.
//
// Restates the reference's particle self-contact path (SolverVBD with
// particle_enable_self_contact=True):
//   detection         TriMeshCollisionDetector.vertex_triangle_collision_detection /
//                     edge_edge_collision_detection (solvers/vbd/tri_mesh_collision.py:645-730;
//                     kernels geometry/kernels.py:1328-1497, :1499-1640), n-ring topological filter
//                     (tri_mesh_collision.py:123-233), rest-shape exclusion radius
//   forces            accumulate_self_contact_force_and_hessian (particle_vbd_kernels.py:1498-1639)
//   truncation        apply_planar_truncation_parallel_by_collision (:2133-2263) + apply_truncation_ts
//                     (:2266-2286) with max displacement margin * relaxation * 0.5
//                     (solver_vbd.py:2026-2063)
//   orchestration     solver_vbd.py:2065-2100 (detection before the forward step), :2540-2545
//                     (detection interval), :3221-3237 (positions become the displacement base)
//
// B200 design.  The reference refits two BVHs and runs 4 threads per primitive with atomics into
// the per-vertex force.  Here:
//   * a hashed uniform grid (cell = margin + longest rest edge) is rebuilt every detection in
//     four device passes -- count per bucket, exclusive scan (CUB), fill, query -- so no host
//     synchronisation is needed and a step stays graph-capturable.  A triangle / edge of at most
//     half a cell sits in the one bucket of its box centre's cell, a larger (stretched) one in
//     every cell its box overlaps; the count pass keeps each element's box;
//   * a query rejects candidates by box overlap before any filter or exact distance, skips
//     entries of other cells that share its bucket, and keeps the survivors in a sorted
//     per-vertex / per-edge list (so each pair is reported once);
//   * forces are gathered per vertex of the current color, one warp per vertex taking the pairs
//     round-robin in a fixed order (own vertex-triangle pairs, then the pairs of each incident
//     triangle, then the edge-edge pairs of each incident edge) and reduced with xor shuffles, so
//     results are deterministic;
//   * truncation ratios are reduced with an integer atomicMin on the (non-negative) float bits,
//     which is exact and order-independent.
// Buffers are fixed-size (reference defaults: 32 triangles per vertex, 64 edges per edge; plus
// 32 vertices per triangle for the gather); candidates beyond a buffer are dropped and counted.
#include "vbd_self_contact.h"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "vbd_self_contact_math.cuh"

namespace vbd {

namespace {

struct CellRange {
    int3 lo, hi;
};

__device__ __forceinline__ int cell_coord(float x, float inv) { return static_cast<int>(floorf(x * inv)); }

__device__ __forceinline__ CellRange cell_range(float3 lo, float3 hi, float inv) {
    CellRange r;
    r.lo = make_int3(cell_coord(lo.x, inv), cell_coord(lo.y, inv), cell_coord(lo.z, inv));
    r.hi = make_int3(cell_coord(hi.x, inv), cell_coord(hi.y, inv), cell_coord(hi.z, inv));
    return r;
}

__device__ __forceinline__ long long cell_count(const CellRange& r) {
    return (static_cast<long long>(r.hi.x) - r.lo.x + 1) * (static_cast<long long>(r.hi.y) - r.lo.y + 1) *
           (static_cast<long long>(r.hi.z) - r.lo.z + 1);
}

__device__ __forceinline__ unsigned cell_hash(int x, int y, int z, unsigned mask) {
    return ((static_cast<unsigned>(x) * 73856093u) ^ (static_cast<unsigned>(y) * 19349663u) ^
            (static_cast<unsigned>(z) * 83492791u)) &
           mask;
}

__device__ __forceinline__ float3 fmin3(float3 a, float3 b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ float3 fmax3(float3 a, float3 b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

struct GridArgs {
    const float4* x;      // positions (internal order)
    const int4* elem;     // triangles or edges
    int n;
    bool tri;
    bool all_cells;       // every element goes into every cell its box overlaps (edge grid)
    float inv_cell;
    unsigned mask;
    int* cnt;
    const int* off;
    int* cur;
    int* items;
    float4* item_box;     // [2 cap] the box of every bucket entry, next to its id (fill pass)
    int cap;
    float4* box;          // [2n] element boxes (lo, hi; lo.w = 1 for a large element), count pass
    unsigned* counters;
};

__device__ __forceinline__ void elem_box(const GridArgs& a, int e, float3& lo, float3& hi) {
    const int4 el = a.elem[e];
    const float3 p0 = xyz(a.x[el.x]), p1 = xyz(a.x[el.y]);
    lo = fmin3(p0, p1);
    hi = fmax3(p0, p1);
    if (a.tri) {
        const float3 p2 = xyz(a.x[el.z]);
        lo = fmin3(lo, p2);
        hi = fmax3(hi, p2);
    }
}

__device__ __forceinline__ int3 center_cell(float4 lo, float4 hi, float inv) {
    return make_int3(cell_coord(0.5f * (lo.x + hi.x), inv), cell_coord(0.5f * (lo.y + hi.y), inv),
                     cell_coord(0.5f * (lo.z + hi.z), inv));
}

// Triangle grid (queried by points): a triangle whose half-extent is at most half a cell goes into
// the one bucket of its box centre's cell; a larger one (stretched) goes into every cell its box
// overlaps, up to kMaxLargeCells, and is flagged (lo.w = 1).  A vertex query then looks margin +
// half a cell around its point, however far the cloth stretches elsewhere.
// Edge grid (queried by edge boxes): every edge goes into every cell its box overlaps (flagged),
// so an edge query only covers its box grown by the margin -- for edges shorter than a cell that
// is fewer bucket entries than centre binning's extra half cell on every side -- and a pair is
// taken only in the first cell the two ranges share.
constexpr int kMaxLargeCells = 4096;

__global__ void grid_count_kernel(GridArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n) return;
    float3 lo, hi;
    elem_box(a, e, lo, hi);
    const float half = 0.5f * fmaxf(fmaxf(hi.x - lo.x, hi.y - lo.y), hi.z - lo.z);
    const bool large = a.all_cells || !(half <= 0.5f / a.inv_cell);
    const float4 l4 = make_float4(lo.x, lo.y, lo.z, large ? 1.f : 0.f), h4 = make_float4(hi.x, hi.y, hi.z, 0.f);
    a.box[2 * e] = l4;
    a.box[2 * e + 1] = h4;
    if (!large) {
        const int3 c = center_cell(l4, h4, a.inv_cell);
        atomicAdd(&a.cnt[cell_hash(c.x, c.y, c.z, a.mask)], 1);
        return;
    }
    const CellRange r = cell_range(lo, hi, a.inv_cell);
    if (!(cell_count(r) <= kMaxLargeCells)) {
        atomicAdd(&a.counters[kScGridOverflow], 1u);
        return;
    }
    for (int z = r.lo.z; z <= r.hi.z; ++z)
        for (int y = r.lo.y; y <= r.hi.y; ++y)
            for (int x = r.lo.x; x <= r.hi.x; ++x) atomicAdd(&a.cnt[cell_hash(x, y, z, a.mask)], 1);
}

__global__ void grid_fill_kernel(GridArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n) return;
    const float4 l4 = a.box[2 * e], h4 = a.box[2 * e + 1];
    if (l4.w == 0.f) {
        const int3 c = center_cell(l4, h4, a.inv_cell);
        const unsigned h = cell_hash(c.x, c.y, c.z, a.mask);
        const int k = a.off[h] + atomicAdd(&a.cur[h], 1);
        if (k < a.cap) {
            a.items[k] = e;
            a.item_box[2 * k] = l4;
            a.item_box[2 * k + 1] = h4;
        } else {
            atomicAdd(&a.counters[kScGridOverflow], 1u);
        }
        return;
    }
    const CellRange r = cell_range(xyz(l4), xyz(h4), a.inv_cell);
    if (!(cell_count(r) <= kMaxLargeCells)) return;
    for (int z = r.lo.z; z <= r.hi.z; ++z)
        for (int y = r.lo.y; y <= r.hi.y; ++y)
            for (int x = r.lo.x; x <= r.hi.x; ++x) {
                const unsigned h = cell_hash(x, y, z, a.mask);
                const int k = a.off[h] + atomicAdd(&a.cur[h], 1);
                if (k < a.cap) {
                    a.items[k] = e;
                    a.item_box[2 * k] = l4;
                    a.item_box[2 * k + 1] = h4;
                } else {
                    atomicAdd(&a.counters[kScGridOverflow], 1u);
                }
            }
}

// whether bucket entry (box blo/bhi) belongs to cell (x, y, z): its centre cell, or for a large
// element any cell its box overlaps
__device__ __forceinline__ bool in_cell(float4 blo, float4 bhi, float inv, int x, int y, int z) {
    if (blo.w == 0.f) {
        const int3 c = center_cell(blo, bhi, inv);
        return c.x == x && c.y == y && c.z == z;
    }
    const CellRange r = cell_range(xyz(blo), xyz(bhi), inv);
    return x >= r.lo.x && x <= r.hi.x && y >= r.lo.y && y <= r.hi.y && z >= r.lo.z && z <= r.hi.z;
}

__device__ __forceinline__ bool boxes_overlap(float3 lo, float3 hi, float4 blo, float4 bhi) {
    return !(blo.x > hi.x || bhi.x < lo.x || blo.y > hi.y || bhi.y < lo.y || blo.z > hi.z || bhi.z < lo.z);
}

// sorted insert without duplicates into row[0..n) of capacity cap; false when full
__device__ __forceinline__ bool sorted_insert(int* row, int& n, int cap, int x) {
    int k = 0;
    while (k < n && row[k] < x) ++k;
    if (k < n && row[k] == x) return true;
    if (n >= cap) return false;
    for (int j = n; j > k; --j) row[j] = row[j - 1];
    row[k] = x;
    ++n;
    return true;
}

__device__ __forceinline__ bool filtered(const int* off, const int* list, int row, int x) {
    if (!off) return false;
    const int* b = list + off[row];
    const int* e = list + off[row + 1];
    while (b < e) {
        const int* mid = b + (e - b) / 2;
        if (*mid < x) b = mid + 1;
        else e = mid;
    }
    return b < list + off[row + 1] && *b == x;
}

__device__ __forceinline__ bool list_contains(const int* b, const int* e, int x) {
    for (const int* p = b; p < e; ++p)
        if (*p == x) return true;
    return false;
}

struct QueryArgs {
    const float4* x;
    const int* vworld;
    const int *vfilt_off, *vfilt, *efilt_off, *efilt;  // external filter lists (NULL: none)
    const float4* rest;
    const int4* tri;
    const int4* edge;
    const int* near_off;
    const int* near;
    const int* vt_order;  // query slot -> vertex
    int V, T, E;
    float margin, inv_cell, par_eps, rest_excl;
    unsigned tri_mask, edge_mask;
    const int *tri_cnt, *tri_off, *tri_items;
    const int *edge_cnt, *edge_off, *edge_items;
    const float4 *tri_item_box, *edge_item_box;
    int tri_cap, edge_cap;
    int vbuf, ebuf;
    int* vt_count;
    int* vt_list;
    int* ee_count;
    int* ee_list;
    unsigned* counters;
};

constexpr int kMaxQueryCells = 512;
constexpr int kWarpUnionCells = 128;  // larger warp unions fall back to one walk per lane
constexpr int kQueryBlock = 128;
constexpr int kQueryWarps = kQueryBlock / 32;
constexpr int kEeLanes = 4;  // lanes per edge-edge query (4 measured best of 2, 4, 8)

// ---- vertex-triangle candidates ------------------------------------------------------------
struct VtQuery {
    int i;
    float3 p, plo, phi;
    CellRange q;
    int wv;
    const int *nb, *ne;
    int* row;
    int n;
    bool full;
};

// the tests after the box pre-filter; appends t to the vertex's sorted list
__device__ __forceinline__ void vt_accept(const QueryArgs& a, VtQuery& v, int t) {
    const int4 tr = a.tri[t];
    const int i = v.i;
    if (tr.x == i || tr.y == i || tr.z == i) return;
    if (v.wv >= 0 && tr.w >= 0 && v.wv != tr.w) return;
    if (list_contains(v.nb, v.ne, tr.x) || list_contains(v.nb, v.ne, tr.y) || list_contains(v.nb, v.ne, tr.z)) return;
    if (filtered(a.vfilt_off, a.vfilt, i, t)) return;
    float3 bary;
    const float dist = length(triangle_closest_point(xyz(a.x[tr.x]), xyz(a.x[tr.y]), xyz(a.x[tr.z]), v.p, bary) - v.p);
    if (!(dist < a.margin)) return;
    if (a.rest_excl > 0.f) {
        const float3 rp = xyz(a.rest[i]);
        const float dr = length(
            triangle_closest_point(xyz(a.rest[tr.x]), xyz(a.rest[tr.y]), xyz(a.rest[tr.z]), rp, bary) - rp);
        if (dr < a.rest_excl) return;
    }
    if (!sorted_insert(v.row, v.n, a.vbuf, t)) v.full = true;
}

__device__ __forceinline__ void vt_scan_lane(const QueryArgs& a, VtQuery& v) {
    for (int z = v.q.lo.z; z <= v.q.hi.z; ++z)
        for (int y = v.q.lo.y; y <= v.q.hi.y; ++y)
            for (int x = v.q.lo.x; x <= v.q.hi.x; ++x) {
                const unsigned h = cell_hash(x, y, z, a.tri_mask);
                const int b = a.tri_off[h];
                const int e = min(b + a.tri_cnt[h], a.tri_cap);
                for (int k = b; k < e; ++k) {
                    const float4 blo = a.tri_item_box[2 * k], bhi = a.tri_item_box[2 * k + 1];
                    if (!boxes_overlap(v.plo, v.phi, blo, bhi)) continue;
                    if (!in_cell(blo, bhi, a.inv_cell, x, y, z)) continue;  // another cell in this bucket
                    vt_accept(a, v, a.tri_items[k]);
                }
            }
}

__device__ __forceinline__ bool warp_union(bool ok, const CellRange& q, CellRange& u) {
    const unsigned all = 0xffffffffu;
    if (__ballot_sync(all, ok) == 0u) return false;
    u.lo = make_int3(__reduce_min_sync(all, ok ? q.lo.x : INT_MAX), __reduce_min_sync(all, ok ? q.lo.y : INT_MAX),
                     __reduce_min_sync(all, ok ? q.lo.z : INT_MAX));
    u.hi = make_int3(__reduce_max_sync(all, ok ? q.hi.x : INT_MIN), __reduce_max_sync(all, ok ? q.hi.y : INT_MIN),
                     __reduce_max_sync(all, ok ? q.hi.z : INT_MIN));
    return true;
}

__device__ __forceinline__ bool in_range(const CellRange& q, int x, int y, int z) {
    return x >= q.lo.x && x <= q.hi.x && y >= q.lo.y && y <= q.hi.y && z >= q.lo.z && z <= q.hi.z;
}

// A warp of 32 consecutive vertices walks the union of their query ranges once: every bucket
// entry is staged in shared memory by one lane and tested by all lanes against their own query,
// so the cheap rejections run with every lane active (a walk per lane diverges: its buckets
// differ in length from its neighbours').
__global__ void __launch_bounds__(kQueryBlock) vt_query_kernel(QueryArgs a) {
    __shared__ int s_id[kQueryWarps][32];
    __shared__ float4 s_box[kQueryWarps][64];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // consecutive query slots are spatially close vertices (Morton order of the rest shape; the
    // internal vertex order is color-major, so neighbours in it are far apart), which keeps the
    // warp's union of cell ranges small
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = slot < a.V ? a.vt_order[slot] : a.V;
    const bool active = i < a.V;
    VtQuery v;
    v.i = i;
    v.n = 0;
    v.full = false;
    bool ok = false;
    if (active) {
        v.p = xyz(a.x[i]);
        const float m = a.margin;
        v.plo = v.p - f3(m, m, m);
        v.phi = v.p + f3(m, m, m);
        // a small triangle within the margin has its box centre within margin + half a cell of p;
        // a large one is in every cell its box overlaps
        const float r = m + 0.5f / a.inv_cell;
        v.q = cell_range(v.p - f3(r, r, r), v.p + f3(r, r, r), a.inv_cell);
        ok = cell_count(v.q) <= kMaxQueryCells;
        if (!ok) {
            atomicAdd(&a.counters[kScGridOverflow], 1u);
            a.vt_count[i] = 0;
        } else {
            v.wv = a.vworld[i];
            v.nb = a.near + a.near_off[i];
            v.ne = a.near + a.near_off[i + 1];
            v.row = a.vt_list + static_cast<size_t>(i) * a.vbuf;
        }
    }
    CellRange u;
    if (!warp_union(ok, v.q, u)) return;
    if (cell_count(u) > kWarpUnionCells) {
        if (ok) vt_scan_lane(a, v);
    } else {
        for (int z = u.lo.z; z <= u.hi.z; ++z)
            for (int y = u.lo.y; y <= u.hi.y; ++y)
                for (int x = u.lo.x; x <= u.hi.x; ++x) {
                    const bool mine = ok && in_range(v.q, x, y, z);
                    if (!__any_sync(0xffffffffu, mine)) continue;
                    const unsigned h = cell_hash(x, y, z, a.tri_mask);
                    const int b = a.tri_off[h];
                    const int cnt = min(b + a.tri_cnt[h], a.tri_cap) - b;
                    for (int c = 0; c < cnt; c += 32) {
                        if (c + lane < cnt) {
                            const int k = b + c + lane;
                            s_id[w][lane] = a.tri_items[k];
                            s_box[w][2 * lane] = a.tri_item_box[2 * k];
                            s_box[w][2 * lane + 1] = a.tri_item_box[2 * k + 1];
                        }
                        __syncwarp();
                        const int mc = min(32, cnt - c);
                        if (mine) {
                            for (int t = 0; t < mc; ++t) {
                                const float4 blo = s_box[w][2 * t], bhi = s_box[w][2 * t + 1];
                                if (!boxes_overlap(v.plo, v.phi, blo, bhi)) continue;
                                if (!in_cell(blo, bhi, a.inv_cell, x, y, z)) continue;
                                vt_accept(a, v, s_id[w][t]);
                            }
                        }
                        __syncwarp();
                    }
                }
    }
    if (ok) {
        a.vt_count[i] = v.n;
        if (v.full) atomicAdd(&a.counters[kScVtOverflow], 1u);
    }
}

// ---- edge-edge candidates ------------------------------------------------------------------
// Edge-edge pairs are symmetric: edge e only searches partners g > e and records the pair in both
// lists through atomic slots; ee_sort_kernel then orders every list.  A partner sits in every
// cell its box overlaps and is taken only in the first cell of the query range it occupies, so
// every pair is met exactly once.
struct EeQuery {
    int e;
    int4 ed;
    float3 a0, a1, qlo, qhi;
    CellRange q;
    const int *n0b, *n0e, *n1b, *n1e;
};

__device__ __forceinline__ bool ee_owns(const EeQuery& v, float4 blo, float4 bhi, float inv, int x, int y, int z) {
    if (blo.w == 0.f) {
        const int3 c = center_cell(blo, bhi, inv);
        return c.x == x && c.y == y && c.z == z;
    }
    const CellRange gr = cell_range(xyz(blo), xyz(bhi), inv);
    if (max(v.q.lo.x, gr.lo.x) != x || max(v.q.lo.y, gr.lo.y) != y || max(v.q.lo.z, gr.lo.z) != z) return false;
    return x <= gr.hi.x && y <= gr.hi.y && z <= gr.hi.z;
}

__device__ __forceinline__ void ee_accept(const QueryArgs& a, const EeQuery& v, int g) {
    const int4 gd = a.edge[g];
    const int4 ed = v.ed;
    if (gd.x == ed.x || gd.x == ed.y || gd.y == ed.x || gd.y == ed.y) return;
    if (ed.z >= 0 && gd.z >= 0 && ed.z != gd.z) return;
    if (list_contains(v.n0b, v.n0e, gd.x) || list_contains(v.n0b, v.n0e, gd.y) || list_contains(v.n1b, v.n1e, gd.x) ||
        list_contains(v.n1b, v.n1e, gd.y))
        return;
    float s, t, dist;
    closest_edge_edge(v.a0, v.a1, xyz(a.x[gd.x]), xyz(a.x[gd.y]), a.par_eps, s, t, dist);
    if (!(dist < a.margin)) return;
    if (a.rest_excl > 0.f) {
        float sr, tr, dr;
        closest_edge_edge(xyz(a.rest[ed.x]), xyz(a.rest[ed.y]), xyz(a.rest[gd.x]), xyz(a.rest[gd.y]), a.par_eps, sr,
                          tr, dr);
        if (dr < a.rest_excl) return;
    }
    // the distance of (e, g) and of (g, e) is the same test; record both sides (each side's
    // external filter applies to its own list)
    const int e = v.e;
    if (!filtered(a.efilt_off, a.efilt, e, g)) {
        const int ke = atomicAdd(&a.ee_count[e], 1);
        if (ke < a.ebuf) a.ee_list[static_cast<size_t>(e) * a.ebuf + ke] = g;
        else atomicAdd(&a.counters[kScEeOverflow], 1u);
    }
    if (!filtered(a.efilt_off, a.efilt, g, e)) {
        const int kg = atomicAdd(&a.ee_count[g], 1);
        if (kg < a.ebuf) a.ee_list[static_cast<size_t>(g) * a.ebuf + kg] = e;
        else atomicAdd(&a.counters[kScEeOverflow], 1u);
    }
}

__device__ __forceinline__ void ee_scan_lane(const QueryArgs& a, const EeQuery& v) {
    for (int z = v.q.lo.z; z <= v.q.hi.z; ++z)
        for (int y = v.q.lo.y; y <= v.q.hi.y; ++y)
            for (int x = v.q.lo.x; x <= v.q.hi.x; ++x) {
                const unsigned h = cell_hash(x, y, z, a.edge_mask);
                const int b = a.edge_off[h];
                const int en = min(b + a.edge_cnt[h], a.edge_cap);
                for (int k = b; k < en; ++k) {
                    const int g = a.edge_items[k];
                    if (g <= v.e) continue;
                    const float4 blo = a.edge_item_box[2 * k], bhi = a.edge_item_box[2 * k + 1];
                    if (!boxes_overlap(v.qlo, v.qhi, blo, bhi)) continue;
                    if (!ee_owns(v, blo, bhi, a.inv_cell, x, y, z)) continue;
                    ee_accept(a, v, g);
                }
            }
}

// kEeLanes lanes serve one edge query, so a warp holds 32 / kEeLanes consecutive (spatially
// adjacent) edges: their union of cell ranges stays close to one query's range, and each lane
// tests every kEeLanes-th staged entry.  Each (edge, partner) test runs on exactly one lane.
__global__ void __launch_bounds__(kQueryBlock) ee_query_kernel(QueryArgs a) {
    __shared__ int s_id[kQueryWarps][32];
    __shared__ float4 s_box[kQueryWarps][64];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) / kEeLanes;
    const int sub = lane % kEeLanes;
    EeQuery v;
    v.e = e;
    bool ok = false;
    if (e < a.E) {
        v.ed = a.edge[e];
        v.a0 = xyz(a.x[v.ed.x]);
        v.a1 = xyz(a.x[v.ed.y]);
        const float m = a.margin;
        v.qlo = fmin3(v.a0, v.a1) - f3(m, m, m);
        v.qhi = fmax3(v.a0, v.a1) + f3(m, m, m);
        // every partner sits in all the cells its box overlaps: the query's own cells suffice
        v.q = cell_range(v.qlo, v.qhi, a.inv_cell);
        ok = cell_count(v.q) <= kMaxQueryCells;
        if (!ok) {
            if (sub == 0) atomicAdd(&a.counters[kScGridOverflow], 1u);
        } else {
            v.n0b = a.near + a.near_off[v.ed.x];
            v.n0e = a.near + a.near_off[v.ed.x + 1];
            v.n1b = a.near + a.near_off[v.ed.y];
            v.n1e = a.near + a.near_off[v.ed.y + 1];
        }
    }
    CellRange u;
    if (!warp_union(ok, v.q, u)) return;
    if (cell_count(u) > kWarpUnionCells) {
        if (ok && sub == 0) ee_scan_lane(a, v);
        return;
    }
    // partners with id <= the warp's smallest query id are rejected by every lane (g > e): they
    // are dropped while staging, so the lanes only walk the entries that can pass
    const int e_min = __reduce_min_sync(0xffffffffu, ok ? e : INT_MAX);
    for (int z = u.lo.z; z <= u.hi.z; ++z)
        for (int y = u.lo.y; y <= u.hi.y; ++y)
            for (int x = u.lo.x; x <= u.hi.x; ++x) {
                const bool mine = ok && in_range(v.q, x, y, z);
                if (!__any_sync(0xffffffffu, mine)) continue;
                const unsigned h = cell_hash(x, y, z, a.edge_mask);
                const int b = a.edge_off[h];
                const int cnt = min(b + a.edge_cnt[h], a.edge_cap) - b;
                for (int c = 0; c < cnt; c += 32) {
                    int gid = -1;
                    if (c + lane < cnt) gid = a.edge_items[b + c + lane];
                    const bool keep = gid > e_min;
                    const unsigned kept = __ballot_sync(0xffffffffu, keep);
                    if (keep) {
                        const int k = b + c + lane;
                        const int slot = __popc(kept & ((1u << lane) - 1u));
                        s_id[w][slot] = gid;
                        s_box[w][2 * slot] = a.edge_item_box[2 * k];
                        s_box[w][2 * slot + 1] = a.edge_item_box[2 * k + 1];
                    }
                    __syncwarp();
                    const int mc = __popc(kept);
                    if (mine) {
                        for (int t = sub; t < mc; t += kEeLanes) {
                            const int g = s_id[w][t];
                            if (g <= e) continue;
                            const float4 blo = s_box[w][2 * t], bhi = s_box[w][2 * t + 1];
                            if (!boxes_overlap(v.qlo, v.qhi, blo, bhi)) continue;
                            if (!ee_owns(v, blo, bhi, a.inv_cell, x, y, z)) continue;
                            ee_accept(a, v, g);
                        }
                    }
                    __syncwarp();
                }
            }
}

__global__ void ee_sort_kernel(int E, int* ee_count, int* ee_list, int ebuf) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int n = min(ee_count[e], ebuf);
    ee_count[e] = n;
    int* row = ee_list + static_cast<size_t>(e) * ebuf;
    for (int a = 1; a < n; ++a) {
        const int x = row[a];
        int b = a - 1;
        while (b >= 0 && row[b] > x) {
            row[b + 1] = row[b];
            --b;
        }
        row[b + 1] = x;
    }
}

__global__ void tri_reverse_kernel(int V, const int* vt_count, const int* vt_list, int vbuf, int* tv_count,
                                   int* tv_list, int tcap, unsigned* counters) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int* row = vt_list + static_cast<size_t>(i) * vbuf;
    for (int k = 0; k < vt_count[i]; ++k) {
        const int t = row[k];
        const int j = atomicAdd(&tv_count[t], 1);
        if (j < tcap) tv_list[static_cast<size_t>(t) * tcap + j] = i;
        else atomicAdd(&counters[kScTvOverflow], 1u);
    }
}

__global__ void tri_sort_kernel(int T, int* tv_count, int* tv_list, int tcap) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int n = min(tv_count[t], tcap);
    tv_count[t] = n;
    int* row = tv_list + static_cast<size_t>(t) * tcap;
    for (int a = 1; a < n; ++a) {
        const int x = row[a];
        int b = a - 1;
        while (b >= 0 && row[b] > x) {
            row[b + 1] = row[b];
            --b;
        }
        row[b + 1] = x;
    }
}

// marks every vertex that takes part in a detected pair (the gather skips the others)
__global__ void mark_contact_vertices_kernel(int V, int E, const int4* tri, const int4* edge, const int* vt_count,
                                             const int* vt_list, int vbuf, const int* ee_count, unsigned char* flag) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < V && vt_count[idx] > 0) {
        flag[idx] = 1;
        const int* row = vt_list + static_cast<size_t>(idx) * vbuf;
        for (int k = 0; k < vt_count[idx]; ++k) {
            const int4 tr = tri[row[k]];
            flag[tr.x] = 1;
            flag[tr.y] = 1;
            flag[tr.z] = 1;
        }
    }
    if (idx < E && ee_count[idx] > 0) {
        const int4 ed = edge[idx];
        flag[ed.x] = 1;
        flag[ed.y] = 1;
    }
}

// compact lists of the work the per-color passes do: contact-touching vertices by color, and
// the non-empty vertex-triangle / edge-edge rows (the truncation planes)
__global__ void compact_kernel(int V, int E, const unsigned char* flag, const int* vcolor, const int* color_start,
                               const int* vt_count, const int* ee_count, int* act_v, int* act_vcnt, int* act_rows,
                               int* act_cnt) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < V && flag[idx]) {
        const int c = vcolor[idx];
        if (c >= 0) act_v[color_start[c] + atomicAdd(&act_vcnt[c], 1)] = idx;
    }
    if (idx < V && vt_count[idx] > 0) act_rows[atomicAdd(&act_cnt[0], 1)] = idx;
    if (idx < E && ee_count[idx] > 0) act_rows[V + atomicAdd(&act_cnt[1], 1)] = idx;
}

__global__ void copy_positions_kernel(int V, const float4* src, float4* cd, float4* disp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    if (src != cd) cd[i] = src[i];
    if (disp) disp[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void load_positions_kernel(int V, const int* perm, const float* q, float4* cd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int o = perm[i];
    cd[i] = make_float4(q[3 * o], q[3 * o + 1], q[3 * o + 2], 0.f);
}

struct AccumArgs {
    const float4* x;
    const float4* x0;   // anchor: the step's start positions
    const int4* tri;
    const int4* edge;
    const int *inc_t_off, *inc_e_off;
    const int2 *inc_t, *inc_e;
    const int *vt_count, *vt_list, *ee_count, *ee_list, *tv_count, *tv_list;
    int vbuf, ebuf, tcap;
    const int* list;    // the color's contact-touching vertices
    const int* count;   // how many (device)
    float r, ke, kd, mu, eps_u, dt, par_eps;
    float4 *f, *h0, *h1;
};

// L lanes per vertex: the vertex's pairs (own vertex-triangle list, then each incident triangle's
// colliding vertices, then each incident edge's colliding edges) are dealt round-robin to the
// lanes, and the partial sums are combined with xor shuffles -- a fixed order, so deterministic.
constexpr int kAccumLanes = 32;

__device__ __forceinline__ float lane_sum(float v) {
    for (int off = kAccumLanes >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// this lane's share of vertex i's pairs (i < 0: an idle slot that only joins the shuffles)
__device__ __forceinline__ void accumulate_lane(const AccumArgs& a, int i, int lane, float3& f, Sym3& H) {
    if (i < 0) return;
    const float3 p = xyz(a.x[i]), p0 = xyz(a.x0[i]);
    int idx = 0;  // running pair index of this vertex; the lane takes idx % L == lane
    const int* row = a.vt_list + static_cast<size_t>(i) * a.vbuf;
    const int nv = a.vt_count[i];
    for (int k = lane; k < nv; k += kAccumLanes) {
        const int4 tr = a.tri[row[k]];
        vt_contact_slot(xyz(a.x[tr.x]), xyz(a.x[tr.y]), xyz(a.x[tr.z]), p, xyz(a.x0[tr.x]), xyz(a.x0[tr.y]),
                        xyz(a.x0[tr.z]), p0, 3, a.r, a.ke, a.kd, a.mu, a.eps_u, a.dt, f, H);
    }
    idx += nv;
    for (int k = a.inc_t_off[i]; k < a.inc_t_off[i + 1]; ++k) {
        const int2 ts = a.inc_t[k];
        const int n = a.tv_count[ts.x];
        int j = (lane - idx) % kAccumLanes;
        if (j < 0) j += kAccumLanes;
        if (j < n) {
            const int4 tr = a.tri[ts.x];
            const float3 t0 = xyz(a.x[tr.x]), t1 = xyz(a.x[tr.y]), t2 = xyz(a.x[tr.z]);
            const float3 s0 = xyz(a.x0[tr.x]), s1 = xyz(a.x0[tr.y]), s2 = xyz(a.x0[tr.z]);
            const int* vl = a.tv_list + static_cast<size_t>(ts.x) * a.tcap;
            for (; j < n; j += kAccumLanes) {
                const int q = vl[j];
                vt_contact_slot(t0, t1, t2, xyz(a.x[q]), s0, s1, s2, xyz(a.x0[q]), ts.y, a.r, a.ke, a.kd, a.mu,
                                a.eps_u, a.dt, f, H);
            }
        }
        idx += n;
    }
    for (int k = a.inc_e_off[i]; k < a.inc_e_off[i + 1]; ++k) {
        const int2 es = a.inc_e[k];
        const int n = a.ee_count[es.x];
        int j = (lane - idx) % kAccumLanes;
        if (j < 0) j += kAccumLanes;
        if (j < n) {
            const int4 ed = a.edge[es.x];
            const float3 e0 = xyz(a.x[ed.x]), e1 = xyz(a.x[ed.y]);
            const float3 e0a = xyz(a.x0[ed.x]), e1a = xyz(a.x0[ed.y]);
            const int* gl = a.ee_list + static_cast<size_t>(es.x) * a.ebuf;
            for (; j < n; j += kAccumLanes) {
                const int4 gd = a.edge[gl[j]];
                ee_contact_slot(e0, e1, xyz(a.x[gd.x]), xyz(a.x[gd.y]), e0a, e1a, xyz(a.x0[gd.x]), xyz(a.x0[gd.y]),
                                es.y, a.r, a.ke, a.kd, a.mu, a.eps_u, a.dt, a.par_eps, f, H);
            }
        }
        idx += n;
    }
}

// Grid-stride over the color's contact-touching vertices (the others hold zero since the last
// detection).  A warp serves 32 / kAccumLanes vertices per round and the round bound is the same
// for the whole warp, so every lane joins every shuffle.
__global__ void accumulate_kernel(AccumArgs a) {
    const int n = *a.count;
    const int lane = threadIdx.x & (kAccumLanes - 1);
    const int sub = (threadIdx.x & 31) / kAccumLanes;  // vertex slot of this lane in its warp
    const int warps = gridDim.x * (blockDim.x >> 5);
    const int warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    constexpr int kVerts = 32 / kAccumLanes;  // vertices per warp and round
    for (int base = kVerts * warp; base < n; base += kVerts * warps) {
        const int slot = base + sub;
        const int i = slot < n ? a.list[slot] : -1;
        float3 f = f3(0.f, 0.f, 0.f);
        Sym3 H = zero_sym();
        accumulate_lane(a, i, lane, f, H);
        f.x = lane_sum(f.x);
        f.y = lane_sum(f.y);
        f.z = lane_sum(f.z);
        H.xx = lane_sum(H.xx);
        H.xy = lane_sum(H.xy);
        H.xz = lane_sum(H.xz);
        H.yy = lane_sum(H.yy);
        H.yz = lane_sum(H.yz);
        H.zz = lane_sum(H.zz);
        if (i >= 0 && lane == 0) {
            a.f[i] = make_float4(f.x, f.y, f.z, 0.f);
            a.h0[i] = make_float4(H.xx, H.xy, H.xz, H.yy);
            a.h1[i] = make_float4(H.yz, H.zz, 0.f, 0.f);
        }
    }
}

struct TruncArgs {
    const float4* cd;
    const float4* disp;
    const int4* tri;
    const int4* edge;
    const int *vt_count, *vt_list, *ee_count, *ee_list;
    const int* rows;     // non-empty vertex-triangle rows [0, V), then edge-edge rows [V, V + E)
    const int* counts;   // [2]
    int V, E, vbuf, ebuf;
    float eps, gamma;
    unsigned* ts;
};

__device__ __forceinline__ void ts_min(unsigned* ts, int i, float3 x, float3 dx, float3 n, float3 d, float eps,
                                       float gamma) {
    const float t = planar_truncation_t(x, dx, n, d, eps, gamma);
    atomicMin(&ts[i], __float_as_uint(t));
}

// grid-stride over the non-empty rows (vertex-triangle rows first, then edge-edge rows), kPlanarLanes
// lanes per row taking its pairs round-robin: the truncation factors are reduced with atomicMin,
// which does not depend on the order
constexpr int kPlanarLanes = 16;

__global__ void planar_kernel(TruncArgs a) {
    const int nv = a.counts[0], ne = a.counts[1];
    const int sub = threadIdx.x % kPlanarLanes;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) / kPlanarLanes; w < nv + ne;
         w += gridDim.x * blockDim.x / kPlanarLanes) {
        if (w < nv) {
            const int i = a.rows[w];
            const float3 v = xyz(a.cd[i]), dv = xyz(a.disp[i]);
            const int* row = a.vt_list + static_cast<size_t>(i) * a.vbuf;
            for (int k = sub; k < a.vt_count[i]; k += kPlanarLanes) {
                const int4 tr = a.tri[row[k]];
                const float3 t1 = xyz(a.cd[tr.x]), t2 = xyz(a.cd[tr.y]), t3 = xyz(a.cd[tr.z]);
                const float3 d1 = xyz(a.disp[tr.x]), d2 = xyz(a.disp[tr.y]), d3 = xyz(a.disp[tr.z]);
                float3 n, d;
                const int dummy = vt_plane(v, dv, t1, d1, t2, d2, t3, d3, n, d);
                if (!(dummy & 1)) ts_min(a.ts, i, v, dv, n, d, a.eps, a.gamma);
                if (!(dummy & 2)) ts_min(a.ts, tr.x, t1, d1, n, d, a.eps, a.gamma);
                if (!(dummy & 4)) ts_min(a.ts, tr.y, t2, d2, n, d, a.eps, a.gamma);
                if (!(dummy & 8)) ts_min(a.ts, tr.z, t3, d3, n, d, a.eps, a.gamma);
            }
        } else {
            const int e = a.rows[a.V + (w - nv)];
            const int4 ed = a.edge[e];
            const float3 a0 = xyz(a.cd[ed.x]), a1 = xyz(a.cd[ed.y]);
            const float3 da0 = xyz(a.disp[ed.x]), da1 = xyz(a.disp[ed.y]);
            const int* row = a.ee_list + static_cast<size_t>(e) * a.ebuf;
            for (int k = sub; k < a.ee_count[e]; k += kPlanarLanes) {
                const int4 gd = a.edge[row[k]];
                const float3 b0 = xyz(a.cd[gd.x]), b1 = xyz(a.cd[gd.y]);
                const float3 db0 = xyz(a.disp[gd.x]), db1 = xyz(a.disp[gd.y]);
                float3 n, d;
                const int dummy = ee_plane(a0, da0, a1, da1, b0, db0, b1, db1, n, d);
                if (!(dummy & 1)) ts_min(a.ts, ed.x, a0, da0, n, d, a.eps, a.gamma);
                if (!(dummy & 2)) ts_min(a.ts, ed.y, a1, da1, n, d, a.eps, a.gamma);
                if (!(dummy & 4)) ts_min(a.ts, gd.x, b0, db0, n, d, a.eps, a.gamma);
                if (!(dummy & 8)) ts_min(a.ts, gd.y, b1, db1, n, d, a.eps, a.gamma);
            }
        }
    }
}

// apply_truncation_ts: disp *= t, clamp |disp| to max_disp, pos = cd + disp; t is reset to 1
__global__ void apply_truncation_kernel(int V, const float4* cd, float4* disp, float4* pos, unsigned* ts,
                                        float max_disp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const float t = __uint_as_float(ts[i]);
    ts[i] = __float_as_uint(1.0f);
    const float4 d4 = disp[i];
    float3 d = f3(d4.x * t, d4.y * t, d4.z * t);
    const float l = length(d);
    if (l > max_disp) d = f3(d.x * max_disp / l, d.y * max_disp / l, d.z * max_disp / l);
    disp[i] = make_float4(d.x, d.y, d.z, 0.f);
    const float4 c = cd[i];
    pos[i] = make_float4(c.x + d.x, c.y + d.y, c.z + d.z, 0.f);
}

__global__ void fill_u32_kernel(unsigned* p, unsigned v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

unsigned next_pow2(long long x) {
    unsigned v = 1024;
    while (static_cast<long long>(v) < x && v < (1u << 30)) v <<= 1;
    return v;
}

template <typename T>
int upload_vec(T** dst, const std::vector<T>& src) {
    *dst = nullptr;
    const size_t n = std::max<size_t>(src.size(), 1);
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), n * sizeof(T)));
    if (!src.empty()) VBD_CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return VBD_OK;
}

// spreads the low 10 bits of x to every third bit (Morton interleaving)
uint32_t spread3(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// indices of pts in Z-order of their position quantised to 1024 steps per axis of the bounding
// box (ties by index), so that consecutive indices are spatially close
std::vector<int> morton_order(const std::vector<float3>& pts) {
    const size_t n = pts.size();
    std::vector<int> order(n);
    for (size_t k = 0; k < n; ++k) order[k] = static_cast<int>(k);
    if (n == 0) return order;
    float3 lo = pts[0], hi = pts[0];
    for (const float3& p : pts) {
        lo = make_float3(std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z));
        hi = make_float3(std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z));
    }
    const float ext = std::max(std::max(hi.x - lo.x, hi.y - lo.y), std::max(hi.z - lo.z, 1e-12f));
    const float s = 1023.0f / ext;
    std::vector<uint32_t> code(n);
    for (size_t k = 0; k < n; ++k) {
        const float3 p = pts[k];
        auto q = [&](float v, float l) {
            const float t = (v - l) * s;
            return static_cast<uint32_t>(std::isfinite(t) ? std::min(std::max(t, 0.0f), 1023.0f) : 0.0f);
        };
        code[k] = (spread3(q(p.x, lo.x)) << 2) | (spread3(q(p.y, lo.y)) << 1) | spread3(q(p.z, lo.z));
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return code[a] < code[b]; });
    return order;
}

int alloc_zero(void** p, size_t bytes) {
    bytes = std::max<size_t>(bytes, 16);
    VBD_CUDA_TRY(cudaMalloc(p, bytes));
    VBD_CUDA_TRY(cudaMemset(*p, 0, bytes));
    return VBD_OK;
}

}  // namespace

bool self_contact_detect_now(const SelfContact& sc, int it) {
    if (!sc.on) return false;
    if (sc.p.interval == 0) return it == 0;
    if (sc.p.interval >= 1) return it % sc.p.interval == 0;
    return false;
}

void self_contact_free(SelfContact& sc) {
    void* ptrs[] = {sc.tri,      sc.edge,     sc.inc_t_off, sc.inc_t,    sc.inc_e_off,  sc.inc_e,     sc.near_off,
                    sc.near,     sc.rest,     sc.vt_order,     sc.tri_cnt,   sc.tri_off,  sc.tri_cur,    sc.tri_items, sc.edge_cnt,
                    sc.edge_off, sc.edge_cur, sc.edge_items, sc.scan_tmp, sc.vt_count,  sc.vt_list,   sc.ee_count,
                    sc.ee_list,  sc.tv_count, sc.tv_list,   sc.cd,       sc.sc_f,       sc.sc_h0,     sc.sc_h1,
                    sc.ts,       sc.counters, sc.vworld,    sc.tri_box,  sc.edge_box,   sc.flag,      sc.tri_item_box, sc.edge_item_box, sc.vfilt_off, sc.vfilt, sc.efilt_off, sc.efilt, sc.color_start, sc.vcolor,
                    sc.act_v,    sc.act_vcnt, sc.act_rows, sc.act_cnt};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    SelfContact empty;
    sc = empty;
}

int self_contact_create(const VbdModelImpl& m, const SelfContactParams& p, SelfContact& sc) {
    self_contact_free(sc);
    if (!(p.margin >= p.radius))
        return fail(VBD_ERR_INVALID_ARGUMENT,
                    "particle_self_contact_margin is smaller than particle_self_contact_radius, this will result in "
                    "missing contacts and cause instability.\nIt is advisable to make particle_self_contact_margin "
                    "1.5-2 times larger than particle_self_contact_radius.");
    if (!(p.radius > 0.f)) return fail(VBD_ERR_INVALID_ARGUMENT, "self contact: radius must be > 0");
    if (p.vertex_buffer < 1 || p.vertex_buffer > 256 || p.edge_buffer < 1 || p.edge_buffer > 512)
        return fail(VBD_ERR_INVALID_ARGUMENT, "self contact: buffer sizes must be in [1, 256] / [1, 512]");
    if (p.filter_threshold > 4)
        return fail(VBD_ERR_UNSUPPORTED, "self contact: topological filter threshold above 4 is not supported");
    auto bad_csr = [](const std::vector<int>& off, const std::vector<int>& lst, int rows, int maxval) {
        if (off.empty()) return false;
        if (static_cast<int>(off.size()) != rows + 1 || off[0] != 0 || off[rows] != static_cast<int>(lst.size()))
            return true;
        for (int r = 0; r < rows; ++r) {
            if (off[r + 1] < off[r]) return true;
            for (int k = off[r]; k < off[r + 1]; ++k)
                if (lst[k] < 0 || lst[k] >= maxval || (k > off[r] && lst[k] <= lst[k - 1])) return true;
        }
        return false;
    };
    if (bad_csr(p.vertex_filter_off, p.vertex_filter, m.V, m.T) || bad_csr(p.edge_filter_off, p.edge_filter, m.E, m.E))
        return fail(VBD_ERR_INVALID_ARGUMENT,
                    "self contact: external filter lists must be CSR rows of ascending element ids in range");
    if (m.rest_q_h.size() != 3 * static_cast<size_t>(m.V))
        return fail(VBD_ERR_INVALID_ARGUMENT, "self contact needs the model's rest positions (VbdModelDesc.particle_q)");
    const int V = m.V, T = m.T, E = m.E;
    sc.p = p;
    sc.V = V;
    sc.T = T;
    sc.E = E;
    sc.max_disp = static_cast<float>(static_cast<double>(p.margin) * static_cast<double>(p.relaxation) * 0.5);
    std::vector<int> inv(V);
    for (int i = 0; i < V; ++i) inv[m.perm_host[i]] = i;
    // topology
    std::vector<int4> tri(T), edge(E);
    for (int t = 0; t < T; ++t) {
        const int* ti = m.tri_raw_h.data() + 3 * t;
        tri[t] = make_int4(inv[ti[0]], inv[ti[1]], inv[ti[2]], m.pworld_h[ti[0]]);
    }
    double max_edge = 0.0;
    for (int e = 0; e < E; ++e) {
        const int* ei = m.edge_raw_h.data() + 4 * e;
        edge[e] = make_int4(inv[ei[2]], inv[ei[3]], m.pworld_h[ei[2]], 0);
        const float* ra = m.rest_q_h.data() + 3 * static_cast<size_t>(inv[ei[2]]);
        const float* rb = m.rest_q_h.data() + 3 * static_cast<size_t>(inv[ei[3]]);
        const double dx = ra[0] - rb[0], dy = ra[1] - rb[1], dz = ra[2] - rb[2];
        max_edge = std::max(max_edge, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    // cell edge: margin + the longest rest edge (twice the largest rest half-extent), so a query
    // spans about three cells per axis while elements keep their rest size
    sc.cell = static_cast<float>(std::max(static_cast<double>(p.margin) + max_edge, 1e-6));
    // incidence (internal vertex -> triangles with slot, endpoint edges with endpoint)
    std::vector<int> it_off(V + 1, 0), ie_off(V + 1, 0);
    std::vector<int2> it_list, ie_list;
    for (int i = 0; i < V; ++i) {
        const int o = m.perm_host[i];
        for (int k = m.adj_t_off_h[o]; k < m.adj_t_off_h[o + 1]; k += 2)
            it_list.push_back(make_int2(m.adj_t_h[k], m.adj_t_h[k + 1]));
        it_off[i + 1] = static_cast<int>(it_list.size());
        for (int k = m.adj_e_off_h[o]; k < m.adj_e_off_h[o + 1]; k += 2)
            if (m.adj_e_h[k + 1] >= 2) ie_list.push_back(make_int2(m.adj_e_h[k], m.adj_e_h[k + 1] - 2));
        ie_off[i + 1] = static_cast<int>(ie_list.size());
    }
    // n-ring filter sets (internal ids): vertices within threshold - 1 edge rings
    std::vector<int> near_off(V + 1, 0), near_list;
    if (p.filter_threshold >= 2) {
        std::vector<std::vector<int>> ring1(V);
        for (int e = 0; e < E; ++e) {
            ring1[edge[e].x].push_back(edge[e].y);
            ring1[edge[e].y].push_back(edge[e].x);
        }
        for (auto& r : ring1) {
            std::sort(r.begin(), r.end());
            r.erase(std::unique(r.begin(), r.end()), r.end());
        }
        const int depth = p.filter_threshold - 1;
        std::vector<int> seen, frontier, next;
        for (int i = 0; i < V; ++i) {
            seen.assign(1, i);
            frontier.assign(1, i);
            for (int k = 0; k < depth && !frontier.empty(); ++k) {
                next.clear();
                for (int u : frontier)
                    for (int w : ring1[u])
                        if (std::find(seen.begin(), seen.end(), w) == seen.end()) {
                            seen.push_back(w);
                            next.push_back(w);
                        }
                frontier.swap(next);
            }
            std::sort(seen.begin(), seen.end());
            for (int w : seen)
                if (w != i) near_list.push_back(w);
            near_off[i + 1] = static_cast<int>(near_list.size());
        }
    }
    std::vector<int> vworld(V);
    for (int i = 0; i < V; ++i) vworld[i] = m.pworld_h[m.perm_host[i]];
    std::vector<float4> rest(V);
    for (int i = 0; i < V; ++i)
        rest[i] = make_float4(m.rest_q_h[3 * i], m.rest_q_h[3 * i + 1], m.rest_q_h[3 * i + 2], 0.f);
    std::vector<float3> vp(V);
    for (int i = 0; i < V; ++i) vp[i] = make_float3(rest[i].x, rest[i].y, rest[i].z);
    const std::vector<int> vt_order = morton_order(vp);

    int rc = VBD_OK;
    if (!rc) rc = upload_vec(&sc.tri, tri);
    if (!rc) rc = upload_vec(&sc.edge, edge);
    if (!rc) rc = upload_vec(&sc.inc_t_off, it_off);
    if (!rc) rc = upload_vec(&sc.inc_t, it_list);
    if (!rc) rc = upload_vec(&sc.inc_e_off, ie_off);
    if (!rc) rc = upload_vec(&sc.inc_e, ie_list);
    if (!rc) rc = upload_vec(&sc.near_off, near_off);
    if (!rc) rc = upload_vec(&sc.near, near_list);
    if (!rc) rc = upload_vec(&sc.vt_order, vt_order);
    if (!rc) rc = upload_vec(&sc.rest, rest);
    if (!rc) rc = upload_vec(&sc.vworld, vworld);
    sc.C = m.C;
    std::vector<int> vcolor(V, -1);
    for (int c = 0; c < m.C; ++c)
        for (int i = m.color_start[c]; i < m.color_start[c + 1]; ++i) vcolor[i] = c;
    if (!rc) rc = upload_vec(&sc.vcolor, vcolor);
    if (!rc) rc = upload_vec(&sc.color_start, m.color_start);
    if (!rc && !p.vertex_filter_off.empty()) {
        std::vector<int> off(V + 1, 0), lst;
        for (int i = 0; i < V; ++i) {
            const int o = m.perm_host[i];
            lst.insert(lst.end(), p.vertex_filter.begin() + p.vertex_filter_off[o],
                       p.vertex_filter.begin() + p.vertex_filter_off[o + 1]);
            off[i + 1] = static_cast<int>(lst.size());
        }
        rc = upload_vec(&sc.vfilt_off, off);
        if (!rc) rc = upload_vec(&sc.vfilt, lst);
    }
    if (!rc && !p.edge_filter_off.empty()) {
        rc = upload_vec(&sc.efilt_off, p.edge_filter_off);
        if (!rc) rc = upload_vec(&sc.efilt, p.edge_filter);
    }
    const unsigned tn = next_pow2(2LL * std::max(T, 1)), en = next_pow2(2LL * std::max(E, 1));
    sc.tri_mask = tn - 1;
    sc.edge_mask = en - 1;
    sc.tri_items_cap = 2 * std::max(T, 1) + 65536;  // large (stretched) elements take several cells
    sc.edge_items_cap = 8 * std::max(E, 1) + 65536;  // an edge shorter than a cell overlaps at most 8 cells
    auto az = [&](void** ptr, size_t bytes) {
        if (!rc) rc = alloc_zero(ptr, bytes);
    };
    az(reinterpret_cast<void**>(&sc.tri_cnt), tn * sizeof(int));
    az(reinterpret_cast<void**>(&sc.tri_off), tn * sizeof(int));
    az(reinterpret_cast<void**>(&sc.tri_cur), tn * sizeof(int));
    az(reinterpret_cast<void**>(&sc.tri_items), static_cast<size_t>(sc.tri_items_cap) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.edge_cnt), en * sizeof(int));
    az(reinterpret_cast<void**>(&sc.edge_off), en * sizeof(int));
    az(reinterpret_cast<void**>(&sc.edge_cur), en * sizeof(int));
    az(reinterpret_cast<void**>(&sc.edge_items), static_cast<size_t>(sc.edge_items_cap) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.tri_box), 2 * static_cast<size_t>(std::max(T, 1)) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.edge_box), 2 * static_cast<size_t>(std::max(E, 1)) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.tri_item_box), 2 * static_cast<size_t>(sc.tri_items_cap) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.edge_item_box), 2 * static_cast<size_t>(sc.edge_items_cap) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.flag), static_cast<size_t>(V));
    az(reinterpret_cast<void**>(&sc.act_v), static_cast<size_t>(V) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.act_vcnt), static_cast<size_t>(std::max(m.C, 1)) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.act_rows), static_cast<size_t>(V + E) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.act_cnt), 2 * sizeof(int));
    az(reinterpret_cast<void**>(&sc.vt_count), static_cast<size_t>(V) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.vt_list), static_cast<size_t>(V) * p.vertex_buffer * sizeof(int));
    az(reinterpret_cast<void**>(&sc.ee_count), static_cast<size_t>(E) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.ee_list), static_cast<size_t>(E) * p.edge_buffer * sizeof(int));
    az(reinterpret_cast<void**>(&sc.tv_count), static_cast<size_t>(T) * sizeof(int));
    az(reinterpret_cast<void**>(&sc.tv_list), static_cast<size_t>(T) * sc.tcap * sizeof(int));
    az(reinterpret_cast<void**>(&sc.cd), static_cast<size_t>(V) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.sc_f), static_cast<size_t>(V) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.sc_h0), static_cast<size_t>(V) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.sc_h1), static_cast<size_t>(V) * sizeof(float4));
    az(reinterpret_cast<void**>(&sc.ts), static_cast<size_t>(V) * sizeof(unsigned));
    az(reinterpret_cast<void**>(&sc.counters), kScCounters * sizeof(unsigned));
    if (!rc) {
        size_t b1 = 0, b2 = 0;
        cudaError_t e1 = cub::DeviceScan::ExclusiveSum(nullptr, b1, sc.tri_cnt, sc.tri_off, static_cast<int>(tn));
        cudaError_t e2 = cub::DeviceScan::ExclusiveSum(nullptr, b2, sc.edge_cnt, sc.edge_off, static_cast<int>(en));
        if (e1 != cudaSuccess) rc = cuda_fail(e1, "cub::DeviceScan::ExclusiveSum (size query)");
        if (!rc && e2 != cudaSuccess) rc = cuda_fail(e2, "cub::DeviceScan::ExclusiveSum (size query)");
        sc.scan_bytes = std::max(b1, b2);
        az(&sc.scan_tmp, sc.scan_bytes);
    }
    if (!rc && V > 0) {
        fill_u32_kernel<<<(V + 255) / 256, 256>>>(sc.ts, 0x3f800000u /* 1.0f */, V);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "fill_u32_kernel");
        if (!rc) {
            const cudaError_t s = cudaDeviceSynchronize();
            if (s != cudaSuccess) rc = cuda_fail(s, "cudaDeviceSynchronize");
        }
    }
    if (rc) {
        self_contact_free(sc);
        return rc;
    }
    sc.on = true;
    return VBD_OK;
}

int self_contact_load_positions(const VbdModelImpl& m, SelfContact& sc, const float* q, cudaStream_t st) {
    if (m.V == 0) return VBD_OK;
    load_positions_kernel<<<(m.V + 255) / 256, 256, 0, st>>>(m.V, m.perm, q, sc.cd);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

int self_contact_detect(const VbdModelImpl& m, SelfContact& sc, const float4* positions, float4* disp,
                        bool reset_disp, cudaStream_t st) {
    const int V = m.V, T = m.T, E = m.E;
    if (V == 0) return VBD_OK;
    copy_positions_kernel<<<(V + 255) / 256, 256, 0, st>>>(V, positions, sc.cd, reset_disp ? disp : nullptr);
    VBD_CUDA_TRY(cudaGetLastError());
    const unsigned tn = sc.tri_mask + 1, en = sc.edge_mask + 1;
    VBD_CUDA_TRY(cudaMemsetAsync(sc.tri_cnt, 0, tn * sizeof(int), st));
    VBD_CUDA_TRY(cudaMemsetAsync(sc.tri_cur, 0, tn * sizeof(int), st));
    VBD_CUDA_TRY(cudaMemsetAsync(sc.edge_cnt, 0, en * sizeof(int), st));
    VBD_CUDA_TRY(cudaMemsetAsync(sc.edge_cur, 0, en * sizeof(int), st));
    if (T > 0) VBD_CUDA_TRY(cudaMemsetAsync(sc.tv_count, 0, static_cast<size_t>(T) * sizeof(int), st));
    const float inv_cell = 1.0f / sc.cell;
    GridArgs g;
    g.x = sc.cd;
    g.counters = sc.counters;
    g.inv_cell = inv_cell;
    // triangle grid
    g.elem = sc.tri;
    g.n = T;
    g.tri = true;
    g.all_cells = false;
    g.mask = sc.tri_mask;
    g.cnt = sc.tri_cnt;
    g.off = sc.tri_off;
    g.cur = sc.tri_cur;
    g.items = sc.tri_items;
    g.item_box = sc.tri_item_box;
    g.cap = sc.tri_items_cap;
    g.box = sc.tri_box;

    if (T > 0) {
        grid_count_kernel<<<(T + 255) / 256, 256, 0, st>>>(g);
        VBD_CUDA_TRY(cudaGetLastError());
        size_t bytes = sc.scan_bytes;
        VBD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.scan_tmp, bytes, sc.tri_cnt, sc.tri_off, static_cast<int>(tn), st));
        grid_fill_kernel<<<(T + 255) / 256, 256, 0, st>>>(g);
        VBD_CUDA_TRY(cudaGetLastError());
    }
    // edge grid
    g.elem = sc.edge;
    g.n = E;
    g.tri = false;
    g.all_cells = true;
    g.mask = sc.edge_mask;
    g.cnt = sc.edge_cnt;
    g.off = sc.edge_off;
    g.cur = sc.edge_cur;
    g.items = sc.edge_items;
    g.item_box = sc.edge_item_box;
    g.cap = sc.edge_items_cap;
    g.box = sc.edge_box;

    if (E > 0) {
        grid_count_kernel<<<(E + 255) / 256, 256, 0, st>>>(g);
        VBD_CUDA_TRY(cudaGetLastError());
        size_t bytes = sc.scan_bytes;
        VBD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.scan_tmp, bytes, sc.edge_cnt, sc.edge_off, static_cast<int>(en), st));
        grid_fill_kernel<<<(E + 255) / 256, 256, 0, st>>>(g);
        VBD_CUDA_TRY(cudaGetLastError());
    }
    QueryArgs q;
    q.x = sc.cd;
    q.vworld = sc.vworld;
    q.vfilt_off = sc.vfilt_off;
    q.vfilt = sc.vfilt;
    q.efilt_off = sc.efilt_off;
    q.efilt = sc.efilt;
    q.rest = sc.rest;
    q.tri = sc.tri;
    q.edge = sc.edge;
    q.near_off = sc.near_off;
    q.vt_order = sc.vt_order;
    q.near = sc.near;
    q.V = V;
    q.T = T;
    q.E = E;
    q.margin = sc.p.margin;
    q.inv_cell = inv_cell;
    q.par_eps = sc.p.edge_parallel_epsilon;
    q.rest_excl = sc.p.rest_exclusion_radius;
    q.tri_mask = sc.tri_mask;
    q.edge_mask = sc.edge_mask;
    q.tri_cnt = sc.tri_cnt;
    q.tri_off = sc.tri_off;
    q.tri_items = sc.tri_items;
    q.edge_cnt = sc.edge_cnt;
    q.edge_off = sc.edge_off;
    q.edge_items = sc.edge_items;
    q.tri_item_box = sc.tri_item_box;
    q.edge_item_box = sc.edge_item_box;
    q.tri_cap = sc.tri_items_cap;
    q.edge_cap = sc.edge_items_cap;
    q.vbuf = sc.p.vertex_buffer;
    q.ebuf = sc.p.edge_buffer;
    q.vt_count = sc.vt_count;
    q.vt_list = sc.vt_list;
    q.ee_count = sc.ee_count;
    q.ee_list = sc.ee_list;
    q.counters = sc.counters;
    if (T > 0) {
        vt_query_kernel<<<(V + kQueryBlock - 1) / kQueryBlock, kQueryBlock, 0, st>>>(q);
        VBD_CUDA_TRY(cudaGetLastError());
        tri_reverse_kernel<<<(V + 255) / 256, 256, 0, st>>>(V, sc.vt_count, sc.vt_list, sc.p.vertex_buffer,
                                                            sc.tv_count, sc.tv_list, sc.tcap, sc.counters);
        VBD_CUDA_TRY(cudaGetLastError());
        tri_sort_kernel<<<(T + 255) / 256, 256, 0, st>>>(T, sc.tv_count, sc.tv_list, sc.tcap);
        VBD_CUDA_TRY(cudaGetLastError());
    } else {
        VBD_CUDA_TRY(cudaMemsetAsync(sc.vt_count, 0, static_cast<size_t>(V) * sizeof(int), st));
    }
    if (E > 0) {
        VBD_CUDA_TRY(cudaMemsetAsync(sc.ee_count, 0, static_cast<size_t>(E) * sizeof(int), st));
        const long long ee_threads = static_cast<long long>(E) * kEeLanes;
        ee_query_kernel<<<static_cast<unsigned>((ee_threads + kQueryBlock - 1) / kQueryBlock), kQueryBlock, 0, st>>>(q);
        VBD_CUDA_TRY(cudaGetLastError());
        ee_sort_kernel<<<(E + 255) / 256, 256, 0, st>>>(E, sc.ee_count, sc.ee_list, sc.p.edge_buffer);
        VBD_CUDA_TRY(cudaGetLastError());
    }
    VBD_CUDA_TRY(cudaMemsetAsync(sc.flag, 0, static_cast<size_t>(V), st));
    const int nm = std::max(V, E);
    mark_contact_vertices_kernel<<<(nm + 255) / 256, 256, 0, st>>>(V, E, sc.tri, sc.edge, sc.vt_count, sc.vt_list,
                                                                   sc.p.vertex_buffer, sc.ee_count, sc.flag);
    VBD_CUDA_TRY(cudaGetLastError());
    VBD_CUDA_TRY(cudaMemsetAsync(sc.act_vcnt, 0, static_cast<size_t>(std::max(sc.C, 1)) * sizeof(int), st));
    VBD_CUDA_TRY(cudaMemsetAsync(sc.act_cnt, 0, 2 * sizeof(int), st));
    compact_kernel<<<(nm + 255) / 256, 256, 0, st>>>(V, E, sc.flag, sc.vcolor, sc.color_start, sc.vt_count,
                                                     sc.ee_count, sc.act_v, sc.act_vcnt, sc.act_rows, sc.act_cnt);
    VBD_CUDA_TRY(cudaGetLastError());
    // vertices that touch no pair keep a zero contact term until the next detection
    VBD_CUDA_TRY(cudaMemsetAsync(sc.sc_f, 0, static_cast<size_t>(V) * sizeof(float4), st));
    VBD_CUDA_TRY(cudaMemsetAsync(sc.sc_h0, 0, static_cast<size_t>(V) * sizeof(float4), st));
    VBD_CUDA_TRY(cudaMemsetAsync(sc.sc_h1, 0, static_cast<size_t>(V) * sizeof(float4), st));
    return VBD_OK;
}

int self_contact_accumulate(const VbdModelImpl& m, SelfContact& sc, const float4* pos, const float4* prev,
                            int color, float dt, float friction_epsilon, cudaStream_t st) {
    if (color < 0) {
        for (int c = 0; c < m.C; ++c) {
            const int rc = self_contact_accumulate(m, sc, pos, prev, c, dt, friction_epsilon, st);
            if (rc) return rc;
        }
        return VBD_OK;
    }
    const int size = m.color_start[color + 1] - m.color_start[color];
    if (size <= 0) return VBD_OK;
    AccumArgs a;
    a.x = pos;
    a.x0 = prev;
    a.tri = sc.tri;
    a.edge = sc.edge;
    a.inc_t_off = sc.inc_t_off;
    a.inc_e_off = sc.inc_e_off;
    a.inc_t = sc.inc_t;
    a.inc_e = sc.inc_e;
    a.vt_count = sc.vt_count;
    a.vt_list = sc.vt_list;
    a.ee_count = sc.ee_count;
    a.ee_list = sc.ee_list;
    a.tv_count = sc.tv_count;
    a.tv_list = sc.tv_list;
    a.vbuf = sc.p.vertex_buffer;
    a.ebuf = sc.p.edge_buffer;
    a.tcap = sc.tcap;
    a.list = sc.act_v + m.color_start[color];
    a.count = sc.act_vcnt + color;
    a.r = sc.p.radius;
    a.ke = m.soft_ke;
    a.kd = m.soft_kd;
    a.mu = m.soft_mu;
    a.eps_u = friction_epsilon * dt;
    a.dt = dt;
    a.par_eps = sc.p.edge_parallel_epsilon;
    a.f = sc.sc_f;
    a.h0 = sc.sc_h0;
    a.h1 = sc.sc_h1;
    // enough warps for every vertex of the color in one round, capped: the kernel strides
    const long long threads = static_cast<long long>(size) * kAccumLanes;
    const int grid = static_cast<int>(std::min<long long>((threads + 127) / 128, 148 * 16));
    accumulate_kernel<<<grid, 128, 0, st>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

int self_contact_truncate(const VbdModelImpl& m, SelfContact& sc, float4* pos, float4* disp, cudaStream_t st) {
    const int V = m.V;
    if (V == 0) return VBD_OK;
    TruncArgs a;
    a.cd = sc.cd;
    a.disp = disp;
    a.tri = sc.tri;
    a.edge = sc.edge;
    a.vt_count = sc.vt_count;
    a.vt_list = sc.vt_list;
    a.ee_count = sc.ee_count;
    a.ee_list = sc.ee_list;
    a.V = V;
    a.E = m.E;
    a.vbuf = sc.p.vertex_buffer;
    a.ebuf = sc.p.edge_buffer;
    a.eps = sc.p.edge_parallel_epsilon;
    a.gamma = sc.p.relaxation;
    a.ts = sc.ts;
    a.rows = sc.act_rows;
    a.counts = sc.act_cnt;
    const long long n = static_cast<long long>(std::max(V, m.E)) * kPlanarLanes;
    planar_kernel<<<static_cast<int>(std::min<long long>((n + 127) / 128, 148 * 32)), 128, 0, st>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    apply_truncation_kernel<<<(V + 255) / 256, 256, 0, st>>>(V, sc.cd, disp, pos, sc.ts, sc.max_disp);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

}  // namespace vbd
