// vbd_setup.cu -- the model set-up tables on the GPU.
//
// Device counterparts of the host functions of vbd_mesh.cpp and vbd_coloring.cpp.  They read and
// write device arrays and produce the same tables, element for element:
//   vbd_mesh_edge_adjacency_device  = vbd_mesh_edge_adjacency  (MeshAdjacency._compute_edge_adjacency,
//                                     newton/_src/utils/mesh.py:465-531)
//   vbd_mesh_vertex_csr_device      = vbd_mesh_vertex_csr      (init_vertex_adjacency and the count /
//                                     fill kernels, utils/mesh.py:595-655, :675-772)
//   vbd_trimesh_graph_edges_device  = vbd_trimesh_graph_edges  (construct_trimesh_graph_edges,
//                                     sim/graph_coloring.py:99-197)
// The host versions are serial passes whose order rules decide the tables: an edge is numbered
// when first met in slot order, a vertex's records are in element order, conflict edges are the
// lexicographically sorted unique pairs.  Here every rule becomes a stable radix sort (CUB) plus
// flag / scan passes:
//   * edge table: the 3 nt edge slots sorted by their undirected key; within a key the slots stay
//     in slot order (stable sort), so a group's first slot is the first occurrence and its second
//     slot the second triangle; edges are numbered by an exclusive scan over "first occurrence"
//     flags indexed by slot, which is the host's numbering in order of first appearance;
//   * vertex CSR: the entries sorted by vertex (stable, so element order within a vertex);
//     offsets from a per-vertex count and an exclusive scan;
//   * conflict edges: the (min, max) pairs as 64-bit keys, sorted and made unique.
// Temporary memory is allocated per call and freed before it returns.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <cstdint>
#include <string>
#include <vector>

#include "vbd_internal.h"

namespace {

using ull = unsigned long long;
constexpr ull kNoPair = ~0ull;

// temporary buffers of one call, freed when the scope ends (after the call has synchronized its
// stream; cudaFree waits for the device anyway).  The set-up path runs once per model.
class Scratch {
  public:
    explicit Scratch(cudaStream_t) {}
    ~Scratch() {
        for (void* p : ptrs_) cudaFree(p);
    }
    template <typename T>
    cudaError_t get(T** p, size_t n) {
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, (n > 0 ? n : 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        ptrs_.push_back(q);
        *p = static_cast<T*>(q);
        return cudaSuccess;
    }

  private:
    std::vector<void*> ptrs_;
};

#define SETUP_TRY(expr)                                                   \
    do {                                                                  \
        const cudaError_t e_ = (expr);                                    \
        if (e_ != cudaSuccess) return vbd::cuda_fail(e_, #expr);          \
    } while (0)

inline int grid_for(size_t n, int block) { return static_cast<int>((n + block - 1) / block); }

// bits needed for keys in [0, n]
inline int key_bits(long long n) {
    int b = 1;
    while (b < 62 && (1ll << b) <= n) ++b;
    return b;
}

// ---- edge table ---------------------------------------------------------------------------------
__global__ void edge_keys_kernel(const int32_t* tris, int32_t nt, ull* keys, int32_t* slot) {
    const long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (j >= 3ll * nt) return;
    const long long t = j / 3;
    const int k = static_cast<int>(j - 3 * t);
    const int32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
    const uint32_t lo = static_cast<uint32_t>(a < b ? a : b), hi = static_cast<uint32_t>(a < b ? b : a);
    keys[j] = (static_cast<ull>(lo) << 32) | hi;
    slot[j] = static_cast<int32_t>(j);
}

// head flags of the sorted keys, and the first-occurrence flag of each group's first slot
__global__ void edge_heads_kernel(const ull* skeys, const int32_t* sslot, int32_t S, int32_t* head, int32_t* first_flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const bool h = i == 0 || skeys[i] != skeys[i - 1];
    head[i] = h ? 1 : 0;
    if (h) first_flag[sslot[i]] = 1;
}

// per group (numbered in key order): its first slot and the sorted position of its head
__global__ void edge_groups_kernel(const int32_t* head, const int32_t* group_incl, const int32_t* sslot, int32_t S,
                                   int32_t* group_first_slot, int32_t* group_head_pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S || !head[i]) return;
    const int g = group_incl[i] - 1;
    group_first_slot[g] = sslot[i];
    group_head_pos[g] = i;
}

__global__ void edge_fill_kernel(const int32_t* tris, const int32_t* sslot, const int32_t* group_incl,
                                 const int32_t* group_first_slot, const int32_t* group_head_pos,
                                 const int32_t* edge_of_slot, int32_t S, int32_t* edge_indices, int32_t* edge_tri,
                                 int32_t* tri_edge, int32_t* extra) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int g = group_incl[i] - 1;
    const int e = edge_of_slot[group_first_slot[g]];
    const int pos = i - group_head_pos[g];
    const int j = sslot[i];
    const int t = j / 3, k = j - 3 * (j / 3);
    tri_edge[j] = e;
    const int32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3], o = tris[3 * t + (k + 2) % 3];
    if (pos == 0) {
        const bool single = i + 1 == S || group_incl[i + 1] != group_incl[i];
        edge_indices[4 * e] = o;
        edge_indices[4 * e + 2] = a;
        edge_indices[4 * e + 3] = b;
        edge_tri[2 * e] = t;
        if (single) {
            edge_indices[4 * e + 1] = -1;
            edge_tri[2 * e + 1] = -1;
        }
    } else if (pos == 1) {
        edge_indices[4 * e + 1] = o;
        edge_tri[2 * e + 1] = t;
    } else {
        atomicAdd(extra, 1);
    }
}

// ---- vertex CSR -----------------------------------------------------------------------------------
struct SlotTable {
    int32_t s[16];
};

__global__ void csr_keys_kernel(const int32_t* entries, long long n, int32_t V, uint32_t* keys, int32_t* idx,
                                int32_t* counts, int32_t* bad) {
    const long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (j >= n) return;
    const int32_t v = entries[j];
    uint32_t key = static_cast<uint32_t>(V);  // skipped entries sort after every vertex
    if (v >= 0 && v < V) {
        key = static_cast<uint32_t>(v);
        atomicAdd(&counts[v], 1);
    } else if (v != -1) {
        atomicExch(bad, 1);
    }
    keys[j] = key;
    idx[j] = static_cast<int32_t>(j);
}

__global__ void csr_offsets_kernel(const int32_t* start, int32_t V, int32_t* offsets) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v <= V) offsets[v] = 2 * start[v];
}

// the valid entries are the first `*total` sorted ones (the skipped ones' key sorts after every
// vertex); `total` lives on the device, so the grid covers all entries and the rest return
__global__ void csr_fill_kernel(const int32_t* sidx, const int32_t* total, int32_t per, SlotTable slots,
                                int32_t* values) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *total) return;
    const int j = sidx[i];
    const int e = j / per;
    values[2 * i] = e;
    values[2 * i + 1] = slots.s[j - e * per];
}

// ---- conflict-graph edges -------------------------------------------------------------------------
__constant__ int kHingePairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

__global__ void pair_keys_kernel(const int32_t* tris, long long nt, const int32_t* bend, long long nb, int32_t N,
                                 ull* keys, int32_t* bad) {
    const long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const long long P = 3 * nt + 6 * nb;
    if (p >= P) return;
    int32_t a, b;
    if (p < 3 * nt) {
        const long long t = p / 3;
        const int q = static_cast<int>(p - 3 * t);  // (0,1) (0,2) (1,2)
        a = tris[3 * t + (q == 2 ? 1 : 0)];
        b = tris[3 * t + (q == 0 ? 1 : 2)];
        if (a < 0 || a >= N || b < 0 || b >= N) {
            atomicExch(bad, 1);
            keys[p] = kNoPair;
            return;
        }
    } else {
        const long long r = p - 3 * nt;
        const long long e = r / 6;
        const int q = static_cast<int>(r - 6 * e);
        a = bend[4 * e + kHingePairs[q][0]];
        b = bend[4 * e + kHingePairs[q][1]];
        if (a >= N || b >= N) {
            atomicExch(bad, 2);
            keys[p] = kNoPair;
            return;
        }
        if (a < 0 || b < 0) {
            keys[p] = kNoPair;
            return;
        }
    }
    if (a == b) {
        keys[p] = kNoPair;
        return;
    }
    const uint32_t lo = static_cast<uint32_t>(a < b ? a : b), hi = static_cast<uint32_t>(a < b ? b : a);
    keys[p] = (static_cast<ull>(lo) << 32) | hi;
}

__global__ void pair_decode_kernel(const ull* ukeys, long long n, int32_t* edges) {
    const long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const ull key = ukeys[k];
    edges[2 * k] = static_cast<int32_t>(key >> 32);
    edges[2 * k + 1] = static_cast<int32_t>(key & 0xffffffffull);
}

}  // namespace

extern "C" int vbd_mesh_edge_adjacency_device(const int32_t* tris, int32_t nt, int32_t* edge_indices, int32_t* edge_tri,
                                              int32_t* tri_edge, int32_t* num_edges, int32_t* nonmanifold,
                                              void* stream) {
    if (nt < 0 || nt > (1 << 29) || (nt > 0 && (!tris || !edge_indices || !edge_tri || !tri_edge)) || !num_edges)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mesh_edge_adjacency_device: invalid arguments");
    *num_edges = 0;
    if (nonmanifold) *nonmanifold = 0;
    if (nt == 0) return VBD_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int32_t S = 3 * nt;
    Scratch scr(st);
    ull *keys = nullptr, *skeys = nullptr;
    int32_t *slot = nullptr, *sslot = nullptr, *head = nullptr, *first_flag = nullptr, *group_incl = nullptr,
            *edge_of_slot = nullptr, *group_first = nullptr, *group_head = nullptr, *counters = nullptr;
    SETUP_TRY(scr.get(&keys, S));
    SETUP_TRY(scr.get(&skeys, S));
    SETUP_TRY(scr.get(&slot, S));
    SETUP_TRY(scr.get(&sslot, S));
    SETUP_TRY(scr.get(&head, S));
    SETUP_TRY(scr.get(&first_flag, S));
    SETUP_TRY(scr.get(&group_incl, S));
    SETUP_TRY(scr.get(&edge_of_slot, S));
    SETUP_TRY(scr.get(&group_first, S));
    SETUP_TRY(scr.get(&group_head, S));
    SETUP_TRY(scr.get(&counters, 1));
    SETUP_TRY(cudaMemsetAsync(first_flag, 0, sizeof(int32_t) * S, st));
    SETUP_TRY(cudaMemsetAsync(counters, 0, sizeof(int32_t), st));
    edge_keys_kernel<<<grid_for(S, 256), 256, 0, st>>>(tris, nt, keys, slot);
    size_t b_sort = 0, b_scan1 = 0, b_scan2 = 0;
    SETUP_TRY(cub::DeviceRadixSort::SortPairs(nullptr, b_sort, keys, skeys, slot, sslot, S, 0, 64, st));
    SETUP_TRY(cub::DeviceScan::InclusiveSum(nullptr, b_scan1, head, group_incl, S, st));
    SETUP_TRY(cub::DeviceScan::ExclusiveSum(nullptr, b_scan2, first_flag, edge_of_slot, S, st));
    void* temp = nullptr;
    const size_t b_temp = std::max(b_sort, std::max(b_scan1, b_scan2));
    SETUP_TRY(scr.get(reinterpret_cast<unsigned char**>(&temp), b_temp));
    size_t b = b_temp;
    SETUP_TRY(cub::DeviceRadixSort::SortPairs(temp, b, keys, skeys, slot, sslot, S, 0, 64, st));
    edge_heads_kernel<<<grid_for(S, 256), 256, 0, st>>>(skeys, sslot, S, head, first_flag);
    b = b_temp;
    SETUP_TRY(cub::DeviceScan::InclusiveSum(temp, b, head, group_incl, S, st));
    b = b_temp;
    SETUP_TRY(cub::DeviceScan::ExclusiveSum(temp, b, first_flag, edge_of_slot, S, st));
    edge_groups_kernel<<<grid_for(S, 256), 256, 0, st>>>(head, group_incl, sslot, S, group_first, group_head);
    edge_fill_kernel<<<grid_for(S, 256), 256, 0, st>>>(tris, sslot, group_incl, group_first, group_head, edge_of_slot,
                                                         S, edge_indices, edge_tri, tri_edge, counters);
    SETUP_TRY(cudaGetLastError());
    int32_t ne = 0, extra = 0;
    SETUP_TRY(cudaMemcpyAsync(&ne, group_incl + (S - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SETUP_TRY(cudaMemcpyAsync(&extra, counters, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SETUP_TRY(cudaStreamSynchronize(st));
    *num_edges = ne;
    if (nonmanifold) *nonmanifold = extra;
    return VBD_OK;
}

extern "C" int vbd_mesh_vertex_csr_device(const int32_t* entries, int32_t n_elements, int32_t per_element,
                                          const int32_t* slot_of, int32_t particle_count, int32_t* values,
                                          int32_t* offsets, int32_t* num_records, void* stream) {
    if (n_elements < 0 || per_element < 1 || per_element > 16 || particle_count < 0 || !offsets || !slot_of ||
        (n_elements > 0 && (!entries || !values)) ||
        static_cast<long long>(n_elements) * per_element > (1ll << 30))
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mesh_vertex_csr_device: invalid arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = static_cast<long long>(n_elements) * per_element;
    const int32_t V = particle_count;
    Scratch scr(st);
    uint32_t *keys = nullptr, *skeys = nullptr;
    int32_t *idx = nullptr, *sidx = nullptr, *counts = nullptr, *start = nullptr, *bad = nullptr;
    SETUP_TRY(scr.get(&keys, n));
    SETUP_TRY(scr.get(&skeys, n));
    SETUP_TRY(scr.get(&idx, n));
    SETUP_TRY(scr.get(&sidx, n));
    SETUP_TRY(scr.get(&counts, static_cast<size_t>(V) + 1));
    SETUP_TRY(scr.get(&start, static_cast<size_t>(V) + 1));
    SETUP_TRY(scr.get(&bad, 1));
    SETUP_TRY(cudaMemsetAsync(counts, 0, sizeof(int32_t) * (static_cast<size_t>(V) + 1), st));
    SETUP_TRY(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
    if (n > 0) csr_keys_kernel<<<grid_for(n, 256), 256, 0, st>>>(entries, n, V, keys, idx, counts, bad);
    size_t b_sort = 0, b_scan = 0;
    const int bits = key_bits(V);
    SETUP_TRY(cub::DeviceScan::ExclusiveSum(nullptr, b_scan, counts, start, V + 1, st));
    if (n > 0)
        SETUP_TRY(cub::DeviceRadixSort::SortPairs(nullptr, b_sort, keys, skeys, idx, sidx, static_cast<int>(n), 0, bits,
                                                  st));
    void* temp = nullptr;
    const size_t b_temp = std::max(b_sort, b_scan);
    SETUP_TRY(scr.get(reinterpret_cast<unsigned char**>(&temp), b_temp));
    size_t b = b_temp;
    SETUP_TRY(cub::DeviceScan::ExclusiveSum(temp, b, counts, start, V + 1, st));
    csr_offsets_kernel<<<grid_for(static_cast<size_t>(V) + 1, 256), 256, 0, st>>>(start, V, offsets);
    int32_t total = 0, badv = 0;
    SETUP_TRY(cudaMemcpyAsync(&total, start + V, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SETUP_TRY(cudaMemcpyAsync(&badv, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    if (n > 0) {
        b = b_temp;
        SETUP_TRY(cub::DeviceRadixSort::SortPairs(temp, b, keys, skeys, idx, sidx, static_cast<int>(n), 0, bits, st));
        SlotTable tab;
        for (int k = 0; k < 16; ++k) tab.s[k] = k < per_element ? slot_of[k] : 0;
        csr_fill_kernel<<<grid_for(n, 256), 256, 0, st>>>(sidx, start + V, per_element, tab, values);
    }
    SETUP_TRY(cudaGetLastError());
    SETUP_TRY(cudaStreamSynchronize(st));
    if (badv) return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mesh_vertex_csr_device: vertex id out of range");
    if (num_records) *num_records = total;
    return VBD_OK;
}

extern "C" int vbd_trimesh_graph_edges_device(int32_t num_nodes, const int32_t* tris, int64_t nt, const int32_t* bend,
                                              int64_t nb, int32_t* edges_out, int64_t* num_edges_out, void* stream) {
    if (num_nodes < 0 || nt < 0 || nb < 0 || (nt > 0 && !tris) || (nb > 0 && !bend) ||
        ((nt > 0 || nb > 0) && !edges_out) || !num_edges_out || 3 * nt + 6 * nb > (1ll << 31) - 1)
        return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_trimesh_graph_edges_device: invalid arguments");
    *num_edges_out = 0;
    const long long P = 3 * nt + 6 * nb;
    if (P == 0) return VBD_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Scratch scr(st);
    ull *keys = nullptr, *skeys = nullptr, *ukeys = nullptr;
    int32_t* bad = nullptr;
    long long* nunique = nullptr;
    SETUP_TRY(scr.get(&keys, P));
    SETUP_TRY(scr.get(&skeys, P));
    SETUP_TRY(scr.get(&ukeys, P));
    SETUP_TRY(scr.get(&bad, 1));
    SETUP_TRY(scr.get(&nunique, 1));
    SETUP_TRY(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
    pair_keys_kernel<<<grid_for(P, 256), 256, 0, st>>>(tris, nt, bend, nb, num_nodes, keys, bad);
    size_t b_sort = 0, b_uniq = 0;
    SETUP_TRY(cub::DeviceRadixSort::SortKeys(nullptr, b_sort, keys, skeys, static_cast<int>(P), 0, 64, st));
    SETUP_TRY(cub::DeviceSelect::Unique(nullptr, b_uniq, skeys, ukeys, nunique, static_cast<int>(P), st));
    void* temp = nullptr;
    const size_t b_temp = std::max(b_sort, b_uniq);
    SETUP_TRY(scr.get(reinterpret_cast<unsigned char**>(&temp), b_temp));
    size_t b = b_temp;
    SETUP_TRY(cub::DeviceRadixSort::SortKeys(temp, b, keys, skeys, static_cast<int>(P), 0, 64, st));
    b = b_temp;
    SETUP_TRY(cub::DeviceSelect::Unique(temp, b, skeys, ukeys, nunique, static_cast<int>(P), st));
    long long nu = 0;
    ull last = 0;
    int32_t badv = 0;
    SETUP_TRY(cudaMemcpyAsync(&nu, nunique, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SETUP_TRY(cudaMemcpyAsync(&badv, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SETUP_TRY(cudaStreamSynchronize(st));
    if (badv == 1) return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_trimesh_graph_edges_device: triangle vertex out of range");
    if (badv == 2) return vbd::fail(VBD_ERR_INVALID_ARGUMENT, "vbd_trimesh_graph_edges_device: hinge vertex out of range");
    if (nu > 0) {
        SETUP_TRY(cudaMemcpyAsync(&last, ukeys + (nu - 1), sizeof(ull), cudaMemcpyDeviceToHost, st));
        SETUP_TRY(cudaStreamSynchronize(st));
        if (last == kNoPair) --nu;  // the skipped pairs' key sorts last
    }
    if (nu > 0) pair_decode_kernel<<<grid_for(nu, 256), 256, 0, st>>>(ukeys, nu, edges_out);
    SETUP_TRY(cudaGetLastError());
    SETUP_TRY(cudaStreamSynchronize(st));
    *num_edges_out = nu;
    return VBD_OK;
}
