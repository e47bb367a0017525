// vbd_internal.h -- host-side structures shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vbd_b200.h"

namespace vbd {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what);

// fn(begin, end) over [0, n) in contiguous chunks on the host's cores, at least `grain` items per
// chunk (serial for small n)
template <typename Fn>
inline void parallel_chunks(int n, Fn&& fn, int grain = 16384) {
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int workers = std::min(std::min(hw, 32), std::max(1, n / std::max(grain, 1)));
    if (workers <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (int w = 0; w < workers; ++w) {
        const int b = static_cast<int>(static_cast<long long>(n) * w / workers);
        const int e = static_cast<int>(static_cast<long long>(n) * (w + 1) / workers);
        pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto& t : pool) t.join();
}

#define VBD_CUDA_TRY(expr)                                       \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return ::vbd::cuda_fail(_e, #expr); \
    } while (0)

// Per-shape data the device needs (16-byte members first).
struct DevShape {
    float4 mat;        // mixed contact (ke, kd, mu) and the shape margin
    float4 pos;        // xyz + geo type (as float)
    float4 rot;        // quaternion xyzw
    float4 scale;      // xyz + flags (as float)
    int world;
    int pad[3];
};

// Device-resident model in the B200 layout:
//  * vertices are renumbered color-major (color c occupies [color_start[c], color_start[c+1]) of
//    the internal order, ascending original index inside a color), so each per-color launch
//    reads its vertices' own data contiguously;
//  * each vertex owns a contiguous run of element records (triangles first, then hinges): the
//    element's vertex ids in internal numbering plus its rest data, replicated per incident
//    vertex, so the sweep streams records instead of chasing CSR -> element -> data.
struct VbdModelImpl {
    int device = 0;
    int V = 0, T = 0, E = 0, S = 0, C = 0;
    int swept = 0;                    // vertices covered by a color (the rest are never solved)
    int n_tri_rec = 0, n_edge_rec = 0;
    bool fused_commit = true;         // colors are conflict-free for every element stencil
    bool any_tri_damping = false, any_edge_damping = false;
    float gravity[3] = {0, 0, 0};
    float gravity_norm = 0.f;
    std::vector<int> color_start;     // [C+1] internal offsets
    std::vector<int> perm_host;       // internal -> original
    // device arrays
    int* perm = nullptr;              // [V] internal -> original
    int* inv_perm = nullptr;          // [V] original -> internal
    float4* pinfo = nullptr;          // [V] (mass, inv_mass, radius, flags as float bits)
    int4* vadj = nullptr;             // [V] (tri_begin, tri_end, edge_begin, edge_end)
    int4* tri_idx = nullptr;          // [n_tri_rec] internal vertex ids (order packed in bits 30-31 of .w)
    float4* tri_D = nullptr;          // [n_tri_rec] DmInv 00, 01, 10, 11
    float4* tri_mat = nullptr;        // [n_tri_rec] area, mu, lambda, kd
    int4* edge_idx = nullptr;         // [n_edge_rec] o0, o1, v0, v1 (internal ids); order in bits 30-31 of .x
    float4* edge_mat = nullptr;       // [n_edge_rec] rest angle, rest length, ke, kd
    DevShape* shapes = nullptr;       // [S]
    int n_worlds = 0;                 // W: 1 + the largest particle or shape world id
    int* world_shape_offsets = nullptr;   // [W+2] CSR rows: world w -> its shapes and the global ones
    int* world_shapes = nullptr;      //     (ascending shape id); row W: every shape (global particles)
    int* nbr8 = nullptr;              // [V*8] first 8 distinct one-ring neighbours (internal ids, -1 padded)
    float4* vfeat = nullptr;          // [V] per-vertex material features: mean log10 tri ke, tri ka,
                                      //     edge ke over incident elements, characteristic length
    int* particle_world = nullptr;    // [V] original order (collide)
    int* particle_flags_orig = nullptr;   // [V] original order (collide)
    float* particle_radius_orig = nullptr;  // [V] original order (collide)
    std::vector<DevShape> shapes_host;
    // host copies of the layout (used to build the shared-memory-resident patches)
    std::vector<float4> pinfo_h;
    std::vector<int4> vadj_h, tri_idx_h, edge_idx_h;
    std::vector<float4> tri_D_h, tri_mat_h, edge_mat_h;
    std::vector<int> tri_elem_h, edge_elem_h;   // element id of each record (dedupe per patch)
    std::vector<float> rest_q_h;                // [3V] initial positions in internal order (may be empty)
    // raw topology in model order (self-contact layer) and the model-level contact material
    std::vector<int> tri_raw_h, edge_raw_h, adj_t_off_h, adj_t_h, adj_e_off_h, adj_e_h, pworld_h;
    float soft_ke = 0.f, soft_kd = 0.f, soft_mu = 0.f;
};

// learned warm start (vbd_mlp.cu): per-vertex features after the forward pass (model-order rows;
// corr_prev in model order), and the warm-start displacement = network output (in characteristic
// lengths) * length.  mode: VBD_FEATURES_CORRECTIONS or VBD_FEATURES_KINEMATIC; dt: the step's
// (kinematic set)
int mlp_features_launch(const VbdModelImpl& m, const float4* prev, const float4* y, const int* ccount,
                        const float* corr_prev, const float* mean, const float* inv_std, float* out, int mode,
                        float dt, cudaStream_t st);
int mlp_scale_launch(const VbdModelImpl& m, const float* pred, float* delta, cudaStream_t st);
// the step mode's learned start in one tcgen05 launch: features of every internal vertex (corr_prev
// in the internal order), inference, the bounded start added to disp and pos
int mlp_step_start(const VbdModelImpl& m, const float* params, const float4* prev, const float4* y, const int* ccount,
                   const float* corr_prev, const float* mean, const float* inv_std, int mode, float dt, float4* disp,
                   float4* pos, cudaStream_t st);

}  // namespace vbd

struct VbdModel {
    vbd::VbdModelImpl m;
};
