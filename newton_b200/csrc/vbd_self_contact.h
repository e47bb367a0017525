// vbd_self_contact.h -- cloth self-contact for the VBD step (host interface).
//
// Mirrors SolverVBD's particle_enable_self_contact path (solver_vbd.py:564-603, :2003-2063,
// :2540-2545, :2612-2633, :3221-3237):
//   * detection of vertex-triangle and edge-edge pairs closer than the margin, at the step start
//     and at the iterations the detection interval selects (positions then become the base of
//     the displacements, pos_prev_collision_detection);
//   * per color, the barrier / friction / damping force and Hessian of every pair a vertex of the
//     color takes part in, added to the vertex's block solve;
//   * after every color, the planar division-plane truncation of all displacements and the
//     isotropic clamp to margin * relaxation / 2.
// Detection runs on a hashed uniform grid rebuilt on the device (count, scan, fill, query), with
// no host synchronisation, so a step stays capturable in a CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "vbd_internal.h"

namespace vbd {

struct SelfContactParams {
    float radius = 0.2f;
    float margin = 0.2f;
    float relaxation = 0.85f;
    float edge_parallel_epsilon = 1e-5f;
    float rest_exclusion_radius = 0.f;
    int vertex_buffer = 32;
    int edge_buffer = 64;
    int interval = 0;
    int filter_threshold = 2;
    // external filter lists (host CSR, ascending per row; may be empty)
    std::vector<int> vertex_filter_off, vertex_filter, edge_filter_off, edge_filter;
};

enum SelfContactCounter { kScVtOverflow = 0, kScEeOverflow = 1, kScTvOverflow = 2, kScGridOverflow = 3, kScCounters = 4 };

struct SelfContact {
    bool on = false;
    SelfContactParams p;
    int V = 0, T = 0, E = 0;
    float cell = 0.f;       // grid cell edge
    float max_disp = 0.f;   // margin * relaxation * 0.5
    int tcap = 32;          // colliding vertices kept per triangle
    unsigned tri_mask = 0, edge_mask = 0;
    int tri_items_cap = 0, edge_items_cap = 0;
    // topology, internal vertex ids
    int4* tri = nullptr;     // [T] a, b, c, world of a
    int4* edge = nullptr;    // [E] v0, v1, world of v0, 0
    int* inc_t_off = nullptr;  // [V+1]
    int2* inc_t = nullptr;     // (triangle, slot 0..2), the vertex's triangle adjacency order
    int* inc_e_off = nullptr;  // [V+1]
    int2* inc_e = nullptr;     // (edge, endpoint 0/1), endpoint edges in adjacency order
    int* near_off = nullptr;   // [V+1]
    int* near = nullptr;       // vertices within (threshold - 1) rings, self excluded
    float4* rest = nullptr;    // [V] rest positions (exclusion radius)
    int* vt_order = nullptr;   // [V] order in which vertex queries run (Morton order of rest positions)
    int* vworld = nullptr;     // [V] particle world
    int* vfilt_off = nullptr;  // [V+1] external vertex-triangle filter (internal vertex order), or NULL
    int* vfilt = nullptr;
    int* efilt_off = nullptr;  // [E+1] external edge-edge filter, or NULL
    int* efilt = nullptr;
    // grids
    int *tri_cnt = nullptr, *tri_off = nullptr, *tri_cur = nullptr, *tri_items = nullptr;
    int *edge_cnt = nullptr, *edge_off = nullptr, *edge_cur = nullptr, *edge_items = nullptr;
    float4 *tri_box = nullptr, *edge_box = nullptr;   // [2T], [2E] element boxes of the last detection
    float4 *tri_item_box = nullptr, *edge_item_box = nullptr;  // [2 cap] boxes next to the bucket entries
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
    // detection results
    int *vt_count = nullptr, *vt_list = nullptr;   // [V], [V * vertex_buffer] triangle ids ascending
    int *ee_count = nullptr, *ee_list = nullptr;   // [E], [E * edge_buffer] edge ids ascending
    int *tv_count = nullptr, *tv_list = nullptr;   // [T], [T * tcap] internal vertex ids ascending
    // per-iteration state
    unsigned char* flag = nullptr;  // [V] 1: the vertex takes part in a detected pair
    int C = 0;
    int* color_start = nullptr;  // [C+1] internal vertex ranges of the colors
    int* vcolor = nullptr;       // [V] color of each internal vertex (-1: none)
    int* act_v = nullptr;        // [V] contact-touching vertices, color c in [color_start[c], ...)
    int* act_vcnt = nullptr;     // [C] how many per color
    int* act_rows = nullptr;     // [V + E] non-empty vertex-triangle rows, then non-empty edge rows
    int* act_cnt = nullptr;      // [2] their counts
    float4* cd = nullptr;    // pos_prev_collision_detection (internal order)
    float4* sc_f = nullptr;  // [V] self-contact force
    float4* sc_h0 = nullptr; // [V] Hessian xx xy xz yy
    float4* sc_h1 = nullptr; // [V] Hessian yz zz
    unsigned* ts = nullptr;  // [V] truncation ratio (float bits), 1.0 between truncations
    unsigned* counters = nullptr;  // [kScCounters]
};

int self_contact_create(const VbdModelImpl& m, const SelfContactParams& p, SelfContact& sc);
void self_contact_free(SelfContact& sc);
// Detection at `positions` (internal order): cd := positions, and disp := 0 when reset_disp.
int self_contact_detect(const VbdModelImpl& m, SelfContact& sc, const float4* positions, float4* disp,
                        bool reset_disp, cudaStream_t st);
// Force / Hessian of every pair of the contact-touching vertices of `color` (-1: all colors)
// into sc_f / sc_h0 / sc_h1 (the other vertices hold zero since the last detection).
int self_contact_accumulate(const VbdModelImpl& m, SelfContact& sc, const float4* pos, const float4* prev,
                            int color, float dt, float friction_epsilon, cudaStream_t st);
// Planar truncation of all displacements, then pos := cd + disp for every vertex.
int self_contact_truncate(const VbdModelImpl& m, SelfContact& sc, float4* pos, float4* disp, cudaStream_t st);
// Whether iteration `it` begins with a detection (particle_collision_detection_interval).
bool self_contact_detect_now(const SelfContact& sc, int it);
// Loads model-order positions [V,3] into cd (internal order) -- for detection from a given state.
int self_contact_load_positions(const VbdModelImpl& m, SelfContact& sc, const float* q, cudaStream_t st);

}  // namespace vbd
