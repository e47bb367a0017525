// vbd_resident.h -- the persistent, shared-memory-resident VBD step (host interface).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "vbd_internal.h"

namespace vbd {

constexpr int kResidentMaxColors = 16;
constexpr int kResidentThreads = 512;

// Per-patch description (device, read once per CTA).
struct PatchMeta {
    int n_local;                              // owned + halo vertices
    int n_owned;
    int n_tri, n_hinge, n_refs;
    int blob_offset;                          // bytes into the static blob (16-byte aligned)
    int blob_bytes;                           // bytes of the static shared-memory image
    int off_refs, off_tri_idx, off_tri_D, off_tri_mat, off_hinge_idx, off_hinge_mat;  // bytes in smem
    int off_pos, off_y, off_prev, off_disp;   // bytes in smem (dynamic part)
    int off_pinfo, off_ccount;
    int l2g_offset;                           // into the local -> global (internal) index array
    int nbr_offset, n_nbr;                    // neighbour patches
    int own_color_start[kResidentMaxColors + 1];   // owned local ranges per color
    int own_color_mid[kResidentMaxColors];         // inside a color: [start, mid) interior, [mid, end) boundary
    int halo_color_start[kResidentMaxColors + 1];  // halo local ranges per color
};

// Everything the resident kernel needs that does not change between steps.
struct ResidentPlan {
    bool ready = false;
    int patches = 0;
    int smem_bytes = 0;
    int max_owned_per_color = 0;
    std::vector<PatchMeta> meta_h;
    PatchMeta* meta = nullptr;
    unsigned char* blob = nullptr;
    int* l2g = nullptr;
    int* nbr = nullptr;
    int* progress = nullptr;                  // [patches], zeroed before every launch
};

struct ResidentLaunch {
    float4* pos;          // GS iterate (internal order), read at start, published per color
    float4* prev;
    float4* y;
    float4* disp;
    const int* ccount;    // contact table (may be NULL)
    const int* cslot;
    int K;
    const int* c_shape;
    const float* c_body_pos;
    const float* c_body_vel;
    const float* c_normal;
    unsigned* status;
    float* q_in;          // outputs (model particle order, [V,3])
    float* q_out;
    float* qd_out;
    int* ccount_clear;    // contact counts to clear at the end (== ccount when contacts were used)
    float dt;
    float friction_epsilon;
    int iterations;
    unsigned spin_limit;
};

// Builds the patch decomposition.  Returns VBD_OK and leaves plan.ready == false when the model
// does not fit (too many colors, patches or shared memory): the caller then uses per-color launches.
int resident_build(const VbdModelImpl& m, ResidentPlan& plan);
void resident_free(ResidentPlan& plan);
// Enqueues one step's resident kernel (plus the progress reset) on `st`.
int resident_enqueue(const VbdModelImpl& m, const ResidentPlan& plan, const ResidentLaunch& L, cudaStream_t st);

}  // namespace vbd
