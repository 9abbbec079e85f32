// Parameter block of the persistent step kernel (host and device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace swb {

constexpr int kDevLevels = 4;

// One CTA-local constraint table (level, kind) as the kernel sees it.
struct DevTable {
    const uint32_t* block_begin;    // [G+1], padded element offsets
    const uint32_t* stage_offsets;  // [G*(stages+1)]
    const uint32_t* ab;             // a | b << 16
    const uint32_t* cd;             // c | d << 16 (dihedral)
    const float* rest;
    const float* comp;              // distance: sign bit = cable
    int stages;
    uint32_t max_count;             // max padded elements per CTA
    uint32_t smem_ab, smem_cd, smem_rest, smem_comp, smem_lambda;  // byte offsets
};

struct DevGlobal {
    const uint32_t* colour_offsets;
    const uint32_t *a, *b, *c, *d;
    const float *rest, *comp;
    float* lambda;
    int colours;
    uint32_t count;
};

// Rigid pilot payload: definition and state, FP32 relative to the origin.
struct DevPayloadDef {
    float mass;
    float3 com_local;
    float3 inertia;          // principal, body frame (diagonal)
    int segments;
    int hang_points;
    // per segment (<= 8): endpoint node local index (in the owner CTA's
    // level-1 patch) or -1, hang point index or -1
    int from_node[8], to_node[8], from_point[8], to_point[8];
    float rest[8], stiffness[8], damping[8];
    float3 hang_local[8];
    float max_residual;
    float min_length;
};

struct DevPayloadState {
    float3 com;
    float4 q;                // w, x, y, z
    float3 v, w;
    float lambda[8];
    float3 line_force, line_moment;
    float max_residual;
    float pad;
};

struct StepParams {
    // state (slot order); in = committed state, out = trial state
    const float4* pos_in;
    const float4* vel_in;
    float4* pos_out;
    float4* vel_out;
    float4* prev_out;
    const float4* force;            // external force per slot (xyz)
    // pressure gather: node CSR of incident triangles (ascending triangle)
    const uint32_t* tri_offsets;    // [N+1] by slot
    const uint32_t* tri_list;
    const uint4* tri;               // slots a, b, c, pressure bits
    // schedule
    int blocks;
    int levels;
    const uint32_t* l1_begin;
    DevTable tab[kDevLevels][2];
    const uint32_t* patch_begin[kDevLevels];
    const uint32_t* patch_slots[kDevLevels];
    DevGlobal glob[2];
    const uint32_t* iface_begin;
    const uint16_t* iface_local;
    const uint32_t* seam_offsets;
    int seam_stages;
    const uint32_t* seam_a;
    const uint32_t* seam_b;
    // physics
    float dt, inv_dt, inv_dt2, damping;
    // 1 - damping, from FP64: the predicted velocity is w - w * damping_loss
    // (w the undamped one), which FP32 keeps unbiased where w * damping
    // would carry the rounding of the factor close to 1, magnified
    // 1 / (1 - damping) times in the velocity it settles to
    float damping_loss;
    float3 gravity, ref_velocity;
    int iterations;
    // suspension
    int susp_block;                 // -1 when absent
    const DevPayloadDef* payload_def;
    const DevPayloadState* payload_in;
    DevPayloadState* payload_out;
    float3* shift_out;              // re-centring shift applied this step
    const double* origin_in;        // frame origin (double3) of the input
    double* origin_out;             // origin_in + shift (written by CTA 0)
    // control
    dev::GridBarrier barrier;
    int* status;
    long long copy_budget;
    // shared memory layout (bytes)
    uint32_t smem_x1, smem_prev1, smem_f1, smem_x2, smem_total;
    uint32_t n1_max, n2_max;
    int recentre;
};

}  // namespace swb
