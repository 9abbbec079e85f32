// Parameter blocks of the cluster step kernel (host and device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "step_params.h"

namespace swb {

namespace dev {
constexpr int kClusterMaxThreads = 768;  // threads per CTA of the cluster step kernels
}

struct ClusterKindDev {
    const uint32_t* offsets;   // [ctas * (stages + 1)]
    const uint32_t* ab;
    const uint32_t* cd;
    const float* rest;
    const float* comp;
    int stages;
    uint32_t smem_lambda;      // byte offset of this kind's multipliers
};

// Per-instance tables and state (one cluster each).
struct ClusterInstance {
    const float4* pos_in;
    const float4* vel_in;
    float4* pos_out;
    float4* vel_out;
    float4* prev_out;
    const float4* force;
    const uint32_t* tri_offsets;
    const uint32_t* tri_list;
    const uint4* tri;
    const uint32_t* patch_begin;   // [ctas + 1]
    ClusterKindDev kind[2];
    const uint32_t* seam_offsets;
    const uint32_t* seam_ab;
    int seam_stages;
    int susp_cta;                  // -1 when absent
    const DevPayloadDef* payload_def;
    const DevPayloadState* payload_in;
    DevPayloadState* payload_out;
    const double* origin_in;
    double* origin_out;
    int* status;
    int recentre;
    int pad;
};

// Packed launches (several structures per cluster): what one CTA runs.
// The loop bounds are those of the whole cluster, so that every CTA of the
// cluster takes the same cluster barriers.
struct ClusterSlot {
    int instance;      // index into the launch's structures; -1 = idle CTA
    int rank_base;     // first cluster rank of that structure
    int stages;        // colour stages per iteration: max over the cluster
    int seam_stages;   // seam stages: max over the cluster
    int suspension;    // 1 when a structure of the cluster has a pilot
    int pad[3];
};

struct ClusterParams {
    const ClusterInstance* instances;  // one per cluster of the launch; packed: [structure][rotation][role]
    int ctas;                          // CTAs per cluster
    const ClusterSlot* slots;          // packed launches: one per CTA
    const int* rotation;               // packed launches: committed buffer per structure
    int role;                          // packed launches: 0 = S->T1, 1 = T1->T2, 2 = T2->T1
    float dt, inv_dt, inv_dt2, damping;
    float3 gravity, ref_velocity;
    int iterations;
    long long copy_budget;
    uint32_t smem_x, smem_v;       // byte offsets of node and force/velocity arrays
    uint32_t smem_offsets;         // byte offset of the CTA's stage offsets
};

}  // namespace swb
