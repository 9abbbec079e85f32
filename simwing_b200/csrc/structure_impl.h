// Host-side state of one device structure (the swb_structure handle).
#pragma once

#include "cluster_params.h"
#include "cluster_schedule.h"
#include "common.h"
#include "contact_surface.h"
#include "schedule.h"
#include "step_params.h"

#include <string>
#include <vector>

namespace swb {

void cuda_check(cudaError_t e, const char* what);

// Device control word block: status[0] = kStatus* bits, status[1] = detail,
// barrier counters and the re-centring shift of the last substep.
struct Control {
    int status[2];
    unsigned int count;
    unsigned int generation;
    float3 shift;
    float pad;
};

constexpr int kDiagBlocks = 148;

// Host entry points of the packed cluster kernel (several structures per
// cluster), defined beside the kernels.
cudaError_t packed_kernel_limits(int max_dynamic_smem, bool non_portable_cluster);
// Dynamic shared memory a step, taping, packed or reverse kernel may request
// on this device: the opt-in maximum less the largest static shared memory
// among those kernels (at least 2 KB).
size_t dynamic_smem_limit(const cudaDeviceProp& prop);
// `membranes`: the launch carries membrane elements (the membrane instantiation)
cudaError_t packed_kernel_occupancy(int* clusters, const cudaLaunchConfig_t& cfg, bool membranes);
cudaError_t packed_kernel_launch(const cudaLaunchConfig_t& cfg, const ClusterParams& params, bool membranes);
// ... and of the single-structure kernels the differentiable rollout drives.
cudaError_t plain_cluster_launch(const cudaLaunchConfig_t& cfg, const ClusterParams& params);
cudaError_t tape_kernel_limits(int max_dynamic_smem, bool non_portable_cluster);
cudaError_t tape_kernel_launch(const cudaLaunchConfig_t& cfg, const ClusterParams& params);
cudaError_t adjoint_kernel_limits(int max_dynamic_smem, bool non_portable_cluster);
cudaError_t adjoint_kernel_launch(const cudaLaunchConfig_t& cfg, const AdjointParams& params);

// Status words written by the step kernels -> status and message.
swb_status decode_status(const int status[2], std::string& message);

// Helper clusters a contact launch may add beside the structure's cluster.
constexpr int kMaxContactHelpers = 8;
// Contact surfaces with fewer candidate rows (vertices plus edges) keep
// their detection phases on the structure's cluster.
constexpr uint32_t kContactHelperRows = 16384;

struct StructureImpl {
    OwnedDefinition def;
    bool cluster_mode = false;
    // the momentum guard of free structures applies (soft_body.cpp:1192-1202)
    bool momentum_guard = false;
    Schedule sched;            // grid schedule (cluster_mode == false)
    ClusterSchedule csched;    // cluster schedule (cluster_mode == true)
    std::vector<uint32_t> slot_of_node, node_of_slot;
    int susp_owner = -1;       // CTA owning the suspension endpoint nodes
    uint32_t susp_base = 0;    // first slot of that CTA's patch
    ClusterParams cparams{};
    ClusterInstance cluster_base{};
    ClusterInstance* d_instances = nullptr;
    uint32_t cluster_smem = 0;
    uint64_t fingerprint = 0;
    int device = -1;
    int sm_count = 0;
    int G = 0;
    int contact_helpers = 0;  // helper clusters of the contact detection phases
    // line-line contact (swb_structure_set_line_contact)
    bool line_contact = false;
    LineContactDev lines_host{};
    LineContactDev* d_lines = nullptr;
    int threads = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void*> owned;
    // state buffers (three so that a multi-substep step can be rolled back)
    float4* d_pos[3] = {};
    float4* d_vel[3] = {};
    float4* d_prev[3] = {};
    DevPayloadState* d_payload[3] = {};
    double* d_origin[3] = {};
    double origin0[3] = {0.0, 0.0, 0.0};  // the FP64 origin the initial FP32 offsets are taken from
    int cur = 0;
    std::vector<float> inv_mass;  // by slot
    float4* d_force = nullptr;
    float4* h_force = nullptr;    // pinned staging
    uint4* d_tri = nullptr;
    uint32_t* d_tri_off = nullptr;
    uint32_t* d_tri_list = nullptr;
    uint32_t* d_diag_a = nullptr;
    float* d_mres[3] = {nullptr, nullptr, nullptr};  // membrane residual per record, per state buffer
    // fabric self-contact: the surface, its device tables and scratch, and
    // the contact diagnostics per state buffer
    ContactSurface contact_surface;
    ContactDev* d_contact = nullptr;
    ContactDev contact_host{};  // host copy of *d_contact (device pointers)
    size_t smem_cap = 0;  // dynamic shared memory a step kernel may request on this device
    ContactDiagDev* d_cdiag[3] = {nullptr, nullptr, nullptr};
    // the committed multiplier table while a step runs (restored on failure)
    ContactEntry* d_table_commit = nullptr;
    uint32_t* d_meta_commit = nullptr;
    uint4* d_diag_mem = nullptr;      // membrane records for the diagnostics: corner slots, record index
    uint32_t* d_diag_b = nullptr;
    float* d_diag_rest = nullptr;
    uint8_t* d_diag_kind = nullptr;
    double* d_diag_partials = nullptr;
    DevPayloadDef* d_payload_def = nullptr;
    DevPayloadDef payload_def_host{};
    std::vector<size_t> segment_order;  // device segment k -> definition index
    Control* d_control = nullptr;
    StepParams params{};
    uint32_t sched_n1_max = 0, sched_n2_max = 0;
    // host mirror of the adapter state
    std::vector<swb_vec3> pending;
    std::vector<double> pressure;
    bool forces_dirty = false;
    bool pressure_dirty = false;
    swb_vec3 last_applied{0, 0, 0};
    uint64_t accepted = 0;
    double time = 0.0;
    double last_dt = 1.0 / 120.0;
    double last_ms = 0.0;

    ~StructureImpl();
    void build(const swb_structure_definition& definition, const swb_solver_options* options);
    void upload_cluster_tables();
    void setup_contact(const swb_solver_options& opt);
    void setup_line_contact();
    void upload_instances();
    // The step with the force buffer already written on the device (the
    // coupling's impulse gather): skips the upload of the pending loads.
    bool device_forces = false;
    // the cluster step kernel for this structure (the membrane
    // instantiation when it has membrane elements)
    void (*step_kernel() const)(ClusterParams);
    void upload_grid_tables();
    void finish_build(const swb_solver_options& opt, const cudaDeviceProp& prop);
    void upload_pressure();
    void upload_forces();
    void validate_settings(const swb_step_settings& st) const;
    // the raw status words of the last step and the exception details of a
    // failed one
    int last_status[2] = {0, 0};
    // autotuner: candidates and choice (empty when not tuned); device time
    // of `reps` trial substeps from the committed state into the spare
    // buffer, which leave the state untouched
    swb_autotune_report tune{};
    double time_trial(const swb_step_settings& st, int warm, int reps);
    swb_error_detail failure_detail(swb_status status, std::string& message);
    void launch_substep(const swb_step_settings& st, int in, int out, bool first);
    swb_status read_status(std::string& message);
    // Accepts `steps` steps that left the state in buffer `new_cur`: the
    // pending loads are consumed, the counters advance.
    void commit(int new_cur, int steps, const swb_step_settings& st);
    swb_status step(const swb_step_settings& st, int steps, swb_diagnostics* out);
    void copy_state(int from, int to);
    void fetch(std::vector<float4>& pos, std::vector<float4>& prev, std::vector<float4>& vel, DevPayloadState& pay,
               double origin[3]) const;
    void diagnostics(swb_diagnostics* out) const;
};

}  // namespace swb

struct swb_structure {
    swb::StructureImpl s;
    bool borrowed = false;  // owned by a batch; swb_structure_destroy leaves it alone
};
