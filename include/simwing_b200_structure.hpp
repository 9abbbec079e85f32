// simwing_b200_structure.hpp -- C++ mirror of SimWing's structural adapter
// `simwing::fsi::Structure` (src/fsi/structure.h:273-309) over the C-ABI in
// simwing_b200.h.
//
// A caller of the reference adapter includes this header in place of
// src/fsi/structure.h and links libsimwing_b200.so instead of the
// simwing_structure/softwing_core libraries.  Type names, field names,
// defaults, member functions and the exceptions they throw are those of the
// reference, so such callers compile unchanged:
//
//   std::invalid_argument  bad definition, settings, force or checkpoint
//                          (structure.cpp:102-455, 782-805, 961-1027)
//   std::out_of_range      force on a node that does not exist (:785)
//   softwing::SuspensionError   suspension certification failed
//   softwing::ContactStepError  contact could not be resolved
//
// A failed step restores the committed state before it throws, like
// Structure::step (structure.cpp:807-831).  The device solver adds three
// failures the CPU solver does not have; they throw
// simwing_b200::DeviceStepError (a std::runtime_error) with the status.
//
// Differences a caller can observe: the state is FP32 on the device (the
// boundary stays FP64); `workerThreads` is ignored; fabric self-contact,
// load-path cable sweeps or membranes on a mesh too large for one cluster
// are rejected with simwing_b200::Unsupported (a std::logic_error) at
// construction or step.
#pragma once

#include "simwing_b200.h"

#include <array>
#include <compare>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace softwing {

// softwing::SuspensionPhase (src/softwing/include/softwing/suspension.h:27-38),
// in the same order as SWB_PHASE_*.
enum class SuspensionPhase {
    Parse,
    Validation,
    AttachmentResolution,
    GraphConstruction,
    Control,
    Prediction,
    LineSolve,
    GroundSolve,
    Certification,
    Diagnostics,
};

// softwing::SuspensionError (src/softwing/include/softwing/suspension.h:40-53).
class SuspensionError : public std::runtime_error {
public:
    SuspensionError(SuspensionPhase phase, std::string entity, const std::string& message)
        : std::runtime_error(message), phase_(phase), entity_(std::move(entity)) {}

    [[nodiscard]] SuspensionPhase phase() const { return phase_; }
    [[nodiscard]] const std::string& entity() const { return entity_; }

private:
    SuspensionPhase phase_;
    std::string entity_;
};

// softwing::ContactFeatureKind and ContactFeatureKey
// (src/softwing/include/softwing/contact.h:27-31, 95-101).
enum class ContactFeatureKind {
    VertexTriangle,
    EdgeEdge,
    SegmentTriangle,
};

struct ContactFeatureKey {
    std::size_t pair = 0;
    ContactFeatureKind kind = ContactFeatureKind::VertexTriangle;
    std::array<std::size_t, 3> firstPrimitive{};
    std::array<std::size_t, 3> secondPrimitive{};

    auto operator<=>(const ContactFeatureKey&) const = default;
};

// softwing::ContactStepError (src/softwing/include/softwing/contact.h:262-270).
class ContactStepError : public std::runtime_error {
public:
    ContactStepError(const ContactFeatureKey& key, const std::string& message)
        : std::runtime_error(message), key_(key) {}

    [[nodiscard]] const ContactFeatureKey& key() const { return key_; }

private:
    ContactFeatureKey key_;
};

}  // namespace softwing

namespace simwing_b200 {

class DeviceStepError : public std::runtime_error {
public:
    DeviceStepError(swb_status status, const std::string& what) : std::runtime_error(what), status_(status) {}
    [[nodiscard]] swb_status status() const noexcept { return status_; }

private:
    swb_status status_;
};

class Unsupported : public std::logic_error {
public:
    using std::logic_error::logic_error;
};

// Throws the exception the reference adapter throws for `status`, with the
// suspension phase and entity or the contact feature key of the failure.
inline void check(swb_status status) {
    if (status == SWB_OK) return;
    const std::string what = swb_last_error() ? swb_last_error() : "simwing_b200 error";
    swb_error_detail detail{};
    if (swb_last_error_detail(&detail) != SWB_OK || detail.status != static_cast<uint32_t>(status))
        detail = swb_error_detail{};
    switch (status) {
    case SWB_INVALID_ARGUMENT: throw std::invalid_argument(what);
    case SWB_OUT_OF_RANGE: throw std::out_of_range(what);
    case SWB_SUSPENSION_ERROR: {
        const char* entity = detail.status ? detail.suspension_entity : "";
        throw softwing::SuspensionError(static_cast<softwing::SuspensionPhase>(detail.suspension_phase),
                                        std::string(entity, strnlen(entity, sizeof detail.suspension_entity)), what);
    }
    case SWB_CONTACT_ERROR: {
        softwing::ContactFeatureKey key{};
        if (detail.has_contact_key) {
            key.pair = static_cast<std::size_t>(detail.contact_key.pair);
            key.kind = static_cast<softwing::ContactFeatureKind>(detail.contact_key.kind);
            for (int i = 0; i < 3; ++i) {
                key.firstPrimitive[i] = static_cast<std::size_t>(detail.contact_key.first[i]);
                key.secondPrimitive[i] = static_cast<std::size_t>(detail.contact_key.second[i]);
            }
        }
        throw softwing::ContactStepError(key, what);
    }
    case SWB_UNSUPPORTED: throw Unsupported(what);
    case SWB_OUT_OF_MEMORY: throw std::bad_alloc();
    default: throw DeviceStepError(status, what);
    }
}

}  // namespace simwing_b200

namespace simwing::fsi {

// ---- definition types (structure.h:16-172) --------------------------------

struct StructureVector2 {
    double x = 0.0;
    double y = 0.0;
};

struct StructureVector3 {
    double x = 0.0;
    double y = 0.0;
    double z = 0.0;

    auto operator<=>(const StructureVector3&) const = default;
};

struct StructureNodeDefinition {
    StructureVector3 positionMeters;
    double massKg = 0.0;
    bool fixed = false;
};

struct StructureTriangleDefinition {
    std::array<std::size_t, 3> nodes{};
};

enum class StructureConstraintKind : std::uint8_t {
    Distance = SWB_CONSTRAINT_DISTANCE,
    Cable = SWB_CONSTRAINT_CABLE,
    SuspensionTie = SWB_CONSTRAINT_SUSPENSION_TIE,
    SeamStitch = SWB_CONSTRAINT_SEAM_STITCH,
};

struct StructureConstraintDefinition {
    StructureConstraintKind kind = StructureConstraintKind::Distance;
    std::size_t firstNode = 0;
    std::size_t secondNode = 0;
    double restLengthMeters = 0.0;
    double complianceMetersPerNewton = 0.0;
};

enum class StructureMaterialRole : std::uint8_t {
    Bulk = SWB_ROLE_BULK,
    Seam = SWB_ROLE_SEAM,
    Reinforcement = SWB_ROLE_REINFORCEMENT,
};

struct StructureMembraneMaterial {
    double warpStiffnessNewtonsPerMeter = 0.0;
    double weftStiffnessNewtonsPerMeter = 0.0;
    double couplingStiffnessNewtonsPerMeter = 0.0;
    double shearStiffnessNewtonsPerMeter = 0.0;
    double warpPreTensionNewtonsPerMeter = 0.0;
    double weftPreTensionNewtonsPerMeter = 0.0;
    double dampingSeconds = 0.0;
    double compressionStiffnessRatio = 1.0;
};

struct StructureMembraneDefinition {
    std::size_t triangle = 0;
    std::array<StructureVector2, 3> materialCoordinates{};
    StructureMembraneMaterial material;
    StructureMaterialRole role = StructureMaterialRole::Bulk;
};

struct StructureDihedralDefinition {
    std::array<std::size_t, 4> nodes{};
    double restAngleRadians = 0.0;
    double complianceRadiansPerNewtonMeter = 0.0;
};

struct StructureFabricContactDefinition {
    double halfThicknessMeters = 0.0;
    double normalComplianceMetersPerNewton = 0.0;
    double staticFriction = 0.0;
    double dynamicFriction = 0.0;

    auto operator<=>(const StructureFabricContactDefinition&) const = default;
};

struct StructureQuaternion {
    double w = 1.0;
    double x = 0.0;
    double y = 0.0;
    double z = 0.0;

    auto operator<=>(const StructureQuaternion&) const = default;
};

enum class StructureSuspensionEndpointKind : std::uint8_t {
    SurfaceAttachment = SWB_ENDPOINT_SURFACE_ATTACHMENT,
    Junction = SWB_ENDPOINT_JUNCTION,
    PilotHarness = SWB_ENDPOINT_PILOT_HARNESS,
};

struct StructureSuspensionEndpointDefinition {
    StructureSuspensionEndpointKind kind = StructureSuspensionEndpointKind::SurfaceAttachment;
    std::uint64_t stableId = 0;
};

struct StructureSuspensionAttachmentDefinition {
    std::uint64_t stableId = 0;
    std::size_t node = 0;
};

struct StructureSuspensionJunctionDefinition {
    std::uint64_t stableId = 0;
    std::size_t node = 0;
};

struct StructurePilotHarnessDefinition {
    std::uint64_t stableId = 0;
    StructureVector3 localPositionMeters;
};

struct StructureSuspensionSegmentDefinition {
    std::uint64_t stableId = 0;
    StructureSuspensionEndpointDefinition from;
    StructureSuspensionEndpointDefinition to;
    double restLengthMeters = 0.0;
    double axialStiffnessNewtons = 0.0;
    double axialDampingNewtonSecondsPerMeter = 0.0;
    std::uint32_t role = 0;
};

struct StructureSuspensionDefinition {
    std::uint64_t pilotStableId = 0;
    double pilotMassKg = 0.0;
    StructureVector3 pilotCenterOfMassLocalMeters;
    StructureVector3 pilotInitialCenterOfMassWorldMeters;
    StructureVector3 pilotInitialLinearVelocityMetersPerSecond;
    StructureVector3 pilotInitialAngularVelocityRadiansPerSecond;
    StructureQuaternion pilotInitialBodyToWorld;
    StructureVector3 pilotPrincipalInertiaKgSquareMeters;
    std::vector<StructureSuspensionAttachmentDefinition> attachments;
    std::vector<StructureSuspensionJunctionDefinition> junctions;
    std::vector<StructurePilotHarnessDefinition> harnessPoints;
    std::vector<StructureSuspensionSegmentDefinition> segments;
    int solverIterations = 12;
    double attachmentTolerance = 1.0e-10;
    double minimumLineLengthMeters = 1.0e-10;
    double maximumLineResidualMeters = 2.0e-4;
    double maximumControlWorkJoules = 1.0e6;
};

struct StructureDefinition {
    std::vector<StructureNodeDefinition> nodes;
    std::vector<StructureTriangleDefinition> triangles;
    std::vector<StructureConstraintDefinition> constraints;
    std::vector<StructureMembraneDefinition> membranes;
    std::vector<StructureDihedralDefinition> dihedrals;
    std::optional<StructureFabricContactDefinition> fabricSelfContact;
    std::optional<StructureSuspensionDefinition> suspension;
};

// ---- state and result types (structure.h:174-246) -------------------------

struct StructureNodeState {
    StructureVector3 positionMeters;
    StructureVector3 previousPositionMeters;
    StructureVector3 velocityMetersPerSecond;

    auto operator<=>(const StructureNodeState&) const = default;
};

struct StructureRigidPayloadState {
    StructureVector3 centerOfMassWorldMeters;
    StructureQuaternion bodyToWorld;
    StructureVector3 linearVelocityMetersPerSecond;
    StructureVector3 angularVelocityRadiansPerSecond;

    auto operator<=>(const StructureRigidPayloadState&) const = default;
};

struct StructureSuspensionSegmentState {
    std::uint64_t stableId = 0;
    double currentLengthMeters = 0.0;
    double commandedRestLengthMeters = 0.0;
    double tensionNewtons = 0.0;

    auto operator<=>(const StructureSuspensionSegmentState&) const = default;
};

struct StructureSuspensionState {
    StructureRigidPayloadState payload;
    std::vector<StructureVector3> harnessPositionsMeters;
    std::vector<StructureVector3> harnessVelocitiesMetersPerSecond;
    std::vector<StructureSuspensionSegmentState> segments;

    auto operator<=>(const StructureSuspensionState&) const = default;
};

struct StructureStepSettings {
    double timeStepSeconds = 1.0 / 120.0;
    int substeps = 2;
    int constraintIterations = 12;
    int cableConstraintSweepPairs = 0;
    StructureVector3 gravityMetersPerSecondSquared{0.0, 0.0, -9.80665};
    double velocityDampingPerSecond = 0.25;
    StructureVector3 dampingReferenceVelocityMetersPerSecond;
    unsigned workerThreads = 0;  // accepted, ignored: the device sweep is always parallel
};

struct StructureDiagnostics {
    std::size_t nodeCount = 0;
    std::size_t dynamicNodeCount = 0;
    std::size_t triangleCount = 0;
    std::size_t constraintCount = 0;
    std::size_t membraneCount = 0;
    std::size_t dihedralCount = 0;
    std::size_t contactPairCount = 0;
    std::size_t activeContactCount = 0;
    std::size_t suspensionSegmentCount = 0;
    double totalDynamicMassKg = 0.0;
    StructureVector3 centerOfMassMeters;
    StructureVector3 linearMomentumKgMetersPerSecond;
    double kineticEnergyJoules = 0.0;
    double maximumDistanceErrorMeters = 0.0;
    double maximumCableExtensionMeters = 0.0;
    double maximumAbsoluteMembraneStrain = 0.0;
    double maximumMembraneResidual = 0.0;
    double maximumContactPenetrationMeters = 0.0;
    double maximumSuspensionResidualMeters = 0.0;
    StructureVector3 pendingExternalForceNewtons;
    StructureVector3 lastAppliedExternalForceNewtons;
    bool finite = true;

    auto operator<=>(const StructureDiagnostics&) const = default;
};

inline constexpr std::uint32_t structureCheckpointVersion = 2;

// StructureCheckpoint (structure.h:248-271).  The public fields are filled
// from the device image; restore() checks them against it, as the reference
// checks them against its private detail (structure.cpp:978-1003).
struct StructureCheckpoint {
    std::uint32_t version = structureCheckpointVersion;
    std::uint64_t definitionFingerprint = 0;
    std::uint64_t acceptedStepCount = 0;
    double simulationTimeSeconds = 0.0;
    std::vector<StructureNodeState> nodes;
    std::vector<StructureVector3> pendingExternalForcesNewtons;
    StructureVector3 lastAppliedExternalForceNewtons;

private:
    friend class Structure;
    struct Detail {
        std::vector<std::uint8_t> image;
        std::vector<StructureNodeState> publicNodes;
    };
    std::shared_ptr<const Detail> detail;
};

namespace detail {

inline swb_vec3 to_swb(const StructureVector3& v) { return {v.x, v.y, v.z}; }
inline StructureVector3 from_swb(const swb_vec3& v) { return {v.x, v.y, v.z}; }

// Flat C-ABI image of a StructureDefinition; the arrays live as long as it.
struct AbiDefinition {
    std::vector<swb_node_def> nodes;
    std::vector<swb_triangle_def> triangles;
    std::vector<swb_constraint_def> constraints;
    std::vector<swb_membrane_def> membranes;
    std::vector<swb_dihedral_def> dihedrals;
    swb_fabric_contact_def contact{};
    std::vector<swb_suspension_attachment> attachments;
    std::vector<swb_suspension_junction> junctions;
    std::vector<swb_pilot_harness> harness;
    std::vector<swb_suspension_segment> segments;
    swb_suspension_def suspension{};
    swb_structure_definition view{};

    explicit AbiDefinition(const StructureDefinition& d) {
        for (const auto& n : d.nodes) nodes.push_back({to_swb(n.positionMeters), n.massKg, n.fixed ? 1u : 0u, 0u});
        for (const auto& t : d.triangles) triangles.push_back({{t.nodes[0], t.nodes[1], t.nodes[2]}, 0.0});
        for (const auto& c : d.constraints)
            constraints.push_back({static_cast<uint32_t>(c.kind), 0u, c.firstNode, c.secondNode, c.restLengthMeters,
                                   c.complianceMetersPerNewton});
        for (const auto& m : d.membranes) {
            swb_membrane_def e{};
            e.triangle = m.triangle;
            for (int k = 0; k < 3; ++k) {
                e.chart[k][0] = m.materialCoordinates[k].x;
                e.chart[k][1] = m.materialCoordinates[k].y;
            }
            const auto& q = m.material;
            e.material = {q.warpStiffnessNewtonsPerMeter, q.weftStiffnessNewtonsPerMeter,
                          q.couplingStiffnessNewtonsPerMeter, q.shearStiffnessNewtonsPerMeter,
                          q.warpPreTensionNewtonsPerMeter, q.weftPreTensionNewtonsPerMeter, q.dampingSeconds,
                          q.compressionStiffnessRatio};
            e.role = static_cast<uint32_t>(m.role);
            membranes.push_back(e);
        }
        for (const auto& h : d.dihedrals)
            dihedrals.push_back({{h.nodes[0], h.nodes[1], h.nodes[2], h.nodes[3]}, h.restAngleRadians,
                                 h.complianceRadiansPerNewtonMeter});
        view.node_count = nodes.size();
        view.nodes = nodes.data();
        view.triangle_count = triangles.size();
        view.triangles = triangles.data();
        view.constraint_count = constraints.size();
        view.constraints = constraints.data();
        view.membrane_count = membranes.size();
        view.membranes = membranes.data();
        view.dihedral_count = dihedrals.size();
        view.dihedrals = dihedrals.data();
        if (d.fabricSelfContact) {
            const auto& c = *d.fabricSelfContact;
            contact = {c.halfThicknessMeters, c.normalComplianceMetersPerNewton, c.staticFriction, c.dynamicFriction};
            view.fabric_self_contact = &contact;
        }
        if (d.suspension) {
            const auto& s = *d.suspension;
            for (const auto& a : s.attachments) attachments.push_back({a.stableId, a.node});
            for (const auto& j : s.junctions) junctions.push_back({j.stableId, j.node});
            for (const auto& h : s.harnessPoints) harness.push_back({h.stableId, to_swb(h.localPositionMeters)});
            for (const auto& g : s.segments) {
                swb_suspension_segment e{};
                e.stable_id = g.stableId;
                e.from = {static_cast<uint32_t>(g.from.kind), 0u, g.from.stableId};
                e.to = {static_cast<uint32_t>(g.to.kind), 0u, g.to.stableId};
                e.rest_length = g.restLengthMeters;
                e.axial_stiffness = g.axialStiffnessNewtons;
                e.axial_damping = g.axialDampingNewtonSecondsPerMeter;
                e.role = g.role;
                segments.push_back(e);
            }
            suspension.pilot_stable_id = s.pilotStableId;
            suspension.pilot_mass = s.pilotMassKg;
            suspension.pilot_com_local = to_swb(s.pilotCenterOfMassLocalMeters);
            suspension.pilot_initial_com_world = to_swb(s.pilotInitialCenterOfMassWorldMeters);
            suspension.pilot_initial_linear_velocity = to_swb(s.pilotInitialLinearVelocityMetersPerSecond);
            suspension.pilot_initial_angular_velocity = to_swb(s.pilotInitialAngularVelocityRadiansPerSecond);
            const auto& q = s.pilotInitialBodyToWorld;
            suspension.pilot_initial_body_to_world = {q.w, q.x, q.y, q.z};
            suspension.pilot_principal_inertia = to_swb(s.pilotPrincipalInertiaKgSquareMeters);
            suspension.attachment_count = attachments.size();
            suspension.attachments = attachments.data();
            suspension.junction_count = junctions.size();
            suspension.junctions = junctions.data();
            suspension.harness_count = harness.size();
            suspension.harness_points = harness.data();
            suspension.segment_count = segments.size();
            suspension.segments = segments.data();
            suspension.solver_iterations = s.solverIterations;
            suspension.attachment_tolerance = s.attachmentTolerance;
            suspension.minimum_line_length = s.minimumLineLengthMeters;
            suspension.maximum_line_residual = s.maximumLineResidualMeters;
            suspension.maximum_control_work = s.maximumControlWorkJoules;
            view.suspension = &suspension;
        }
    }
};

inline StructureDiagnostics from_swb(const swb_diagnostics& d) {
    StructureDiagnostics r;
    r.nodeCount = d.node_count;
    r.dynamicNodeCount = d.dynamic_node_count;
    r.triangleCount = d.triangle_count;
    r.constraintCount = d.constraint_count;
    r.membraneCount = d.membrane_count;
    r.dihedralCount = d.dihedral_count;
    r.contactPairCount = d.contact_pair_count;
    r.activeContactCount = d.active_contact_count;
    r.suspensionSegmentCount = d.suspension_segment_count;
    r.totalDynamicMassKg = d.total_dynamic_mass;
    r.centerOfMassMeters = from_swb(d.center_of_mass);
    r.linearMomentumKgMetersPerSecond = from_swb(d.linear_momentum);
    r.kineticEnergyJoules = d.kinetic_energy;
    r.maximumDistanceErrorMeters = d.maximum_distance_error;
    r.maximumCableExtensionMeters = d.maximum_cable_extension;
    r.maximumAbsoluteMembraneStrain = d.maximum_absolute_membrane_strain;
    r.maximumMembraneResidual = d.maximum_membrane_residual;
    r.maximumContactPenetrationMeters = d.maximum_contact_penetration;
    r.maximumSuspensionResidualMeters = d.maximum_suspension_residual;
    r.pendingExternalForceNewtons = from_swb(d.pending_external_force);
    r.lastAppliedExternalForceNewtons = from_swb(d.last_applied_external_force);
    r.finite = d.finite != 0;
    return r;
}

inline swb_step_settings to_swb(const StructureStepSettings& s) {
    swb_step_settings r{};
    r.time_step = s.timeStepSeconds;
    r.substeps = s.substeps;
    r.constraint_iterations = s.constraintIterations;
    r.cable_sweep_pairs = s.cableConstraintSweepPairs;
    r.worker_threads = s.workerThreads;
    r.gravity = to_swb(s.gravityMetersPerSecondSquared);
    r.velocity_damping = s.velocityDampingPerSecond;
    r.damping_reference_velocity = to_swb(s.dampingReferenceVelocityMetersPerSecond);
    return r;
}

// Reads the public fields of a checkpoint image (layout written by
// swb_structure_checkpoint: magic, version, suspension flag, contact flag,
// a reserved word, fingerprint, accepted steps, time, last dt, origin, node
// count, per node position / previous / velocity, pending forces, last
// applied force, ...).
class ImageReader {
public:
    explicit ImageReader(const std::vector<std::uint8_t>& b) : b_(b) {}
    template <class T> T get() {
        if (at_ + sizeof(T) > b_.size()) throw std::invalid_argument("Invalid structure checkpoint");
        T v;
        std::memcpy(&v, b_.data() + at_, sizeof(T));
        at_ += sizeof(T);
        return v;
    }
    StructureVector3 vec() {
        StructureVector3 v;
        v.x = get<double>();
        v.y = get<double>();
        v.z = get<double>();
        return v;
    }
    void skip(std::size_t n) { at_ += n; }

private:
    const std::vector<std::uint8_t>& b_;
    std::size_t at_ = 0;
};

}  // namespace detail

// simwing::fsi::Structure (structure.h:273-309) on the device solver.
class Structure {
public:
    explicit Structure(StructureDefinition definition, const swb_solver_options* options = nullptr)
        : definition_(std::move(definition)) {
        detail::AbiDefinition abi(definition_);
        swb_structure* h = nullptr;
        simwing_b200::check(swb_structure_create(&abi.view, options, &h));
        handle_.reset(h);
    }

    Structure(Structure&&) noexcept = default;
    Structure& operator=(Structure&&) noexcept = default;
    Structure(const Structure&) = delete;
    Structure& operator=(const Structure&) = delete;

    [[nodiscard]] const StructureDefinition& definition() const noexcept { return definition_; }
    [[nodiscard]] std::uint64_t definitionFingerprint() const noexcept { return swb_structure_fingerprint(h()); }
    [[nodiscard]] std::uint64_t acceptedStepCount() const noexcept { return swb_structure_accepted_steps(h()); }
    [[nodiscard]] double simulationTimeSeconds() const noexcept { return swb_structure_simulation_time(h()); }

    [[nodiscard]] std::vector<StructureNodeState> nodeStates() const {
        std::vector<swb_node_state> raw(definition_.nodes.size());
        simwing_b200::check(swb_structure_read_nodes(h(), raw.data(), raw.size()));
        std::vector<StructureNodeState> out(raw.size());
        for (std::size_t i = 0; i < raw.size(); ++i)
            out[i] = {detail::from_swb(raw[i].position), detail::from_swb(raw[i].previous_position),
                      detail::from_swb(raw[i].velocity)};
        return out;
    }

    // Structure::suspensionState (structure.cpp:736-776): payload and
    // segment states; harness positions and velocities follow from the
    // payload pose and twist.
    [[nodiscard]] std::optional<StructureSuspensionState> suspensionState() const {
        if (!definition_.suspension) return std::nullopt;
        const auto& s = *definition_.suspension;
        swb_payload_state p{};
        std::vector<swb_segment_state> seg(s.segments.size());
        simwing_b200::check(swb_structure_read_suspension(h(), &p, seg.data(), seg.size(), nullptr));
        StructureSuspensionState r;
        r.payload.centerOfMassWorldMeters = detail::from_swb(p.center_of_mass);
        r.payload.bodyToWorld = {p.body_to_world.w, p.body_to_world.x, p.body_to_world.y, p.body_to_world.z};
        r.payload.linearVelocityMetersPerSecond = detail::from_swb(p.linear_velocity);
        r.payload.angularVelocityRadiansPerSecond = detail::from_swb(p.angular_velocity);
        for (const auto& hp : s.harnessPoints) {
            const StructureVector3 arm = rotate(r.payload.bodyToWorld, sub(hp.localPositionMeters,
                                                                             s.pilotCenterOfMassLocalMeters));
            r.harnessPositionsMeters.push_back(add(r.payload.centerOfMassWorldMeters, arm));
            r.harnessVelocitiesMetersPerSecond.push_back(
                add(r.payload.linearVelocityMetersPerSecond, cross(r.payload.angularVelocityRadiansPerSecond, arm)));
        }
        for (const auto& g : seg)
            r.segments.push_back({g.stable_id, g.current_length, g.commanded_rest_length, g.tension});
        return r;
    }

    void clearExternalForces() noexcept { swb_structure_clear_external_forces(h()); }
    void addExternalForce(std::size_t node, const StructureVector3& forceNewtons) {
        const swb_vec3 f = detail::to_swb(forceNewtons);
        simwing_b200::check(swb_structure_add_external_force(h(), node, &f));
    }
    void setExternalForces(std::span<const StructureVector3> forcesNewtons) {
        std::vector<swb_vec3> f(forcesNewtons.size());
        for (std::size_t i = 0; i < f.size(); ++i) f[i] = detail::to_swb(forcesNewtons[i]);
        simwing_b200::check(swb_structure_set_external_forces(h(), f.data(), f.size()));
    }

    // A failed step restores the committed state before it throws; pending
    // loads are consumed only by an accepted step.
    [[nodiscard]] StructureDiagnostics step(const StructureStepSettings& settings) {
        const swb_step_settings s = detail::to_swb(settings);
        swb_diagnostics d{};
        simwing_b200::check(swb_structure_step(h(), &s, &d));
        return detail::from_swb(d);
    }
    [[nodiscard]] StructureDiagnostics diagnostics() const {
        swb_diagnostics d{};
        simwing_b200::check(swb_structure_diagnostics(h(), &d));
        return detail::from_swb(d);
    }

    [[nodiscard]] StructureCheckpoint checkpoint() const {
        std::uint64_t bytes = 0;
        simwing_b200::check(swb_structure_checkpoint_size(h(), &bytes));
        auto det = std::make_shared<StructureCheckpoint::Detail>();
        det->image.resize(bytes);
        simwing_b200::check(swb_structure_checkpoint(h(), det->image.data(), bytes));
        StructureCheckpoint c;
        detail::ImageReader r(det->image);
        r.skip(8 + 4 + 4 + 4 + 4);
        c.definitionFingerprint = r.get<std::uint64_t>();
        c.acceptedStepCount = r.get<std::uint64_t>();
        c.simulationTimeSeconds = r.get<double>();
        r.skip(8);
        const StructureVector3 origin = r.vec();
        (void)origin;
        const std::uint64_t n = r.get<std::uint64_t>();
        c.nodes.resize(n);
        for (auto& node : c.nodes) {
            node.positionMeters = r.vec();
            node.previousPositionMeters = r.vec();
            node.velocityMetersPerSecond = r.vec();
        }
        c.pendingExternalForcesNewtons.resize(n);
        for (auto& f : c.pendingExternalForcesNewtons) f = r.vec();
        c.lastAppliedExternalForceNewtons = r.vec();
        // node states of the image are relative to the frame origin
        for (auto& node : c.nodes) {
            node.positionMeters = add(node.positionMeters, origin);
            node.previousPositionMeters = add(node.previousPositionMeters, origin);
        }
        det->publicNodes = c.nodes;
        c.detail = std::move(det);
        return c;
    }

    // Structure::restore (structure.cpp:978-1027): version, fingerprint and
    // public fields are checked against the private image before the device
    // state is replaced; a rejected checkpoint throws std::invalid_argument
    // and leaves the structure unchanged.
    void restore(const StructureCheckpoint& c) {
        if (c.version != structureCheckpointVersion)
            throw std::invalid_argument("Unsupported structure checkpoint version");
        if (c.definitionFingerprint != definitionFingerprint())
            throw std::invalid_argument("Structure checkpoint belongs to a different definition");
        if (!c.detail || c.nodes.size() != definition_.nodes.size() ||
            c.pendingExternalForcesNewtons.size() != definition_.nodes.size() || c.detail->publicNodes != c.nodes)
            throw std::invalid_argument("Invalid structure checkpoint");
        simwing_b200::check(swb_structure_restore(h(), c.detail->image.data(), c.detail->image.size()));
    }

    // Access to the C-ABI handle for the calls the reference adapter lacks
    // (face pressure, schedule report, device timing).
    [[nodiscard]] swb_structure* handle() const noexcept { return handle_.get(); }

private:
    struct Deleter {
        void operator()(swb_structure* s) const noexcept { swb_structure_destroy(s); }
    };
    swb_structure* h() const noexcept { return handle_.get(); }

    static StructureVector3 add(const StructureVector3& a, const StructureVector3& b) {
        return {a.x + b.x, a.y + b.y, a.z + b.z};
    }
    static StructureVector3 sub(const StructureVector3& a, const StructureVector3& b) {
        return {a.x - b.x, a.y - b.y, a.z - b.z};
    }
    static StructureVector3 cross(const StructureVector3& a, const StructureVector3& b) {
        return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    }
    static StructureVector3 rotate(const StructureQuaternion& q, const StructureVector3& v) {
        const StructureVector3 u{q.x, q.y, q.z};
        const StructureVector3 t = cross(u, v);
        const StructureVector3 t2{2.0 * t.x, 2.0 * t.y, 2.0 * t.z};
        const StructureVector3 c = cross(u, t2);
        return {v.x + q.w * t2.x + c.x, v.y + q.w * t2.y + c.y, v.z + q.w * t2.z + c.z};
    }

    StructureDefinition definition_;
    std::unique_ptr<swb_structure, Deleter> handle_;
};

}  // namespace simwing::fsi
