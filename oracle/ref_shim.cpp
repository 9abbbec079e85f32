// ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked into the product library.
//
// C shim over the reference's own, unmodified structural adapter
// `simwing::fsi::Structure` (src/fsi/structure.h:273-309) and XPBD core
// (src/softwing).  oracle/Makefile compiles the reference sources where they
// lie and links them with this file into oracle/_ref/libswref.so, which the
// tests and bench.py's CPU-baseline leg load through ctypes.
//
// The shim takes the same `swb_structure_definition` as the device solver.
// Per-face pressure: the adapter's StructureDefinition carries no face
// pressure (structure.h:38-40), so the shim computes the softwing nodal
// pressure load Δp·½(b−a)×(c−a)/3 (soft_body.cpp:1497-1508) from the state at
// step start and adds it to the pending external forces.  With one substep
// this is the force SoftBody::integrateSubstepTrial accumulates
// (soft_body.cpp:1185), up to FP64 summation order.
#include "simwing_b200.h"

#include "structure.h"
#include "scene.h"
#include "scene_structure.h"
#include <softwing/parallel.h>
#include <softwing/soft_body.h>
#include <softwing/suspension.h>
#include <softwing/cell_volume.h>
#include <softwing/pneumatics.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

// The reference's own test hook (soft_body.h:22, 504): runs one contact
// iteration of a body and reads the candidate keys its broadphase streamed.
namespace softwing {
struct ContactAuditTestAccess {
    static void begin(SoftBody& body) { body.beginContactSubstep(); }
    static void iterate(SoftBody& body, double dt, const StepSettings& settings) {
        body.solveContactIteration(dt, settings);
    }
    static const std::vector<ContactFeatureKey>& candidates(const SoftBody& body) {
        return body.contactAudit_.iterationCandidateKeys;
    }
};
}  // namespace softwing

namespace {

thread_local std::string g_error;
// The reference's exception details of the last failure (SuspensionError
// phase/entity, ContactStepError key), for comparison with the device's.
thread_local swb_error_detail g_detail{};

using namespace simwing::fsi;

StructureDefinition convert(const swb_structure_definition& d) {
    StructureDefinition out;
    out.nodes.reserve(d.node_count);
    for (uint64_t i = 0; i < d.node_count; ++i) {
        const swb_node_def& n = d.nodes[i];
        out.nodes.push_back({{n.position.x, n.position.y, n.position.z},
                             n.mass,
                             n.fixed != 0});
    }
    for (uint64_t i = 0; i < d.triangle_count; ++i) {
        const swb_triangle_def& t = d.triangles[i];
        out.triangles.push_back({{t.nodes[0], t.nodes[1], t.nodes[2]}});
    }
    for (uint64_t i = 0; i < d.constraint_count; ++i) {
        const swb_constraint_def& c = d.constraints[i];
        out.constraints.push_back(
            {static_cast<StructureConstraintKind>(c.kind), c.first_node,
             c.second_node, c.rest_length, c.compliance});
    }
    for (uint64_t i = 0; i < d.membrane_count; ++i) {
        const swb_membrane_def& m = d.membranes[i];
        StructureMembraneDefinition md;
        md.triangle = m.triangle;
        for (int k = 0; k < 3; ++k)
            md.materialCoordinates[k] = {m.chart[k][0], m.chart[k][1]};
        md.material.warpStiffnessNewtonsPerMeter = m.material.warp_stiffness;
        md.material.weftStiffnessNewtonsPerMeter = m.material.weft_stiffness;
        md.material.couplingStiffnessNewtonsPerMeter =
            m.material.coupling_stiffness;
        md.material.shearStiffnessNewtonsPerMeter = m.material.shear_stiffness;
        md.material.warpPreTensionNewtonsPerMeter = m.material.warp_pretension;
        md.material.weftPreTensionNewtonsPerMeter = m.material.weft_pretension;
        md.material.dampingSeconds = m.material.damping_seconds;
        md.material.compressionStiffnessRatio =
            m.material.compression_stiffness_ratio;
        md.role = static_cast<StructureMaterialRole>(m.role);
        out.membranes.push_back(md);
    }
    for (uint64_t i = 0; i < d.dihedral_count; ++i) {
        const swb_dihedral_def& h = d.dihedrals[i];
        out.dihedrals.push_back(
            {{h.nodes[0], h.nodes[1], h.nodes[2], h.nodes[3]},
             h.rest_angle,
             h.compliance});
    }
    if (d.fabric_self_contact) {
        const swb_fabric_contact_def& c = *d.fabric_self_contact;
        out.fabricSelfContact = StructureFabricContactDefinition{
            c.half_thickness, c.normal_compliance, c.static_friction,
            c.dynamic_friction};
    }
    if (d.suspension) {
        const swb_suspension_def& s = *d.suspension;
        StructureSuspensionDefinition sd;
        sd.pilotStableId = s.pilot_stable_id;
        sd.pilotMassKg = s.pilot_mass;
        sd.pilotCenterOfMassLocalMeters = {s.pilot_com_local.x,
                                           s.pilot_com_local.y,
                                           s.pilot_com_local.z};
        sd.pilotInitialCenterOfMassWorldMeters = {
            s.pilot_initial_com_world.x, s.pilot_initial_com_world.y,
            s.pilot_initial_com_world.z};
        sd.pilotInitialLinearVelocityMetersPerSecond = {
            s.pilot_initial_linear_velocity.x,
            s.pilot_initial_linear_velocity.y,
            s.pilot_initial_linear_velocity.z};
        sd.pilotInitialAngularVelocityRadiansPerSecond = {
            s.pilot_initial_angular_velocity.x,
            s.pilot_initial_angular_velocity.y,
            s.pilot_initial_angular_velocity.z};
        sd.pilotInitialBodyToWorld = {
            s.pilot_initial_body_to_world.w, s.pilot_initial_body_to_world.x,
            s.pilot_initial_body_to_world.y, s.pilot_initial_body_to_world.z};
        sd.pilotPrincipalInertiaKgSquareMeters = {
            s.pilot_principal_inertia.x, s.pilot_principal_inertia.y,
            s.pilot_principal_inertia.z};
        for (uint64_t i = 0; i < s.attachment_count; ++i)
            sd.attachments.push_back(
                {s.attachments[i].stable_id, s.attachments[i].node});
        for (uint64_t i = 0; i < s.junction_count; ++i)
            sd.junctions.push_back(
                {s.junctions[i].stable_id, s.junctions[i].node});
        for (uint64_t i = 0; i < s.harness_count; ++i) {
            const swb_pilot_harness& h = s.harness_points[i];
            sd.harnessPoints.push_back(
                {h.stable_id,
                 {h.local_position.x, h.local_position.y,
                  h.local_position.z}});
        }
        for (uint64_t i = 0; i < s.segment_count; ++i) {
            const swb_suspension_segment& g = s.segments[i];
            StructureSuspensionSegmentDefinition gd;
            gd.stableId = g.stable_id;
            gd.from = {static_cast<StructureSuspensionEndpointKind>(
                           g.from.kind),
                       g.from.stable_id};
            gd.to = {static_cast<StructureSuspensionEndpointKind>(g.to.kind),
                     g.to.stable_id};
            gd.restLengthMeters = g.rest_length;
            gd.axialStiffnessNewtons = g.axial_stiffness;
            gd.axialDampingNewtonSecondsPerMeter = g.axial_damping;
            gd.role = g.role;
            sd.segments.push_back(gd);
        }
        sd.solverIterations = s.solver_iterations;
        sd.attachmentTolerance = s.attachment_tolerance;
        sd.minimumLineLengthMeters = s.minimum_line_length;
        sd.maximumLineResidualMeters = s.maximum_line_residual;
        sd.maximumControlWorkJoules = s.maximum_control_work;
        out.suspension = std::move(sd);
    }
    return out;
}

struct RefHandle {
    std::unique_ptr<Structure> structure;
    std::vector<std::array<uint64_t, 3>> triangles;
    std::vector<double> pressure;
    bool anyPressure = false;
    double lastStepSeconds = 0.0;
};

swb_status fail(swb_status status, const std::exception& error) {
    g_error = error.what();
    g_detail = swb_error_detail{};
    return status;
}

swb_status translate() {
    try {
        throw;
    } catch (const softwing::SuspensionError& e) {
        const swb_status st = fail(SWB_SUSPENSION_ERROR, e);
        g_detail.status = st;
        g_detail.suspension_phase = static_cast<uint32_t>(e.phase());
        std::snprintf(g_detail.suspension_entity, sizeof g_detail.suspension_entity, "%s", e.entity().c_str());
        return st;
    } catch (const softwing::ContactStepError& e) {
        const swb_status st = fail(SWB_CONTACT_ERROR, e);
        const softwing::ContactFeatureKey& k = e.key();
        g_detail.status = st;
        g_detail.has_contact_key = 1;
        g_detail.contact_key.pair = k.pair;
        g_detail.contact_key.kind = static_cast<uint32_t>(k.kind);
        for (int i = 0; i < 3; ++i) {
            g_detail.contact_key.first[i] = k.firstPrimitive[i];
            g_detail.contact_key.second[i] = k.secondPrimitive[i];
        }
        return st;
    } catch (const std::out_of_range& e) {
        return fail(SWB_OUT_OF_RANGE, e);
    } catch (const std::invalid_argument& e) {
        return fail(SWB_INVALID_ARGUMENT, e);
    } catch (const std::exception& e) {
        return fail(SWB_INVALID_ARGUMENT, e);
    } catch (...) {
        g_error = "unknown exception";
        return SWB_INVALID_ARGUMENT;
    }
}

void toDiagnostics(const StructureDiagnostics& d, swb_diagnostics* o) {
    std::memset(o, 0, sizeof(*o));
    o->node_count = d.nodeCount;
    o->dynamic_node_count = d.dynamicNodeCount;
    o->triangle_count = d.triangleCount;
    o->constraint_count = d.constraintCount;
    o->membrane_count = d.membraneCount;
    o->dihedral_count = d.dihedralCount;
    o->contact_pair_count = d.contactPairCount;
    o->active_contact_count = d.activeContactCount;
    o->suspension_segment_count = d.suspensionSegmentCount;
    o->total_dynamic_mass = d.totalDynamicMassKg;
    o->center_of_mass = {d.centerOfMassMeters.x, d.centerOfMassMeters.y,
                         d.centerOfMassMeters.z};
    o->linear_momentum = {d.linearMomentumKgMetersPerSecond.x,
                          d.linearMomentumKgMetersPerSecond.y,
                          d.linearMomentumKgMetersPerSecond.z};
    o->kinetic_energy = d.kineticEnergyJoules;
    o->maximum_distance_error = d.maximumDistanceErrorMeters;
    o->maximum_cable_extension = d.maximumCableExtensionMeters;
    o->maximum_absolute_membrane_strain = d.maximumAbsoluteMembraneStrain;
    o->maximum_membrane_residual = d.maximumMembraneResidual;
    o->maximum_contact_penetration = d.maximumContactPenetrationMeters;
    o->maximum_suspension_residual = d.maximumSuspensionResidualMeters;
    o->pending_external_force = {d.pendingExternalForceNewtons.x,
                                 d.pendingExternalForceNewtons.y,
                                 d.pendingExternalForceNewtons.z};
    o->last_applied_external_force = {d.lastAppliedExternalForceNewtons.x,
                                      d.lastAppliedExternalForceNewtons.y,
                                      d.lastAppliedExternalForceNewtons.z};
    o->finite = d.finite ? 1u : 0u;
}

StructureStepSettings convert(const swb_step_settings& s) {
    StructureStepSettings out;
    out.timeStepSeconds = s.time_step;
    out.substeps = s.substeps;
    out.constraintIterations = s.constraint_iterations;
    out.cableConstraintSweepPairs = s.cable_sweep_pairs;
    out.gravityMetersPerSecondSquared = {s.gravity.x, s.gravity.y,
                                         s.gravity.z};
    out.velocityDampingPerSecond = s.velocity_damping;
    out.dampingReferenceVelocityMetersPerSecond = {
        s.damping_reference_velocity.x, s.damping_reference_velocity.y,
        s.damping_reference_velocity.z};
    out.workerThreads = s.worker_threads;
    return out;
}

}  // namespace

// A reference StructureDefinition held as the C-ABI's plain arrays.
struct RefAssembly {
    std::vector<swb_node_def> nodes;
    std::vector<swb_triangle_def> triangles;
    std::vector<swb_constraint_def> constraints;
    std::vector<swb_membrane_def> membranes;
    std::vector<swb_dihedral_def> dihedrals;
    swb_fabric_contact_def contact{};
    swb_suspension_def suspension{};
    std::vector<swb_suspension_attachment> attachments;
    std::vector<swb_suspension_junction> junctions;
    std::vector<swb_pilot_harness> harness;
    std::vector<swb_suspension_segment> segments;
    swb_structure_definition view{};
};

void export_definition(const StructureDefinition& d, RefAssembly& a) {
    for (const auto& n : d.nodes)
        a.nodes.push_back({{n.positionMeters.x, n.positionMeters.y, n.positionMeters.z}, n.massKg,
                           n.fixed ? 1u : 0u, 0u});
    for (const auto& t : d.triangles) {
        swb_triangle_def x{};
        for (int k = 0; k < 3; ++k) x.nodes[k] = t.nodes[k];
        a.triangles.push_back(x);
    }
    for (const auto& c : d.constraints)
        a.constraints.push_back({static_cast<uint32_t>(c.kind), 0u, c.firstNode, c.secondNode, c.restLengthMeters,
                                 c.complianceMetersPerNewton});
    for (const auto& m : d.membranes) {
        swb_membrane_def x{};
        x.triangle = m.triangle;
        for (int k = 0; k < 3; ++k) {
            x.chart[k][0] = m.materialCoordinates[k].x;
            x.chart[k][1] = m.materialCoordinates[k].y;
        }
        x.material.warp_stiffness = m.material.warpStiffnessNewtonsPerMeter;
        x.material.weft_stiffness = m.material.weftStiffnessNewtonsPerMeter;
        x.material.coupling_stiffness = m.material.couplingStiffnessNewtonsPerMeter;
        x.material.shear_stiffness = m.material.shearStiffnessNewtonsPerMeter;
        x.material.warp_pretension = m.material.warpPreTensionNewtonsPerMeter;
        x.material.weft_pretension = m.material.weftPreTensionNewtonsPerMeter;
        x.material.damping_seconds = m.material.dampingSeconds;
        x.material.compression_stiffness_ratio = m.material.compressionStiffnessRatio;
        x.role = static_cast<uint32_t>(m.role);
        a.membranes.push_back(x);
    }
    for (const auto& h : d.dihedrals) {
        swb_dihedral_def x{};
        for (int k = 0; k < 4; ++k) x.nodes[k] = h.nodes[k];
        x.rest_angle = h.restAngleRadians;
        x.compliance = h.complianceRadiansPerNewtonMeter;
        a.dihedrals.push_back(x);
    }
    a.view = swb_structure_definition{};
    if (d.fabricSelfContact) {
        const auto& c = *d.fabricSelfContact;
        a.contact = {c.halfThicknessMeters, c.normalComplianceMetersPerNewton, c.staticFriction, c.dynamicFriction};
        a.view.fabric_self_contact = &a.contact;
    }
    if (d.suspension) {
        const auto& sd = *d.suspension;
        swb_suspension_def& x = a.suspension;
        x.pilot_stable_id = sd.pilotStableId;
        x.pilot_mass = sd.pilotMassKg;
        x.pilot_com_local = {sd.pilotCenterOfMassLocalMeters.x, sd.pilotCenterOfMassLocalMeters.y,
                             sd.pilotCenterOfMassLocalMeters.z};
        x.pilot_initial_com_world = {sd.pilotInitialCenterOfMassWorldMeters.x, sd.pilotInitialCenterOfMassWorldMeters.y,
                                     sd.pilotInitialCenterOfMassWorldMeters.z};
        x.pilot_initial_linear_velocity = {sd.pilotInitialLinearVelocityMetersPerSecond.x,
                                           sd.pilotInitialLinearVelocityMetersPerSecond.y,
                                           sd.pilotInitialLinearVelocityMetersPerSecond.z};
        x.pilot_initial_angular_velocity = {sd.pilotInitialAngularVelocityRadiansPerSecond.x,
                                            sd.pilotInitialAngularVelocityRadiansPerSecond.y,
                                            sd.pilotInitialAngularVelocityRadiansPerSecond.z};
        x.pilot_initial_body_to_world = {sd.pilotInitialBodyToWorld.w, sd.pilotInitialBodyToWorld.x,
                                         sd.pilotInitialBodyToWorld.y, sd.pilotInitialBodyToWorld.z};
        x.pilot_principal_inertia = {sd.pilotPrincipalInertiaKgSquareMeters.x, sd.pilotPrincipalInertiaKgSquareMeters.y,
                                     sd.pilotPrincipalInertiaKgSquareMeters.z};
        for (const auto& t : sd.attachments) a.attachments.push_back({t.stableId, t.node});
        for (const auto& j : sd.junctions) a.junctions.push_back({j.stableId, j.node});
        for (const auto& h : sd.harnessPoints)
            a.harness.push_back({h.stableId, {h.localPositionMeters.x, h.localPositionMeters.y, h.localPositionMeters.z}});
        for (const auto& g : sd.segments) {
            swb_suspension_segment y{};
            y.stable_id = g.stableId;
            y.from = {static_cast<uint32_t>(g.from.kind), 0u, g.from.stableId};
            y.to = {static_cast<uint32_t>(g.to.kind), 0u, g.to.stableId};
            y.rest_length = g.restLengthMeters;
            y.axial_stiffness = g.axialStiffnessNewtons;
            y.axial_damping = g.axialDampingNewtonSecondsPerMeter;
            y.role = g.role;
            a.segments.push_back(y);
        }
        x.attachment_count = a.attachments.size();
        x.attachments = a.attachments.data();
        x.junction_count = a.junctions.size();
        x.junctions = a.junctions.data();
        x.harness_count = a.harness.size();
        x.harness_points = a.harness.data();
        x.segment_count = a.segments.size();
        x.segments = a.segments.data();
        x.solver_iterations = sd.solverIterations;
        x.attachment_tolerance = sd.attachmentTolerance;
        x.minimum_line_length = sd.minimumLineLengthMeters;
        x.maximum_line_residual = sd.maximumLineResidualMeters;
        x.maximum_control_work = sd.maximumControlWorkJoules;
        a.view.suspension = &a.suspension;
    }
    a.view.node_count = a.nodes.size();
    a.view.nodes = a.nodes.data();
    a.view.triangle_count = a.triangles.size();
    a.view.triangles = a.triangles.data();
    a.view.constraint_count = a.constraints.size();
    a.view.constraints = a.constraints.data();
    a.view.membrane_count = a.membranes.size();
    a.view.membranes = a.membranes.data();
    a.view.dihedral_count = a.dihedrals.size();
    a.view.dihedrals = a.dihedrals.data();
}

// The reference Scene of a swb_scene: the structural fields as given, plus
// what validateScene wants that a swb_scene does not carry (metadata, one
// outside and one cell region on the two sides of every triangle, names).
Scene scene_of(const swb_scene& c) {
    Scene s;
    s.metadata.designChecksum = "synthetic";
    s.metadata.exporterVersion = "synthetic";
    s.regions.push_back({1, RegionKind::Outside, "outside"});
    s.regions.push_back({2, RegionKind::Cell, "cell"});
    for (uint64_t i = 0; i < c.vertex_count; ++i)
        s.vertices.push_back({c.vertices[i].id, {c.vertices[i].position.x, c.vertices[i].position.y,
                                                 c.vertices[i].position.z}});
    for (uint64_t i = 0; i < c.fabric_count; ++i) {
        const swb_scene_fabric& f = c.fabrics[i];
        FabricMaterial m;
        m.id = f.id;
        m.name = "fabric";
        m.warpStiffnessNewtonsPerMeter = f.warp_stiffness;
        m.weftStiffnessNewtonsPerMeter = f.weft_stiffness;
        m.shearStiffnessNewtonsPerMeter = f.shear_stiffness;
        m.bendingStiffnessNewtonMeters = f.bending_stiffness;
        m.arealDensityKgPerSquareMeter = f.areal_density;
        m.dampingSeconds = f.damping_seconds;
        m.porosityFraction = f.porosity;
        m.permeabilitySquareMeters = f.permeability;
        s.fabricMaterials.push_back(m);
    }
    for (uint64_t i = 0; i < c.triangle_count; ++i) {
        const swb_scene_triangle& t = c.triangles[i];
        Triangle x;
        x.id = t.id;
        for (int k = 0; k < 3; ++k) {
            x.vertexIds[k] = t.vertex_ids[k];
            x.materialCoordinates[k] = {t.chart[k][0], t.chart[k][1]};
        }
        x.negativeSideRegionId = 2;
        x.positiveSideRegionId = 1;
        x.materialId = t.material_id;
        x.sheetId = t.sheet_id;
        x.role = SurfaceRole::Skin;
        s.triangles.push_back(x);
    }
    for (uint64_t i = 0; i < c.seam_material_count; ++i)
        s.seamMaterials.push_back({c.seam_materials[i].id, "seam", c.seam_materials[i].linear_density,
                                   c.seam_materials[i].axial_stiffness});
    for (uint64_t i = 0; i < c.seam_count; ++i) {
        const swb_scene_seam& m = c.seams[i];
        Seam x;
        x.id = m.id;
        x.materialId = m.material_id;
        x.firstOrderedVertexIds.assign(c.seam_vertex_ids + m.first_begin, c.seam_vertex_ids + m.first_begin + m.count);
        x.secondOrderedVertexIds.assign(c.seam_vertex_ids + m.second_begin,
                                        c.seam_vertex_ids + m.second_begin + m.count);
        s.seams.push_back(x);
    }
    for (uint64_t i = 0; i < c.line_material_count; ++i) {
        const swb_scene_line_material& m = c.line_materials[i];
        s.lineMaterials.push_back({m.id, "line", m.diameter, m.linear_density, m.axial_stiffness, m.drag_coefficient});
    }
    for (uint64_t i = 0; i < c.pilot_count; ++i) {
        const swb_scene_pilot& p = c.pilots[i];
        Pilot x;
        x.id = p.id;
        x.name = "pilot";
        x.massKg = p.mass;
        x.centerOfMassPositionMeters = {p.center_of_mass.x, p.center_of_mass.y, p.center_of_mass.z};
        x.linearVelocityMetersPerSecond = {p.linear_velocity.x, p.linear_velocity.y, p.linear_velocity.z};
        x.bodyToWorld = {p.body_to_world.w, p.body_to_world.x, p.body_to_world.y, p.body_to_world.z};
        x.principalInertiaKgSquareMeters = {p.principal_inertia.x, p.principal_inertia.y, p.principal_inertia.z};
        s.pilots.push_back(x);
    }
    for (uint64_t i = 0; i < c.junction_count; ++i) {
        const swb_scene_junction& j = c.junctions[i];
        s.suspensionJunctions.push_back({j.id, {j.position.x, j.position.y, j.position.z}, j.mass, j.fixed != 0});
    }
    for (uint64_t i = 0; i < c.attachment_count; ++i) {
        const swb_scene_attachment& a = c.attachments[i];
        Attachment x;
        x.id = a.id;
        x.kind = static_cast<AttachmentKind>(a.kind);
        x.vertexId = a.vertex_id;
        x.pilotId = a.pilot_id;
        x.pilotLocalPositionMeters = {a.pilot_local_position.x, a.pilot_local_position.y, a.pilot_local_position.z};
        x.suspensionJunctionId = a.junction_id;
        s.attachments.push_back(x);
    }
    for (uint64_t i = 0; i < c.line_count; ++i) {
        const swb_scene_line& l = c.lines[i];
        SuspensionLine x;
        x.id = l.id;
        x.startAttachmentId = l.start_attachment_id;
        x.endAttachmentId = l.end_attachment_id;
        x.materialId = l.material_id;
        x.restLengthMeters = l.rest_length;
        x.role = static_cast<SuspensionLineRole>(l.role);
        s.suspensionLines.push_back(x);
    }
    return s;
}

extern "C" {

const char* swref_last_error(void) { return g_error.c_str(); }

// assembleSceneStructure on the reference build: the definition (valid
// until swref_assembly_destroy) and the first diagnostic.
int swref_assemble_scene(const swb_scene* scene, const swb_scene_settings* settings, void** out,
                         swb_scene_report* report) {
    try {
        *out = nullptr;
        SceneStructureSettings st;
        st.seamCoincidenceToleranceMeters = settings->seam_coincidence_tolerance;
        st.suspensionSolverIterations = settings->suspension_solver_iterations;
        st.suspensionAttachmentTolerance = settings->suspension_attachment_tolerance;
        st.suspensionMinimumLineLengthMeters = settings->suspension_minimum_line_length;
        st.suspensionMaximumLineResidualMeters = settings->suspension_maximum_line_residual;
        st.suspensionMaximumControlWorkJoules = settings->suspension_maximum_control_work;
        if (settings->has_fabric_self_contact) {
            const auto& c = settings->fabric_self_contact;
            st.fabricSelfContact = StructureFabricContactDefinition{c.half_thickness, c.normal_compliance,
                                                                    c.static_friction, c.dynamic_friction};
        }
        const SceneStructureAssembly a = assembleSceneStructure(scene_of(*scene), {}, st);
        std::memset(report, 0, sizeof(*report));
        report->diagnostic_count = static_cast<uint32_t>(a.diagnostics.size());
        if (!a.diagnostics.empty()) {
            const auto& d = a.diagnostics.front();
            report->first_code = static_cast<uint32_t>(d.code);
            report->first_validation_code = d.sceneValidationCode ? static_cast<uint32_t>(*d.sceneValidationCode) : 0u;
            report->first_entity_kind = static_cast<uint32_t>(d.entityKind);
            report->first_entity_id = d.entityId;
            std::snprintf(report->first_message, sizeof report->first_message, "%s", d.message.c_str());
        }
        if (!a.ok()) return SWB_INVALID_ARGUMENT;
        report->assembled = 1;
        report->total_fabric_mass = a.totalFabricMassKg;
        report->total_seam_mass = a.totalSeamMassKg;
        auto* r = new RefAssembly;
        export_definition(a.definition, *r);
        *out = r;
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

const swb_structure_definition* swref_assembly_view(void* assembly) {
    return &static_cast<RefAssembly*>(assembly)->view;
}

void swref_assembly_destroy(void* assembly) { delete static_cast<RefAssembly*>(assembly); }

int swref_last_error_detail(swb_error_detail* out) {
    if (!out) return SWB_INVALID_ARGUMENT;
    *out = g_detail;
    return SWB_OK;
}

unsigned swref_physical_cores(void) {
    return softwing::hardwarePhysicalCoreCount();
}

swb_status swref_create(const swb_structure_definition* definition,
                        void** out) {
    try {
        auto handle = std::make_unique<RefHandle>();
        handle->structure =
            std::make_unique<Structure>(convert(*definition));
        handle->triangles.reserve(definition->triangle_count);
        handle->pressure.reserve(definition->triangle_count);
        for (uint64_t i = 0; i < definition->triangle_count; ++i) {
            const swb_triangle_def& t = definition->triangles[i];
            handle->triangles.push_back({t.nodes[0], t.nodes[1], t.nodes[2]});
            handle->pressure.push_back(t.pressure_difference);
            handle->anyPressure =
                handle->anyPressure || t.pressure_difference != 0.0;
        }
        *out = handle.release();
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

void swref_destroy(void* handle) { delete static_cast<RefHandle*>(handle); }

// Structure::definitionFingerprint (structure.h:284).
uint64_t swref_fingerprint(void* handle) {
    return static_cast<RefHandle*>(handle)->structure->definitionFingerprint();
}

swb_status swref_set_external_forces(void* handle,
                                     const swb_vec3* forces,
                                     uint64_t count) {
    try {
        auto* h = static_cast<RefHandle*>(handle);
        std::vector<StructureVector3> values(count);
        for (uint64_t i = 0; i < count; ++i)
            values[i] = {forces[i].x, forces[i].y, forces[i].z};
        h->structure->setExternalForces(values);
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

swb_status swref_add_external_force(void* handle,
                                    uint64_t node,
                                    const swb_vec3* force) {
    try {
        static_cast<RefHandle*>(handle)->structure->addExternalForce(
            node, {force->x, force->y, force->z});
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

swb_status swref_step(void* handle,
                      const swb_step_settings* settings,
                      swb_diagnostics* out) {
    try {
        auto* h = static_cast<RefHandle*>(handle);
        const auto start = std::chrono::steady_clock::now();
        if (h->anyPressure) {
            const std::vector<StructureNodeState> nodes =
                h->structure->nodeStates();
            for (std::size_t t = 0; t < h->triangles.size(); ++t) {
                if (h->pressure[t] == 0.0) continue;
                const auto& tri = h->triangles[t];
                const StructureVector3& a = nodes[tri[0]].positionMeters;
                const StructureVector3& b = nodes[tri[1]].positionMeters;
                const StructureVector3& c = nodes[tri[2]].positionMeters;
                const double ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
                const double vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
                const double ax = 0.5 * (uy * vz - uz * vy);
                const double ay = 0.5 * (uz * vx - ux * vz);
                const double az = 0.5 * (ux * vy - uy * vx);
                const StructureVector3 f{h->pressure[t] * ax / 3.0,
                                         h->pressure[t] * ay / 3.0,
                                         h->pressure[t] * az / 3.0};
                for (int k = 0; k < 3; ++k)
                    h->structure->addExternalForce(tri[k], f);
            }
        }
        const StructureDiagnostics d =
            h->structure->step(convert(*settings));
        h->lastStepSeconds = std::chrono::duration<double>(
                                 std::chrono::steady_clock::now() - start)
                                 .count();
        if (out) toDiagnostics(d, out);
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

double swref_last_step_seconds(void* handle) {
    return static_cast<RefHandle*>(handle)->lastStepSeconds;
}

swb_status swref_diagnostics(void* handle, swb_diagnostics* out) {
    try {
        toDiagnostics(static_cast<RefHandle*>(handle)->structure->diagnostics(),
                      out);
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

swb_status swref_read_nodes(void* handle, swb_node_state* out, uint64_t count) {
    try {
        const auto nodes =
            static_cast<RefHandle*>(handle)->structure->nodeStates();
        if (count != nodes.size())
            throw std::invalid_argument("node count mismatch");
        for (uint64_t i = 0; i < count; ++i) {
            out[i].position = {nodes[i].positionMeters.x,
                               nodes[i].positionMeters.y,
                               nodes[i].positionMeters.z};
            out[i].previous_position = {nodes[i].previousPositionMeters.x,
                                        nodes[i].previousPositionMeters.y,
                                        nodes[i].previousPositionMeters.z};
            out[i].velocity = {nodes[i].velocityMetersPerSecond.x,
                               nodes[i].velocityMetersPerSecond.y,
                               nodes[i].velocityMetersPerSecond.z};
        }
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

// Reads the payload state and the per-segment tension, in definition order.
swb_status swref_read_suspension(void* handle,
                                 swb_payload_state* payload,
                                 swb_segment_state* segments,
                                 uint64_t capacity) {
    try {
        const auto state =
            static_cast<RefHandle*>(handle)->structure->suspensionState();
        if (!state) throw std::invalid_argument("no suspension");
        const auto& p = state->payload;
        payload->center_of_mass = {p.centerOfMassWorldMeters.x,
                                   p.centerOfMassWorldMeters.y,
                                   p.centerOfMassWorldMeters.z};
        payload->body_to_world = {p.bodyToWorld.w, p.bodyToWorld.x,
                                  p.bodyToWorld.y, p.bodyToWorld.z};
        payload->linear_velocity = {p.linearVelocityMetersPerSecond.x,
                                    p.linearVelocityMetersPerSecond.y,
                                    p.linearVelocityMetersPerSecond.z};
        payload->angular_velocity = {p.angularVelocityRadiansPerSecond.x,
                                     p.angularVelocityRadiansPerSecond.y,
                                     p.angularVelocityRadiansPerSecond.z};
        for (uint64_t i = 0; i < capacity && i < state->segments.size(); ++i) {
            segments[i].stable_id = state->segments[i].stableId;
            segments[i].current_length = state->segments[i].currentLengthMeters;
            segments[i].commanded_rest_length =
                state->segments[i].commandedRestLengthMeters;
            segments[i].tension = state->segments[i].tensionNewtons;
        }
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

// softwing::SoftBody::constraintColouringView (soft_body.h:463-467) on a body
// holding the definition's nodes and distance-like constraints.
swb_status swref_colouring(const swb_structure_definition* d,
                           uint64_t* order,
                           uint64_t* offsets,
                           uint64_t offsets_capacity,
                           uint64_t* colour_count,
                           uint64_t* parallel_colours) {
    try {
        softwing::SoftBody body;
        for (uint64_t i = 0; i < d->node_count; ++i) {
            const swb_node_def& n = d->nodes[i];
            const softwing::Vec3 p{n.position.x, n.position.y, n.position.z};
            if (n.fixed)
                body.addFixedNode(p);
            else
                body.addNode(p, n.mass);
        }
        for (uint64_t i = 0; i < d->constraint_count; ++i) {
            const swb_constraint_def& c = d->constraints[i];
            switch (c.kind) {
            case SWB_CONSTRAINT_CABLE:
                body.addCableConstraint(c.first_node, c.second_node,
                                        c.rest_length, c.compliance);
                break;
            case SWB_CONSTRAINT_SUSPENSION_TIE:
                body.addSuspensionTieConstraint(c.first_node, c.second_node,
                                                c.rest_length, c.compliance);
                break;
            case SWB_CONSTRAINT_SEAM_STITCH:
                body.addSeamStitchConstraint(c.first_node, c.second_node);
                break;
            default:
                body.addDistanceConstraint(c.first_node, c.second_node,
                                           c.rest_length, c.compliance);
            }
        }
        const auto view = body.constraintColouringView();
        const auto report = body.constraintColouringReport();
        for (std::size_t i = 0; i < view.order.size(); ++i)
            order[i] = view.order[i];
        if (view.colourOffsets.size() > offsets_capacity)
            throw std::invalid_argument("offsets capacity too small");
        for (std::size_t i = 0; i < view.colourOffsets.size(); ++i)
            offsets[i] = view.colourOffsets[i];
        *colour_count =
            view.colourOffsets.empty() ? 0 : view.colourOffsets.size() - 1;
        *parallel_colours = report.parallelColours;
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

// Candidate keys of the fabric self-contact pair (structure.cpp:626-636) for
// the motion previous -> current: one SoftBody contact iteration
// (contact.cpp:1057-1290) on a body holding the definition's nodes and
// triangles, read back through the reference's audit hook.  possible /
// excluded from SoftBody::contactTopology (contact.cpp:2448).
swb_status swref_contact_candidates(const swb_structure_definition* d,
                                    double half_thickness,
                                    const double* previous,
                                    const double* current,
                                    swb_contact_key* keys,
                                    uint64_t capacity,
                                    uint64_t* count,
                                    uint64_t* possible,
                                    uint64_t* excluded) {
    try {
        softwing::SoftBody body;
        for (uint64_t i = 0; i < d->node_count; ++i) {
            const swb_node_def& n = d->nodes[i];
            const softwing::Vec3 p{n.position.x, n.position.y, n.position.z};
            if (n.fixed)
                body.addFixedNode(p);
            else
                body.addNode(p, n.mass);
        }
        for (uint64_t i = 0; i < d->triangle_count; ++i)
            body.addTriangle(d->triangles[i].nodes[0], d->triangles[i].nodes[1],
                             d->triangles[i].nodes[2]);
        const softwing::ContactSurfaceHandle surface = body.addContactSurface(
            body.surfaceGroup(0, d->triangle_count), half_thickness);
        const softwing::ContactPairHandle pair = body.addContactPair(
            surface.collider(), surface.collider(), {0.0, 0.0, 0.0});
        const softwing::ContactTopologyReport topology = body.contactTopology(pair);
        for (uint64_t i = 0; i < d->node_count; ++i) {
            softwing::Node& n = body.nodes()[i];
            n.previousPosition = {previous[3 * i], previous[3 * i + 1], previous[3 * i + 2]};
            n.position = {current[3 * i], current[3 * i + 1], current[3 * i + 2]};
        }
        softwing::ContactAuditTestAccess::begin(body);
        softwing::StepSettings settings;
        try {
            softwing::ContactAuditTestAccess::iterate(body, 1.0 / 120.0, settings);
        } catch (const softwing::ContactStepError&) {
            // The candidate list is complete before any feature is queried.
        }
        const auto& found = softwing::ContactAuditTestAccess::candidates(body);
        *count = found.size();
        if (possible) *possible = topology.possibleCount;
        if (excluded) *excluded = topology.excludedCount;
        if (found.size() > capacity)
            throw std::out_of_range("candidate capacity too small");
        for (std::size_t k = 0; k < found.size(); ++k) {
            swb_contact_key& out = keys[k];
            std::memset(&out, 0, sizeof out);
            out.pair = found[k].pair;
            out.kind = static_cast<uint32_t>(found[k].kind);
            for (int j = 0; j < 3; ++j) {
                out.first[j] = found[k].firstPrimitive[j];
                out.second[j] = found[k].secondPrimitive[j];
            }
        }
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

namespace {

softwing::Vec3 vec_at(const double* p, uint64_t feature, int point) {
    const double* q = p + 9 * feature + 3 * point;
    return {q[0], q[1], q[2]};
}

void store_vec(double* out, const softwing::Vec3& v) {
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

void store_closest(swb_closest_result& o, const softwing::ClosestFeatureResult& r) {
    std::memset(&o, 0, sizeof o);
    o.status = static_cast<uint32_t>(r.status);
    o.first_feature = static_cast<uint32_t>(r.firstFeature);
    o.second_feature = static_cast<uint32_t>(r.secondFeature);
    store_vec(o.first_point, r.firstPoint);
    store_vec(o.second_point, r.secondPoint);
    for (int k = 0; k < 3; ++k) {
        o.first_weights[k] = r.firstWeights[k];
        o.second_weights[k] = r.secondWeights[k];
    }
    store_vec(o.normal, r.normal);
    o.distance = r.distance;
    o.gap = r.gap;
}

}  // namespace

// closestVertexTriangle / closestEdgeEdge (contact.h:70-93), per feature.
swb_status swref_contact_closest(uint32_t kind, uint64_t count,
                                 const double* first, const double* second,
                                 double separation,
                                 swb_closest_result* results) {
    try {
        for (uint64_t i = 0; i < count; ++i) {
            const softwing::ClosestFeatureResult r =
                kind == SWB_FEATURE_VERTEX_TRIANGLE
                    ? softwing::closestVertexTriangle(
                          vec_at(first, i, 0), vec_at(second, i, 0),
                          vec_at(second, i, 1), vec_at(second, i, 2), separation)
                    : softwing::closestEdgeEdge(
                          vec_at(first, i, 0), vec_at(first, i, 1),
                          vec_at(second, i, 0), vec_at(second, i, 1), separation);
            store_closest(results[i], r);
        }
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

// sweptContact (contact.h:265-270), per feature.
swb_status swref_contact_sweep(uint32_t kind, uint64_t count,
                               const double* first_previous,
                               const double* first_current,
                               const double* second_previous,
                               const double* second_current,
                               double separation,
                               const swb_ccd_settings* settings,
                               swb_ccd_result* results) {
    try {
        softwing::CcdSettings cs;
        cs.conservativeIterations = settings->conservative_iterations;
        cs.intervalSubdivisions = settings->interval_subdivisions;
        cs.timeTolerance = settings->time_tolerance;
        cs.distanceTolerance = settings->distance_tolerance;
        const bool vt = kind == SWB_FEATURE_VERTEX_TRIANGLE;
        const auto kindValue = vt ? softwing::ContactFeatureKind::VertexTriangle
                                  : softwing::ContactFeatureKind::EdgeEdge;
        for (uint64_t i = 0; i < count; ++i) {
            softwing::LinearContactPrimitive f, s;
            f.count = vt ? 1 : 2;
            s.count = vt ? 3 : 2;
            for (std::size_t k = 0; k < f.count; ++k) {
                f.previous[k] = vec_at(first_previous, i, static_cast<int>(k));
                f.current[k] = vec_at(first_current, i, static_cast<int>(k));
            }
            for (std::size_t k = 0; k < s.count; ++k) {
                s.previous[k] = vec_at(second_previous, i, static_cast<int>(k));
                s.current[k] = vec_at(second_current, i, static_cast<int>(k));
            }
            const softwing::CcdResult r =
                softwing::sweptContact(kindValue, f, s, separation, cs);
            swb_ccd_result& o = results[i];
            std::memset(&o, 0, sizeof o);
            o.state = static_cast<uint32_t>(r.state);
            o.conservative_iterations = r.conservativeIterations;
            o.interval_subdivisions = r.intervalSubdivisions;
            o.used_interval_fallback = r.usedIntervalFallback ? 1u : 0u;
            o.time_of_impact = r.timeOfImpact;
            o.bracket_lower = r.bracketLower;
            o.bracket_upper = r.bracketUpper;
            store_closest(o.geometry, r.geometry);
        }
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

// softwing::estimateClosedCellVolume (cell_volume.h:38-44) per cell, on the
// definition's triangles at `positions`.
swb_status swref_cell_volumes(const swb_structure_definition* d,
                              const uint64_t* face_indices,
                              const uint64_t* loop_nodes,
                              const swb_cell_def* cells,
                              uint64_t cell_count,
                              const double* positions,
                              swb_cell_volume* out) {
    try {
        std::vector<softwing::Node> nodes(d->node_count);
        for (uint64_t i = 0; i < d->node_count; ++i)
            nodes[i].position = {positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
        std::vector<softwing::Triangle> triangles(d->triangle_count);
        for (uint64_t t = 0; t < d->triangle_count; ++t) {
            triangles[t].a = d->triangles[t].nodes[0];
            triangles[t].b = d->triangles[t].nodes[1];
            triangles[t].c = d->triangles[t].nodes[2];
        }
        for (uint64_t k = 0; k < cell_count; ++k) {
            const swb_cell_def& c = cells[k];
            const std::vector<std::size_t> faces(face_indices + c.face_begin,
                                                 face_indices + c.face_begin + c.face_count);
            const std::vector<std::size_t> low(loop_nodes + c.low_begin, loop_nodes + c.low_begin + c.low_count);
            const std::vector<std::size_t> high(loop_nodes + c.high_begin,
                                                loop_nodes + c.high_begin + c.high_count);
            const softwing::ClosedCellVolumeEstimate e =
                softwing::estimateClosedCellVolume(nodes, triangles, faces, low, high);
            swb_cell_volume& o = out[k];
            std::memset(&o, 0, sizeof o);
            o.signed_volume = e.signedVolume;
            o.volume = e.volume;
            o.skin_boundary_edges = e.skinBoundaryEdges;
            o.cap_boundary_edges_matched = e.capBoundaryEdgesMatched;
            o.non_manifold_skin_edges = e.nonManifoldSkinEdges;
            o.degenerate_skin_faces = e.degenerateSkinFaces;
            o.valid = e.valid;
            o.watertight_after_capping = e.watertightAfterCapping;
            o.used_geometric_orientation_fallback = e.usedGeometricOrientationFallback;
            o.ambiguous_skin_orientation = e.ambiguousSkinOrientation;
        }
        return SWB_OK;
    } catch (...) {
        return translate();
    }
}

}  // extern "C"

// evaluateOrificeMassFlow / evaluateConductanceMassFlow (pneumatics.cpp:
// 132-232) over many ports, with swb_port_mass_flows's conventions: the first
// port the reference refuses is reported, as SWB_INVALID_ARGUMENT.
extern "C" swb_status swref_port_mass_flows(const swb_air_properties* air,
                                            const swb_flow_zone_state* zones,
                                            uint64_t zone_count,
                                            const swb_port_def* ports,
                                            uint64_t port_count,
                                            swb_mass_flow* out,
                                            uint64_t* failed_port) {
    if (failed_port) *failed_port = port_count;
    softwing::AirProperties a;
    a.specificGasConstant = air->specific_gas_constant;
    a.heatCapacityRatio = air->heat_capacity_ratio;
    for (uint64_t i = 0; i < port_count; ++i)
        if (ports[i].first >= zone_count || ports[i].second >= zone_count) return SWB_OUT_OF_RANGE;
    for (uint64_t i = 0; i < port_count; ++i) {
        const swb_port_def& p = ports[i];
        softwing::FlowZoneState first{zones[p.first].absolute_pressure, zones[p.first].absolute_temperature};
        softwing::FlowZoneState second{zones[p.second].absolute_pressure, zones[p.second].absolute_temperature};
        try {
            if (p.reserved != 0 || p.kind > SWB_PORT_CONDUCTANCE) throw std::invalid_argument("port kind");
            softwing::MassFlowEvaluation e;
            if (p.kind == SWB_PORT_ORIFICE) {
                softwing::OrificeDefinition d;
                d.dischargeCoefficient = p.discharge_coefficient;
                d.effectiveArea = p.effective_area;
                d.openingFraction = p.opening_fraction;
                e = softwing::evaluateOrificeMassFlow(first, second, a, d);
            } else {
                softwing::ConductanceDefinition d;
                d.massConductance = p.mass_conductance;
                d.openingFraction = p.opening_fraction;
                e = softwing::evaluateConductanceMassFlow(first, second, d);
            }
            swb_mass_flow& o = out[i];
            std::memset(&o, 0, sizeof o);
            o.signed_mass_rate = e.signedMassRate;
            o.magnitude = e.magnitude;
            o.pressure_ratio = e.pressureRatio;
            o.critical_pressure_ratio = e.criticalPressureRatio;
            o.direction = static_cast<uint32_t>(e.direction);
            o.choked = e.choked ? 1u : 0u;
        } catch (const std::invalid_argument&) {
            if (failed_port && *failed_port == port_count) *failed_port = i;
        }
    }
    return failed_port && *failed_port != port_count ? SWB_INVALID_ARGUMENT : SWB_OK;
}
