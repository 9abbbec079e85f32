// Exercises the C++ mirror of simwing::fsi::Structure
// (include/simwing_b200_structure.hpp) the way the reference's adapter test
// exercises the original (tests/simwing_structure_test.cpp): construction
// and validation errors, typed exceptions on bad loads, accepted-step load
// consumption, checkpoint / restore bit replay and tamper rejection.
//
//   structure_mirror_test cpu   checks that need no device
//   structure_mirror_test gpu   steps the synthetic patch and wing on device 0
//
// Prints one line per check and exits non-zero on the first failure.
#include "simwing_b200_structure.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <string>

using namespace simwing::fsi;

namespace {

int failures = 0;

void expect(bool ok, const char* what) {
    std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
    if (!ok) ++failures;
}

template <class E>
void expect_throw(const std::function<void()>& f, const char* what) {
    bool thrown = false;
    try {
        f();
    } catch (const E&) {
        thrown = true;
    } catch (const std::exception& e) {
        std::printf("     unexpected exception: %s\n", e.what());
    }
    expect(thrown, what);
}

StructureDefinition from_view(const swb_structure_definition& v) {
    StructureDefinition d;
    for (uint64_t i = 0; i < v.node_count; ++i) {
        const auto& n = v.nodes[i];
        d.nodes.push_back({{n.position.x, n.position.y, n.position.z}, n.mass, n.fixed != 0});
    }
    for (uint64_t i = 0; i < v.triangle_count; ++i) {
        const auto& t = v.triangles[i];
        d.triangles.push_back({{t.nodes[0], t.nodes[1], t.nodes[2]}});
    }
    for (uint64_t i = 0; i < v.constraint_count; ++i) {
        const auto& c = v.constraints[i];
        d.constraints.push_back({static_cast<StructureConstraintKind>(c.kind), c.first_node, c.second_node,
                                 c.rest_length, c.compliance});
    }
    for (uint64_t i = 0; i < v.dihedral_count; ++i) {
        const auto& h = v.dihedrals[i];
        d.dihedrals.push_back({{h.nodes[0], h.nodes[1], h.nodes[2], h.nodes[3]}, h.rest_angle, h.compliance});
    }
    if (v.suspension) {
        const auto& s = *v.suspension;
        StructureSuspensionDefinition r;
        r.pilotStableId = s.pilot_stable_id;
        r.pilotMassKg = s.pilot_mass;
        auto vec = [](const swb_vec3& x) { return StructureVector3{x.x, x.y, x.z}; };
        r.pilotCenterOfMassLocalMeters = vec(s.pilot_com_local);
        r.pilotInitialCenterOfMassWorldMeters = vec(s.pilot_initial_com_world);
        r.pilotInitialLinearVelocityMetersPerSecond = vec(s.pilot_initial_linear_velocity);
        r.pilotInitialAngularVelocityRadiansPerSecond = vec(s.pilot_initial_angular_velocity);
        r.pilotInitialBodyToWorld = {s.pilot_initial_body_to_world.w, s.pilot_initial_body_to_world.x,
                                     s.pilot_initial_body_to_world.y, s.pilot_initial_body_to_world.z};
        r.pilotPrincipalInertiaKgSquareMeters = vec(s.pilot_principal_inertia);
        for (uint64_t i = 0; i < s.attachment_count; ++i)
            r.attachments.push_back({s.attachments[i].stable_id, s.attachments[i].node});
        for (uint64_t i = 0; i < s.junction_count; ++i)
            r.junctions.push_back({s.junctions[i].stable_id, s.junctions[i].node});
        for (uint64_t i = 0; i < s.harness_count; ++i)
            r.harnessPoints.push_back({s.harness_points[i].stable_id, vec(s.harness_points[i].local_position)});
        for (uint64_t i = 0; i < s.segment_count; ++i) {
            const auto& g = s.segments[i];
            StructureSuspensionSegmentDefinition e;
            e.stableId = g.stable_id;
            e.from = {static_cast<StructureSuspensionEndpointKind>(g.from.kind), g.from.stable_id};
            e.to = {static_cast<StructureSuspensionEndpointKind>(g.to.kind), g.to.stable_id};
            e.restLengthMeters = g.rest_length;
            e.axialStiffnessNewtons = g.axial_stiffness;
            e.axialDampingNewtonSecondsPerMeter = g.axial_damping;
            e.role = g.role;
            r.segments.push_back(e);
        }
        r.solverIterations = s.solver_iterations;
        r.attachmentTolerance = s.attachment_tolerance;
        r.minimumLineLengthMeters = s.minimum_line_length;
        r.maximumLineResidualMeters = s.maximum_line_residual;
        r.maximumControlWorkJoules = s.maximum_control_work;
        d.suspension = r;
    }
    return d;
}

StructureDefinition patch_definition() {
    swb_patch_params p;
    swb_default_patch_params(&p);
    swb_definition* def = nullptr;
    simwing_b200::check(swb_generate_patch(&p, &def));
    StructureDefinition d = from_view(*swb_definition_view(def));
    swb_definition_destroy(def);
    return d;
}

StructureDefinition small_wing_definition() {
    swb_wing_params p;
    swb_default_wing_params(&p);
    p.cells = 4;
    p.chordwise = 10;
    p.spanwise_per_cell = 2;
    p.rib_layers = 2;
    p.pressure = 0.0;  // the adapter definition carries no face pressure
    swb_definition* def = nullptr;
    simwing_b200::check(swb_generate_wing(&p, &def));
    StructureDefinition d = from_view(*swb_definition_view(def));
    swb_definition_destroy(def);
    return d;
}

StructureStepSettings settings() {
    StructureStepSettings s;
    s.substeps = 1;
    s.constraintIterations = 48;
    s.gravityMetersPerSecondSquared = {0.0, 0.0, -9.81};
    return s;
}

void cpu_checks() {
    StructureStepSettings s;
    expect(s.timeStepSeconds == 1.0 / 120.0 && s.substeps == 2 && s.constraintIterations == 12 &&
               s.gravityMetersPerSecondSquared.z == -9.80665 && s.velocityDampingPerSecond == 0.25,
           "step settings defaults are the reference's");
    StructureDefinition bad = patch_definition();
    bad.triangles[3].nodes[1] = bad.triangles[3].nodes[0];
    expect_throw<std::invalid_argument>([&] { Structure x(bad); }, "triangle repeating a node is rejected");
    StructureDefinition bad2 = patch_definition();
    bad2.constraints[0].restLengthMeters = -1.0;
    expect_throw<std::invalid_argument>([&] { Structure x(bad2); }, "negative rest length is rejected");
    StructureDefinition mem = patch_definition();
    mem.membranes.push_back({});
    expect_throw<std::invalid_argument>([&] { Structure x(mem); }, "invalid membrane definition is rejected");
    expect_throw<std::out_of_range>([] { simwing_b200::check(SWB_OUT_OF_RANGE); }, "status maps to out_of_range");
    expect_throw<softwing::SuspensionError>([] { simwing_b200::check(SWB_SUSPENSION_ERROR); },
                                            "status maps to SuspensionError");
    expect_throw<softwing::ContactStepError>([] { simwing_b200::check(SWB_CONTACT_ERROR); },
                                             "status maps to ContactStepError");
    expect_throw<simwing_b200::DeviceStepError>([] { simwing_b200::check(SWB_SYNC_TIMEOUT); },
                                                "status maps to DeviceStepError");
}

bool same_nodes(const std::vector<StructureNodeState>& a, const std::vector<StructureNodeState>& b) {
    return a == b;
}

void gpu_checks() {
    // the mirror and the C-ABI on the same definition step bit-identically
    const StructureDefinition d = patch_definition();
    Structure s(d);
    detail::AbiDefinition abi(d);
    swb_structure* raw = nullptr;
    simwing_b200::check(swb_structure_create(&abi.view, nullptr, &raw));
    const swb_step_settings rs = detail::to_swb(settings());
    for (int i = 0; i < 5; ++i) {
        (void)s.step(settings());
        simwing_b200::check(swb_structure_step(raw, &rs, nullptr));
    }
    std::vector<swb_node_state> direct(d.nodes.size());
    simwing_b200::check(swb_structure_read_nodes(raw, direct.data(), direct.size()));
    const auto mirrored = s.nodeStates();
    bool equal = true;
    for (size_t i = 0; i < direct.size(); ++i)
        equal = equal && direct[i].position.x == mirrored[i].positionMeters.x &&
                direct[i].position.y == mirrored[i].positionMeters.y &&
                direct[i].position.z == mirrored[i].positionMeters.z;
    expect(equal, "mirror steps bit-identically to the C-ABI");
    swb_structure_destroy(raw);
    expect(s.acceptedStepCount() == 5 && std::fabs(s.simulationTimeSeconds() - 5.0 / 120.0) < 1e-12,
           "accepted steps and simulation time advance");

    // typed load errors, loads consumed only by an accepted step
    expect_throw<std::out_of_range>([&] { s.addExternalForce(d.nodes.size(), {1, 0, 0}); },
                                    "force on a missing node throws out_of_range");
    expect_throw<std::invalid_argument>([&] { s.addExternalForce(0, {NAN, 0, 0}); },
                                        "non-finite force throws invalid_argument");
    std::vector<StructureVector3> short_forces(3);
    expect_throw<std::invalid_argument>([&] { s.setExternalForces(short_forces); },
                                        "force span of the wrong size throws invalid_argument");
    s.addExternalForce(7, {0.0, 0.0, 1e-3});
    expect(s.diagnostics().pendingExternalForceNewtons.z == 1e-3, "pending force is reported");
    StructureStepSettings bad = settings();
    bad.timeStepSeconds = -1.0;
    expect_throw<std::invalid_argument>([&] { (void)s.step(bad); }, "negative time step throws invalid_argument");
    expect(s.diagnostics().pendingExternalForceNewtons.z == 1e-3, "a rejected step keeps the pending load");
    const auto diag = s.step(settings());
    expect(diag.lastAppliedExternalForceNewtons.z == 1e-3 && diag.pendingExternalForceNewtons.z == 0.0,
           "an accepted step consumes the pending load");

    // checkpoint / restore: bit replay and tamper rejection
    const StructureCheckpoint c = s.checkpoint();
    expect(c.definitionFingerprint == s.definitionFingerprint() && c.nodes == s.nodeStates(),
           "checkpoint public fields match the state");
    for (int i = 0; i < 4; ++i) (void)s.step(settings());
    const auto first = s.nodeStates();
    s.restore(c);
    expect(s.acceptedStepCount() == c.acceptedStepCount, "restore resets the step count");
    for (int i = 0; i < 4; ++i) (void)s.step(settings());
    expect(same_nodes(first, s.nodeStates()), "replay after restore is bit-identical");
    StructureCheckpoint tampered = c;
    tampered.nodes[0].positionMeters.x += 1.0;
    expect_throw<std::invalid_argument>([&] { s.restore(tampered); }, "tampered checkpoint is rejected");
    StructureCheckpoint foreign = c;
    foreign.definitionFingerprint ^= 1u;
    expect_throw<std::invalid_argument>([&] { s.restore(foreign); }, "foreign checkpoint is rejected");
    expect(same_nodes(first, s.nodeStates()), "rejected restores leave the state unchanged");

    // move-only ownership
    Structure moved(std::move(s));
    expect(moved.acceptedStepCount() == c.acceptedStepCount + 4, "structure is movable");

    // suspension state of the wing with its rigid pilot
    Structure w(small_wing_definition());
    for (int i = 0; i < 3; ++i) (void)w.step(settings());
    const auto susp = w.suspensionState();
    expect(susp.has_value() && susp->segments.size() == 2 && susp->harnessPositionsMeters.size() == 2,
           "suspension state reports both risers and harness points");
    bool tensioned = susp && susp->segments[0].tensionNewtons > 0.0 && susp->segments[1].tensionNewtons > 0.0;
    expect(tensioned, "risers carry the pilot");
    const auto& p = susp->payload;
    const double qn = p.bodyToWorld.w * p.bodyToWorld.w + p.bodyToWorld.x * p.bodyToWorld.x +
                      p.bodyToWorld.y * p.bodyToWorld.y + p.bodyToWorld.z * p.bodyToWorld.z;
    expect(std::fabs(qn - 1.0) < 1e-5, "payload orientation stays a unit quaternion");

    // typed step failures with the reference's details; the caller compares
    // the printed details with what the reference build throws on the same
    // definitions (tests/test_cpp_mirror.py)
    StructureDefinition strict = small_wing_definition();
    strict.suspension->maximumLineResidualMeters = 0.0;
    Structure sw(strict);
    bool caught = false;
    try {
        for (int i = 0; i < 20; ++i) (void)sw.step(settings());
    } catch (const softwing::SuspensionError& e) {
        caught = true;
        std::printf("detail suspension %d %s\n", static_cast<int>(e.phase()), e.entity().c_str());
    }
    expect(caught, "a zero line residual bound throws SuspensionError");
    StructureDefinition pinned;
    const double z[2] = {0.0, 0.005};
    for (int sheet = 0; sheet < 2; ++sheet) {
        pinned.nodes.push_back({{-1.0, -1.0, z[sheet]}, 1.0, true});
        pinned.nodes.push_back({{sheet ? 0.0 : 1.0, sheet ? 1.0 : -1.0, z[sheet]}, 1.0, true});
        pinned.nodes.push_back({{sheet ? 1.0 : 0.0, sheet ? -1.0 : 1.0, z[sheet]}, 1.0, true});
    }
    pinned.nodes.push_back({{3.0, 3.0, 3.0}, 1.0, false});
    pinned.triangles.push_back({{0, 1, 2}});
    pinned.triangles.push_back({{3, 4, 5}});
    pinned.fabricSelfContact = StructureFabricContactDefinition{0.01, 0.0, 0.0, 0.0};
    Structure sc(pinned);
    StructureStepSettings four = settings();
    four.constraintIterations = 4;
    caught = false;
    try {
        (void)sc.step(four);
    } catch (const softwing::ContactStepError& e) {
        caught = true;
        const softwing::ContactFeatureKey& k = e.key();
        std::printf("detail contact %zu %d %zu %zu %zu %zu %zu %zu\n", k.pair, static_cast<int>(k.kind),
                    k.firstPrimitive[0], k.firstPrimitive[1], k.firstPrimitive[2], k.secondPrimitive[0],
                    k.secondPrimitive[1], k.secondPrimitive[2]);
    }
    expect(caught, "unresolvable contact throws ContactStepError");
}

}  // namespace

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "cpu";
    try {
        if (mode == "cpu") cpu_checks();
        else if (mode == "gpu") gpu_checks();
        else return 2;
    } catch (const std::exception& e) {
        std::printf("FAIL uncaught exception: %s\n", e.what());
        return 1;
    }
    return failures == 0 ? 0 : 1;
}
