"""Benchmark: wing steps/s of the plain XPBD structure step on one B200.

Workload (per rank): the synthetic ram-air wing -- 40 cells, 60 chordwise,
about 67k triangles, about 39k nodes, 121k distance-like constraints, 99k
dihedrals, 2 risers to a 90 kg rigid pilot -- stepped at dt = 1/120 s with
1 substep and 48 constraint iterations, 30 Pa outward pressure and gravity.
One step = one `swb_structure_step`.  Inputs are synthetic (seeded
generator); the reference's wing meshes are not shipped.

  value   device steps/s: CUDA events on the solver stream around each step
          (state resident in device memory), L2 flushed before every timed
          step with a 256 MiB write;
  e2e     the same through the public C-ABI with host buffers: every step
          uploads that step's external forces from host memory
          (swb_structure_set_external_forces) and reads the step's
          diagnostics back (swb_structure_step with a diagnostics output);
  roofline  algorithmic bytes per step (the per-visit byte model:
          S*[144 N + 52 T + I*(88 E_d + 160 E_b + 52 E_s) + 4 (E_d + E_b)])
          over the device time per step, against the measured HBM copy
          bandwidth; `traffic` is the DRAM bytes per launch of the committed
          ncu capture of this workload (profiles/), not measured in the run;
  cpu_baseline  the reference Structure::step (oracle/_ref, serial) on a
          bounded sample of the same workload, timed on this host.

`--impl reference` times the reference CPU solver alone (all physical
cores through its own worker pool) and prints its line.
Multi-GPU: replicas only -- each rank steps its own wing; value is the sum
of steps/s over ranks (max time over ranks).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "wing steps/s (70k tri, 48 it) plain vs batched; adjoint/forward time ratio"
UNIT = "wing-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--e2e-steps", type=int, default=100)
    p.add_argument("--cpu-sample-steps", type=int, default=12)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--batch-size", type=int, default=64)
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-batched-adjoint", action="store_true")
    p.add_argument("--no-membrane-wing", action="store_true")
    p.add_argument("--no-contact", action="store_true")
    p.add_argument("--no-coupling", action="store_true")
    p.add_argument("--only-adjoint", action="store_true",
                   help="run the adjoint leg alone and print its record (profiling)")
    p.add_argument("--only-contact", action="store_true",
                   help="run the fabric self-contact leg alone and print its record (profiling)")
    p.add_argument("--adjoint-steps", type=int, default=240)
    p.add_argument("--adjoint-interval", type=int, default=16)
    return p.parse_args()


def max_over_ranks(value, dist, device):
    """Largest `value` over the ranks of the process group (`value` itself
    without one).  Every rank calls it at the same point."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, seconds):
    """Whole-job rate of `world` independent replicas that each processed
    `units_per_rank` units, over the slowest rank's time."""
    return world * units_per_rank / seconds


def wing_config():
    return {"workload": "plain ram-air wing, 40 cells x 60 chordwise (68,412 tri, 39,155 nodes), 48 iterations, 1 substep, "
                        "dt 1/120 s, 30 Pa + gravity, rigid pilot on 2 risers",
            "cells": 40, "chordwise": 60, "iterations": 48, "substeps": 1,
            "l2": "flushed before every timed step (256 MiB write)"}


def settings(sw=None):
    """The workload's step settings (dt 1/120 s, 1 substep, 48 iterations,
    gravity, damping 0.25; no cable sweep pairs, serial), filled in plain
    ctypes so that the reference arm needs no product library."""
    from simwing_b200 import abi

    s = abi.StepSettings()
    s.time_step = 1.0 / 120.0
    s.substeps = 1
    s.constraint_iterations = 48
    s.gravity = abi.Vec3(0.0, 0.0, -9.81)
    s.velocity_damping = 0.25
    return s


def algorithmic_bytes(definition, iterations=48, substeps=1):
    """Per step: S*[144 N + 52 T + I*(88 E_d + 160 E_b + 236 E_m + 52 E_s) + 4 (E_d + E_b) + 12 E_m]."""
    v = definition.view
    n, t = v.node_count, v.triangle_count
    e_d, e_b, e_m = v.constraint_count, v.dihedral_count, v.membrane_count
    e_s = v.suspension.contents.segment_count if v.suspension else 0
    return substeps * (144 * n + 52 * t + iterations * (88 * e_d + 160 * e_b + 236 * e_m + 52 * e_s)
                       + 4 * (e_d + e_b) + 12 * e_m)


def membrane_wing_leg(sw, st, steps, device, flush):
    """The same wing with its fabric as the reference's scene assembly builds
    it: one orthotropic membrane element per skin and rib triangle (68,412)
    and no fabric edge constraints; seams, lines and pilot as before.  Device
    steps/s from CUDA events, L2 flushed before every timed step."""
    import torch

    d = sw.generate_wing(fabric=1)
    s = sw.Structure(d, sw.SolverOptions(device=device))
    for _ in range(5):
        s.step(st, diagnostics=False)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        s.step(st, diagnostics=False)
        times.append(s.last_step_ms())
    diag = s.diagnostics()
    rep = s.schedule_report()
    s.close()
    total = float(sum(times))
    return {"workload": "ram-air wing, 40 cells x 60 chordwise, fabric as membrane elements (68,412), 48 iterations",
            "membranes": d.counts()["membranes"], "constraints": d.counts()["constraints"],
            "stages_per_iteration": rep.local_stages_per_iteration, "steps": steps,
            "ms_per_step": total / steps, "wing_steps_per_s": steps / (total / 1000.0),
            "max_membrane_strain": diag.maximum_absolute_membrane_strain, "finite": bool(diag.finite)}


def contact_leg(sw, steps, device, reference_steps, with_reference):
    """Fabric self-contact: two stacked sheets, the free one 1 mm inside the
    contact envelope of the pinned one, compliant contact (1e-3 m/N) with
    friction, 8 iterations, tilted gravity.  16 x 16 (512 nodes, 900
    triangles): one step from the same initial state, repeated (the state
    is restored between steps), the reference build's Structure timed on
    the host beside it.  80 x 80 (12,800 nodes, 24,964 triangles, the
    contact configuration's size): the first step from rest (restored and
    repeated) and the steps that follow it, consecutive, until the swept
    query gives up on the persistent resting contact (as the reference's
    does after a few steps) or four steps.  Device time from CUDA events."""
    st = sw.StepSettings(time_step=1.0 / 120.0, substeps=1, constraint_iterations=8, gravity=(2.0, 0.0, -9.81),
                         velocity_damping=0.25)

    def first_step(s, repeats):
        image = s.checkpoint()
        for _ in range(2):
            s.step(st, diagnostics=False)
            s.restore(image)
        times = []
        for _ in range(repeats):
            s.step(st, diagnostics=False)
            times.append(s.last_step_ms())
            s.restore(image)
        return float(sum(times)) / len(times)

    d = sw.stacked_sheets(n=16, compliance=1e-3)
    s = sw.Structure(d, sw.SolverOptions(device=device))
    first = first_step(s, steps)
    diag = s.step(st)
    s.close()
    out = {"workload": "stacked 16x16 sheets, compliant fabric self-contact with friction, 8 iterations, "
                       "one step from rest", "nodes": d.counts()["nodes"], "triangles": d.counts()["triangles"],
           "active_contacts": int(diag.active_contact_count), "steps": steps, "device_ms_per_step": first}
    big = sw.stacked_sheets(n=80, compliance=1e-3)
    s = sw.Structure(big, sw.SolverOptions(device=device))
    first = first_step(s, 3)
    consecutive = []
    try:
        s.step(st, diagnostics=False)
        for _ in range(3):
            s.step(st, diagnostics=False)
            consecutive.append(s.last_step_ms())
    except sw.ContactStepError:
        pass
    s.close()
    out["sheets_80x80"] = {"triangles": big.counts()["triangles"], "nodes": big.counts()["nodes"],
                           "first_step_ms": first, "consecutive_steps": len(consecutive),
                           "consecutive_ms_per_step": float(sum(consecutive)) / len(consecutive) if consecutive
                           else None}
    if with_reference:
        from oracle import oracle as O

        if O.ref_available():
            ref_times = []
            for _ in range(reference_steps):
                ref = O.RefStructure(d)
                ref.step(st)
                ref_times.append(ref.last_step_seconds() * 1000.0)
            out["reference_ms_per_step"] = float(sum(ref_times)) / len(ref_times)
            out["reference_cores"] = 1
    return out


def coupling_leg(sw, st, steps, device):
    """A macro-step of the coupling caller (ConservativeMacroStepCoupling::
    advanceStructure) on the wing, one interface node per structure node:
    the interface impulses handed over from device memory
    (swb_coupling_advance_impulses) against the same loads handed over from
    host memory (set_external_forces, then step).  Wall-clock time per
    macro-step, each call synchronised."""
    import time

    import numpy as np
    import torch

    d = sw.generate_wing()
    n = d.view.node_count
    rng = np.random.default_rng(11)
    impulses = rng.normal(scale=1e-4, size=(n, 3))
    forces = impulses * (1.0 / st.time_step)
    d_impulses = torch.tensor(impulses, dtype=torch.float64, device=f"cuda:{device}")
    out = {"workload": "ram-air wing, 39,155 interface nodes bound one to one, 48 iterations", "steps": steps}
    s = sw.Structure(d, sw.SolverOptions(device=device))
    coupling = sw.Coupling(s, np.arange(n, dtype=np.uint64))
    for _ in range(3):
        coupling.advance_impulses(d_impulses, st.time_step, st)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        coupling.advance_impulses(d_impulses, st.time_step, st)
    out["device_loads_ms_per_step"] = (time.perf_counter() - t) * 1000.0 / steps
    coupling.close()
    s.close()
    s = sw.Structure(d, sw.SolverOptions(device=device))
    for _ in range(3):
        s.set_external_forces(forces)
        s.step(st)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        s.set_external_forces(forces)
        s.step(st)
    out["host_loads_ms_per_step"] = (time.perf_counter() - t) * 1000.0 / steps
    s.close()
    return out


def batched_leg(sw, st, count, rank, world, dist, device):
    """Batched wings: `count` structures of uneven sizes in one packed
    launch per step, 120-step CUDA-graph blocks; against the same wings
    solved one after another by the plain solver."""
    import concurrent.futures as cf

    import torch

    defs = sw.generate_wing_batch(count, seed=2024)
    tris = [d.counts()["triangles"] for d in defs]
    batch = sw.Batch(defs, sw.BatchOptions(device=device, flags=sw.abi.BATCH_AUTOTUNE))
    rep = batch.report()
    block = 120
    batch.step(st, block)  # warm-up block (captures the graph)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    batch.step(st, block)
    ms = max_over_ranks(batch.last_step_ms(), dist, f"cuda:{device}")
    ms_per_step = ms / block
    out = {"workload": f"{count} wings, cells U{{20..60}}, chordwise {{30,45,60}}, aspect ratio U(4.5,7), "
                       "compliance x lognormal(0,0.2), seed 2024; 48 iterations, 1 substep",
           "structures": count, "triangles_min": min(tris), "triangles_max": max(tris),
           "triangles_total": sum(tris), "graph_steps": block, "launches_per_step": 1,
           "ms_per_step": ms_per_step, "wing_steps_per_s": replica_rate(count, world, ms_per_step / 1000.0),
           "target_patch_nodes": rep.target_patch_nodes, "clusters": rep.clusters,
           "cluster_ctas": rep.cluster_ctas, "resident_clusters": rep.resident_clusters,
           "block_threads": rep.block_threads,
           "autotune_ms_per_step": {f"patch {rep.candidate_patch_nodes[k]}, "
                                    f"{rep.candidate_block_threads[k] or 'widest-stage'} threads":
                                    rep.candidate_ms_per_step[k] for k in range(rep.autotune_candidates)}}
    batch.close()
    if rank == 0:
        # the same wings, one plain structure after another
        opts = sw.SolverOptions(device=device)
        with cf.ThreadPoolExecutor(8) as pool:
            plains = list(pool.map(lambda d: sw.Structure(d, opts), defs))
        total = 0.0
        for s in plains:
            for _ in range(2):
                s.step(st, diagnostics=False)
            times = []
            for _ in range(3):
                s.step(st, diagnostics=False)
                times.append(s.last_step_ms())
            total += min(times)
            s.close()
        out["sequential_plain_ms_per_step"] = total / count
        out["sequential_plain_wing_steps_per_s"] = count / (total / 1000.0)
        out["speedup_vs_sequential"] = out["wing_steps_per_s"] / world / out["sequential_plain_wing_steps_per_s"]
    return out


def adjoint_leg(sw, st, device, steps=240, interval=16):
    """Adjoint calibration workload: the wing generator at 20 cells x 30
    chordwise with two line attachments per cell and row (13,338 triangles,
    266 line rest lengths), settled for 60 steps; the target is the shape after `steps`
    (240) steps with every line's rest length scaled by lognormal(0, 0.02);
    the loss is the mean squared distance of the fabric (triangle) nodes to
    it; one gradient = a forward of `steps` steps with a checkpoint every
    `interval` (16) steps plus the backward (segment recompute with tape +
    reverse sweep).  Launches: 60 settle and `steps` target steps, then two
    repetitions of `steps` forward, `steps` taping and `steps` reverse."""
    import numpy as np

    d = sw.generate_calibration_wing()
    opts = sw.SolverOptions(device=device)
    s = sw.Structure(d, opts)
    for _ in range(60):
        s.step(st, diagnostics=False)
    state = s.node_states()
    pilot = s.suspension_state()
    # target: perturbed line rest lengths from the same state
    rng = np.random.default_rng(2024)
    perturbed = d.copy()
    lines = sw.line_groups(d)
    rest = perturbed.constraints()["rest_length"]
    for g in lines:
        rest[g] *= float(np.exp(rng.normal(0.0, 0.02)))
    t = sw.Structure(perturbed, opts)
    t.write_node_states(state)
    t.write_payload_state(pilot.center_of_mass, pilot.body_to_world, pilot.linear_velocity, pilot.angular_velocity)
    for _ in range(steps):
        t.step(st, diagnostics=False)
    target = t.positions()
    t.close()
    weights = np.zeros(s.node_count)
    weights[d.triangles()["nodes"].astype(np.int64).ravel()] = 1.0
    r = sw.Rollout(s, steps, interval)
    r.forward(st, target, weights)
    r.backward()  # warm-up (allocates the tapes)
    loss = r.forward(st, target, weights)
    g = r.backward()
    fwd, bwd = r.forward_ms(), r.backward_ms()
    cons = d.constraints()
    line_grad = [float(np.sum(g["d_rest"][x] * cons["rest_length"][x]) / np.sum(cons["rest_length"][x])) for x in lines]
    counts = d.counts()
    out = {"workload": f"wing 20 cells x 30 chordwise, 2 line attachments per cell, settled 60 steps; {steps}-step rollout, checkpoint every "
                       f"{interval} steps; "
                       "target from line rest lengths x lognormal(0, 0.02); loss = mean squared distance of the "
                       "fabric nodes",
           "triangles": counts["triangles"], "nodes": counts["nodes"], "steps": steps, "checkpoint_interval": interval,
           "parameters": {"line_rest_lengths": len(lines), "compliance_classes": 3,
                          "riser_rest_lengths": int(counts["suspension_segments"]), "pilot_mass": 1},
           "loss": loss, "forward_ms": fwd, "backward_ms": bwd,
           "backward_over_forward": bwd / fwd, "gradient_over_forward": (fwd + bwd) / fwd,
           "gradient_norm_lines": float(np.linalg.norm(line_grad)), "d_pilot_mass": g["d_mass"],
           "d_riser_rest": [float(v) for v in g["d_segment_rest"]]}
    r.close()
    s.close()
    return out


# line-line contact of the batched adjoint workload: 1 mm line radius, 2 mm
# margin (candidates within 4 mm of each other by box)
LINE_RADIUS, LINE_MARGIN = 0.001, 0.002


def batched_adjoint_leg(sw, st, device, wings=32, steps=240, interval=16, group=16):
    """Batched adjoint with contact: `wings` (32) wings of cells ~ U{30..50}
    x 45 chordwise (about 20-35k triangles), each with its line rest
    lengths scaled by lognormal(0, 0.03) from its own seed, settled 20
    steps, against a frictionless contact plane: the ground plane's
    projection with a horizontal normal, standing 1 cm inside the wing's
    trailing edge, so that the trailing edge slides along it while the wing
    falls (a plane under the pilot would let the falling pilot through, as
    the plane holds nodes only, and the stretched lines would fail the
    suspension's residual bound), with line-line contact of the cascaded
    lines' cable segments (LINE_RADIUS, LINE_MARGIN); per wing a `steps`-step rollout with a checkpoint every
    `interval` steps, forward plus backward, the loss the mean squared
    distance of the fabric nodes to their settled positions.  The rollouts
    run side by side, `group` at a time (swb_rollout_forward_many and
    swb_rollout_backward_many); the time is the host's around those calls,
    tape allocation of the first backward included."""
    import time

    import numpy as np

    rng = np.random.default_rng(2025)
    specs = [dict(cells=int(rng.integers(30, 51)), chordwise=45, seed=7000 + i) for i in range(wings)]
    opts = sw.SolverOptions(device=device)
    total_fwd = total_bwd = 0.0
    tri, hits, overflowed, failed = [], 0, 0, 0
    for start in range(0, wings, group):
        structures, rollouts, targets, weights = [], [], [], []
        for spec in specs[start:start + group]:
            d = sw.generate_wing(**spec)
            tri.append(int(d.counts()["triangles"]))
            wrng = np.random.default_rng(spec["seed"])
            rest = d.constraints()["rest_length"]
            for g in sw.line_groups(d):
                rest[g] *= float(np.exp(wrng.normal(0.0, 0.03)))
            s = sw.Structure(d, opts)
            for _ in range(20):
                s.step(st, diagnostics=False)
            x_max = float(s.positions()[:, 0].max())
            s.set_ground((-1.0, 0.0, 0.0), -(x_max - 0.01), 0.0)
            s.set_line_contact(LINE_RADIUS, LINE_MARGIN)
            w = np.zeros(s.node_count)
            w[d.triangles()["nodes"].astype(np.int64).ravel()] = 1.0
            structures.append(s)
            targets.append(s.positions())
            weights.append(w)
            rollouts.append(sw.Rollout(s, steps, interval))
        t0 = time.perf_counter()
        sw.rollout_forward_many(rollouts, st, targets, weights)
        t1 = time.perf_counter()
        statuses = np.zeros(len(rollouts), dtype=np.int32)
        sw.rollout_backward_many(rollouts, statuses)
        t2 = time.perf_counter()
        total_fwd += t1 - t0
        total_bwd += t2 - t1
        hits += int((statuses == sw.abi.OK).sum())
        failed += int(((statuses != sw.abi.OK) & (statuses != sw.abi.NON_FINITE)).sum())
        overflowed += int((statuses == sw.abi.NON_FINITE).sum())
        for r in rollouts:
            r.close()
        for s in structures:
            s.close()
    return {"workload": f"{wings} wings, cells U{{30..50}} x 45 chordwise, line rest lengths x lognormal(0, 0.03), "
                        f"frictionless contact plane 1 cm inside each trailing edge, line-line contact "
                        f"({LINE_RADIUS * 1000:g} mm radius, {LINE_MARGIN * 1000:g} mm margin); {steps}-step rollout forward + backward "
                        f"per wing, checkpoint every {interval} steps, {group} rollouts side by side",
            "wings": wings, "triangles_min": min(tri), "triangles_max": max(tri), "steps": steps,
            "forward_s": total_fwd, "backward_s": total_bwd,
            "wing_gradients_per_s": wings / (total_fwd + total_bwd), "finite_gradients": hits,
            "overflowed_gradients": overflowed,
            "overflow_note": "SWB_NON_FINITE: the free-falling wing's tip trailing edge flutters, and the rollout's "
                             "sensitivity outgrows FP32 in the reverse sweep (the FP64 adjoint along the same device "
                             "trajectory reaches 3.5e19 after 48 steps on such a wing)",
            "line_line_contact": {"radius_m": LINE_RADIUS, "margin_m": LINE_MARGIN},
            "backward_failures": failed}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "xpbd_cluster_kernel_wing70k.md")
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index):
        self.device = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_run(definition, steps, threads):
    """Reference Structure::step on this host (oracle/_ref when built,
    otherwise the C restatement)."""
    from oracle import oracle as O

    st = settings()
    st.worker_threads = threads
    if O.ref_available():
        ref = O.RefStructure(definition)
        kind = "reference"
    else:
        ref = O.PortStructure(definition)
        kind = "port"
        threads = 1
    ref.step(st)  # warm caches
    t0 = time.perf_counter()
    for _ in range(steps):
        ref.step(st)
    dt = time.perf_counter() - t0
    return steps / dt, kind, threads


def physical_cores():
    from oracle import oracle as O

    if O.ref_available():
        return int(O.ref_library().swref_physical_cores())
    return os.cpu_count() or 1


def run_reference_arm(args):
    """The reference's own CPU step (oracle/_ref: src/softwing + src/fsi
    compiled from source) on this host's cores, through Structure::step with
    workerThreads = physical cores; each timed step is one wing step of the
    same workload.  Rank 0 alone runs under torchrun."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import tempfile

    from oracle import definition_file

    # The wing comes from the product's generator, run in a child process
    # that writes it to a file: this process maps only the reference build.
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "wing.npz")
        subprocess.run([sys.executable, "-c",
                        "import sys; sys.path.insert(0, sys.argv[1]); import simwing_b200 as sw; "
                        "from oracle import definition_file as F; F.save(sw.generate_wing(), sys.argv[2])",
                        ROOT, path], check=True)
        definition = definition_file.FileDefinition(path)
    cores = physical_cores()
    sample = max(1, min(args.steps, 8))
    value, kind, used = cpu_reference_run(definition, sample, cores)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": sample,
            "warmup": 1, "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": wing_config(),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind,
                             "sample": f"{sample} wing steps (workerThreads={used})"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)

    import numpy as np
    import torch

    import simwing_b200 as sw

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    if args.warmup < 3:
        raise SystemExit("warmup must be >= 3")
    if args.only_contact:
        if rank == 0:
            print(json.dumps({"contact": contact_leg(sw, args.steps, local, 1, False)}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    if args.only_adjoint:
        if rank == 0:
            print(json.dumps({"adjoint": adjoint_leg(sw, settings(sw), local, args.adjoint_steps,
                                                     args.adjoint_interval)}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    definition = sw.generate_wing()
    st = settings(sw)
    # the autotuner picks block size, split stages and cluster width at
    # creation (trial substeps that leave the state untouched)
    structure = sw.Structure(definition, sw.SolverOptions(device=local, flags=sw.abi.OPT_AUTOTUNE))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    # warm-up
    for _ in range(args.warmup):
        structure.step(st, diagnostics=False)
    torch.cuda.synchronize()

    # device-timed region: per-step CUDA events inside the library (solver
    # stream), L2 flush between steps (outside the events)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            structure.step(st, diagnostics=False)
            times.append(structure.last_step_ms())
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(times), dist, f"cuda:{local}")
    if dist is not None:
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = replica_rate(args.steps, world, total_ms / 1000.0)

    # end-to-end through the C-ABI with host buffers
    rng = np.random.default_rng(5)
    forces = rng.normal(0.0, 1e-4, size=(structure.node_count, 3))
    e2e_steps = max(3, args.e2e_steps)
    for _ in range(3):
        structure.set_external_forces(forces)
        structure.step(st, diagnostics=True)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        structure.set_external_forces(forces)
        diag = structure.step(st, diagnostics=True)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    e2e_value = replica_rate(e2e_steps, world, e2e_s)
    h2d = structure.node_count * 16
    d2h = 148 * 16 * 8 + 16 + 128  # diagnostics partials + control word + payload

    bytes_per_step = algorithmic_bytes(definition)
    peak, peak_kind = measured_peak()
    achieved = bytes_per_step / (ms_per_step / 1000.0) / 1e9
    report = structure.schedule_report()

    batched = None
    if not args.no_batched:
        batched = batched_leg(sw, st, args.batch_size, rank, world, dist, local)

    adjoint = None
    if not args.no_adjoint and rank == 0:
        adjoint = adjoint_leg(sw, st, local, args.adjoint_steps, args.adjoint_interval)
    batched_adjoint = None
    if not args.no_batched_adjoint and rank == 0:
        batched_adjoint = batched_adjoint_leg(sw, st, local)

    membrane_wing = None
    if not args.no_membrane_wing and rank == 0:
        membrane_wing = membrane_wing_leg(sw, st, min(args.steps, 50), local, flush)
    coupling = None
    if not args.no_coupling and rank == 0:
        coupling = coupling_leg(sw, st, min(args.steps, 50), local)
    contact = None
    if not args.no_contact and rank == 0:
        contact = contact_leg(sw, min(args.steps, 50), local, 2, not args.no_cpu_baseline)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu_value, kind, used = cpu_reference_run(definition, args.cpu_sample_steps, 0)
        cpu = {"value": cpu_value, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"{args.cpu_sample_steps} wing steps, serial (workerThreads=0)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": wing_config(),
            "parallelism": "replicas" if world > 1 else "single",
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(),
                         "peak_source": peak_kind, "algorithmic_bytes_per_step": bytes_per_step},
            "clocks": clocks.summary(),
            "schedule": {"blocks": report.blocks, "threads": report.block_threads,
                         "cluster_ctas": report.cluster_ctas,
                         "cluster_barriers_per_iteration": report.cluster_barriers_per_iteration,
                         "stages_per_iteration": report.local_stages_per_iteration,
                         "shared_bytes": report.shared_bytes,
                         "autotune": structure.autotune_report()},
            "final_diagnostics": {"finite": bool(diag.finite), "max_distance_error": diag.maximum_distance_error},
            "batched": batched,
            "adjoint": adjoint,
            "batched_adjoint": batched_adjoint,
            "membrane_wing": membrane_wing,
            "contact": contact,
            "coupling": coupling,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    structure.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
