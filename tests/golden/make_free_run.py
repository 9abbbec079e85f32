"""Generates tests/golden/free_run.npz: free-running FP64 trajectories of the
wing configurations, for the device's long-run parity tests.

Each case steps the FP64 oracle port (pinned bit for bit to the reference
build) on the definition permuted into the device sweep order, from rest,
with the benchmark's settings (dt 1/120 s, 1 substep, 48 iterations,
gravity, damping 0.25, 30 Pa), without ever re-synchronising to another
solver:

  full    the 40-cell x 60-chordwise wing (68,412 triangles), 600 steps;
          positions after 300 and 600 steps
  mid     an 8-cell x 20-chordwise wing, 600 steps; positions every 100
  fabric  the 40 x 60 wing with membrane-element fabric, 25 steps;
          positions after 25 steps

and, after every step, the largest distance error, the largest cable
extension, the largest membrane strain and the centre of mass.  Positions
are stored in FP32 (the tests compare at 1e-3 m).  A hash of each case's
sweep order is stored too: the tests check that the device still sweeps in
that order.

Each case also runs a second time with FP32 arithmetic: the restatement
with every vector result rounded to FP32 (oracle.RecentredF32), in the
frame the device keeps (FP32 offsets from an FP64 origin that follows the
pilot on a 1/256 m grid).  How far that run ends from the FP64 run measures
how far FP32 arithmetic of the reference algorithm itself drifts over the
free run.  Stored per case: the largest deviation of the fabric (triangle)
nodes and of the other (line) nodes from the FP64 shape at the position
steps (each relative to its centre of mass), and the largest differences
of the two norms and of the centre of mass over all steps.

    python tests/golden/make_free_run.py       (about 15 minutes, 6 cores)
"""
import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "free_run.npz")

# name: (generator overrides, steps, steps at which positions are kept)
CASES = {
    "full": ({}, 600, (300, 600)),
    "mid": ({"cells": 8, "chordwise": 20, "spanwise_per_cell": 2, "rib_layers": 3}, 600,
            (100, 200, 300, 400, 500, 600)),
    "fabric": ({"fabric": 1}, 25, (25,)),
}


def order_hash(*orders):
    h = hashlib.sha256()
    for o in orders:
        h.update(np.ascontiguousarray(o, dtype=np.uint64).tobytes())
    return h.hexdigest()


def run_case(job):
    """One run of a case, FP64 or FP32 (see above).  Returns the per-step
    diagnostics (centre of mass in world coordinates) and the positions at
    the position steps."""
    name, kind = job
    import simwing_b200 as sw
    from oracle import oracle as O

    kw, steps, keep = CASES[name]
    d = sw.generate_wing(**kw)
    _, do, ho = sw.plan_schedule(d)
    orders = [do, ho]
    if d.view.membrane_count:
        orders.append(sw.plan_membrane_order(d))
    od = d.permuted(*orders)
    st = sw.StepSettings(time_step=1.0 / 120.0, substeps=1, constraint_iterations=48, gravity=(0.0, 0.0, -9.81),
                         velocity_damping=0.25)
    orc = O.PortStructure(od) if kind == "fp64" else O.RecentredF32(od)
    positions, diag = {}, []
    t0 = time.time()
    for k in range(1, steps + 1):
        g = orc.step(st)
        diag.append((g.maximum_distance_error, g.maximum_cable_extension, g.maximum_absolute_membrane_strain,
                     g.center_of_mass.x, g.center_of_mass.y, g.center_of_mass.z))
        if k in keep:
            positions[k] = orc.positions()
    fabric = np.zeros(d.node_count, dtype=bool)
    fabric[d.triangles()["nodes"].astype(np.int64).ravel()] = True
    print(name, kind, "%.0f s" % (time.time() - t0), diag[-1][:3], flush=True)
    return {"diag": np.array(diag), "positions": positions, "order_hash": order_hash(*orders), "fabric": fabric}


def main():
    jobs = [(name, kind) for name in CASES for kind in ("fp64", "f32")]
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        runs = dict(zip(jobs, pool.map(run_case, jobs)))
    out = {}
    for name, (_, steps, keep) in CASES.items():
        a, b = runs[(name, "fp64")], runs[(name, "f32")]
        out[f"{name}_diag"] = a["diag"]
        out[f"{name}_order_hash"] = np.array(a["order_hash"])
        out[f"{name}_steps"] = np.array(steps)
        out[f"{name}_fabric"] = a["fabric"]
        shape_fabric, shape_lines = [], []
        for k in keep:
            out[f"{name}_x{k}"] = a["positions"][k].astype(np.float32)
            dev = np.abs((b["positions"][k] - b["diag"][k - 1, 3:6]) -
                         (a["positions"][k] - a["diag"][k - 1, 3:6])).max(axis=1)
            shape_fabric.append(float(dev[a["fabric"]].max()))
            shape_lines.append(float(dev[~a["fabric"]].max()) if (~a["fabric"]).any() else 0.0)
        out[f"{name}_f32_shape_fabric"] = np.array(shape_fabric)
        out[f"{name}_f32_shape_lines"] = np.array(shape_lines)
        out[f"{name}_f32_norms"] = np.array(float(np.abs(b["diag"][:, :2] - a["diag"][:, :2]).max()))
        out[f"{name}_f32_com"] = np.array(float(np.abs(b["diag"][:, 3:6] - a["diag"][:, 3:6]).max()))
        out[f"{name}_f32_strain"] = np.array(float(np.max(np.abs(b["diag"][:, 2] - a["diag"][:, 2]) /
                                                         np.maximum(a["diag"][:, 2], 1e-300))))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, {k: out[k] for k in out if "_f32_" in k})


if __name__ == "__main__":
    main()
