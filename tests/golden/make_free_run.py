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

    python tests/golden/make_free_run.py       (about 10 minutes)
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


def run_case(name):
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
    orc = O.PortStructure(od)
    out = {}
    diag = []
    t0 = time.time()
    for k in range(1, steps + 1):
        g = orc.step(st)
        diag.append((g.maximum_distance_error, g.maximum_cable_extension, g.maximum_absolute_membrane_strain,
                     g.center_of_mass.x, g.center_of_mass.y, g.center_of_mass.z))
        if k in keep:
            out[f"{name}_x{k}"] = orc.positions().astype(np.float32)
    out[f"{name}_diag"] = np.array(diag)
    out[f"{name}_order_hash"] = np.array(order_hash(*orders))
    out[f"{name}_steps"] = np.array(steps)
    print(name, "%.0f s" % (time.time() - t0), diag[-1][:3], flush=True)
    return out


def main():
    with mp.get_context("spawn").Pool(len(CASES)) as pool:
        parts = pool.map(run_case, list(CASES))
    out = {}
    for p in parts:
        out.update(p)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, sorted(out))


if __name__ == "__main__":
    main()
