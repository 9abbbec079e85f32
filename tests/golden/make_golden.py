"""Generates tests/golden/*.npz from the reference's own solver.

Runs only where the reference build exists (oracle/_ref/libswref.so, made
by `make -C oracle ref` from the reference sources).  The fixtures hold
FP64 positions after a fixed number of steps of three small seeded
definitions (a cloth patch, a wing with pilot, a patch of membrane
elements), the reference colouring of their constraint lists, and the
reference definition fingerprints; tests compare the oracle port and the
device solver against them without needing the reference at run time.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import simwing_b200 as sw  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def settings():
    return sw.StepSettings(time_step=1.0 / 120.0, substeps=1, constraint_iterations=48, gravity=(0, 0, -9.81),
                           velocity_damping=0.25)


def main():
    if not O.ref_available():
        raise SystemExit("reference build missing: run `make -C oracle ref` first")
    cases = {
        "patch": (sw.generate_patch(nx=17, ny=17, seed=7), 20),
        "wing": (sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=3), 5),
        "membrane_patch": (sw.generate_patch(nx=12, ny=12, seed=9, membranes=2), 10),
    }
    out = {}
    for name, (d, steps) in cases.items():
        ref = O.RefStructure(d)
        for _ in range(steps):
            ref.step(settings())
        out[f"{name}_steps"] = np.array(steps)
        out[f"{name}_positions"] = ref.positions()
        out[f"{name}_fingerprint"] = np.array(ref.fingerprint(), dtype=np.uint64)
        order, offsets, parallel = O.ref_colouring(d)
        out[f"{name}_colour_order"] = order
        out[f"{name}_colour_offsets"] = offsets
        out[f"{name}_parallel_colours"] = np.array(parallel)
    np.savez_compressed(os.path.join(OUT, "trajectories.npz"), **out)
    print("wrote", os.path.join(OUT, "trajectories.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
