"""Generates tests/golden/calibration.npz: the FP64 reference of the adjoint
calibration workload (the rollout gradient of the calibration wing).

The calibration wing (simwing_b200.CALIBRATION_WING: 20 cells x 30
chordwise, 13,338 triangles, 266 line rest lengths) is settled for 60 steps
from rest by the FP64 oracle port on the definition permuted into the device
sweep order.  From that state the target is the fabric's shape after 240
steps with every line's rest length scaled by lognormal(0, 0.02); the loss
is the mean squared distance of the fabric (triangle) nodes to it after a
240-step rollout of the unperturbed wing.  The fixture holds:

  * the settled state and pilot state, the target;
  * the FP64 reference gradient (oracle/libadjoint.so) of the loss with
    respect to the calibration parameters -- each line's rest length (its
    cables scaled together, per unit length), the scale of each compliance
    class (distance, cable, dihedral), the riser rest lengths and the pilot
    mass -- and the loss;
  * central finite differences (h = 1e-4, relative) of the FP64 loss for a
    sample of those parameters, and the same with h = 1e-6: where the two
    differ, a line cable crosses its slack/taut switch within +-1e-4 along
    the rollout, and the wide difference is no derivative;
  * the loss of the same rollout with FP32 arithmetic (the restatement with
    every vector result rounded to FP32, in the device's frame:
    oracle.RecentredF32), which shows how far FP32 arithmetic of the
    reference algorithm moves the loss over the rollout;
  * a hash of the device sweep order the FP64 runs used (the test checks
    that the device still sweeps in that order).

    python tests/golden/make_calibration.py      (about 15 minutes, 8 cores)
"""
import hashlib
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "calibration.npz")
SETTLE, STEPS, H, H_FINE = 60, 240, 1e-4, 1e-6


def settings():
    import simwing_b200 as sw

    return sw.StepSettings(time_step=1.0 / 120.0, substeps=1, constraint_iterations=48, gravity=(0, 0, -9.81),
                           velocity_damping=0.25)


def order_hash(distance_order, dihedral_order):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(distance_order, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(dihedral_order, dtype=np.uint64).tobytes())
    return h.hexdigest()


def weights_of(definition):
    w = np.zeros(definition.node_count)
    w[definition.triangles()["nodes"].astype(np.int64).ravel()] = 1.0
    return w


def perturbed(definition, kind, index, factor, lines):
    """A copy with one calibration parameter scaled by `factor`."""
    from simwing_b200 import abi

    d = definition.copy()
    cons = d.constraints()
    if kind == "line":
        cons["rest_length"][lines[index]] *= factor
    elif kind == "class":
        if index == 2:
            d.dihedrals()["compliance"][:] *= factor
        else:
            mask = (cons["kind"] == abi.CABLE) if index == 1 else \
                ((cons["kind"] == abi.DISTANCE) | (cons["kind"] == abi.SUSPENSION_TIE))
            cons["compliance"][mask] *= factor
    elif kind == "riser":
        d.view.suspension.contents.segments[index].rest_length *= factor
    elif kind == "mass":
        d.view.suspension.contents.pilot_mass *= factor
    return d


def rollout_loss(args):
    """FP64 loss of the rollout of one perturbed definition (pool worker):
    the oracle port's forward, which the reference gradient's forward equals
    bit for bit."""
    kind, index, factor = args
    import simwing_b200 as sw
    from oracle import oracle as O

    d = sw.generate_calibration_wing()
    _, do, ho = sw.plan_schedule(d)
    data = np.load(OUT + ".partial.npz")
    orc = O.PortStructure(perturbed(d, kind, index, factor, sw.line_groups(d)).permuted(do, ho))
    orc.write_node_states(data["state"])
    orc.write_payload(payload_struct(data["payload"]))
    for _ in range(STEPS):
        orc.step(settings())
    x = orc.positions()
    w = weights_of(d)
    return float(np.sum(w[:, None] * (x - data["target"]) ** 2) / np.sum(w))


def f32_loss(_):
    """The loss of the rollout with FP32 arithmetic (pool worker)."""
    import simwing_b200 as sw
    from oracle import oracle as O

    d = sw.generate_calibration_wing()
    _, do, ho = sw.plan_schedule(d)
    data = np.load(OUT + ".partial.npz")
    orc = O.RecentredF32(d.permuted(do, ho))
    orc.write_state(data["state"], payload_struct(data["payload"]))
    for _ in range(STEPS):
        orc.step(settings())
    x = orc.positions()
    w = weights_of(d)
    return float(np.sum(w[:, None] * (x - data["target"]) ** 2) / np.sum(w))


def payload_struct(v):
    from simwing_b200 import abi

    return abi.PayloadState(abi.Vec3(*v[0:3]), abi.Quat(*v[3:7]), abi.Vec3(*v[7:10]), abi.Vec3(*v[10:13]))


def payload_vector(p):
    c, q, lv, av = p.center_of_mass, p.body_to_world, p.linear_velocity, p.angular_velocity
    return np.array([c.x, c.y, c.z, q.w, q.x, q.y, q.z, lv.x, lv.y, lv.z, av.x, av.y, av.z])


def main():
    import simwing_b200 as sw
    from simwing_b200 import abi
    from oracle import oracle as O

    d = sw.generate_calibration_wing()
    _, do, ho = sw.plan_schedule(d)
    od = d.permuted(do, ho)
    st = settings()
    lines = sw.line_groups(d)
    # settle from rest
    orc = O.PortStructure(od)
    for _ in range(SETTLE):
        orc.step(st)
    state = orc.node_states()
    payload = payload_vector(orc.payload()[0])
    # target: perturbed line rest lengths, same start
    rng = np.random.default_rng(2024)
    pd = d.copy()
    rest = pd.constraints()["rest_length"]
    for g in lines:
        rest[g] *= float(np.exp(rng.normal(0.0, 0.02)))
    t = O.PortStructure(pd.permuted(do, ho))
    t.write_node_states(state)
    t.write_payload(payload_struct(payload))
    for _ in range(STEPS):
        t.step(st)
    target = t.positions()
    np.savez(OUT + ".partial.npz", state=state, payload=payload, target=target)
    # FP64 reference gradient along its own trajectory
    w = weights_of(d)
    ref = O.rollout_gradient(od, st, STEPS, target, w, state=state, payload=payload)
    d_rest = np.zeros_like(ref["d_rest"])
    d_rest[do] = ref["d_rest"]
    d_comp = np.zeros_like(ref["d_comp"])
    d_comp[do] = ref["d_comp"]
    d_dih = np.zeros_like(ref["d_dihedral_comp"])
    d_dih[ho] = ref["d_dihedral_comp"]
    cons = d.constraints()
    kinds, rest0, comp0 = cons["kind"], cons["rest_length"], cons["compliance"]
    grad_lines = np.array([np.sum(d_rest[g] * rest0[g]) / np.sum(rest0[g]) for g in lines])
    grad_classes = np.array([np.sum((d_comp * comp0)[(kinds == abi.DISTANCE) | (kinds == abi.SUSPENSION_TIE)]),
                             np.sum((d_comp * comp0)[kinds == abi.CABLE]),
                             np.sum(d_dih * d.dihedrals()["compliance"])])
    segs = d.view.suspension.contents
    seg_rest = np.array([segs.segments[k].rest_length for k in range(segs.segment_count)])
    # central differences of the FP64 loss for a sample of the parameters
    sample = [("line", int(i)) for i in np.linspace(0, len(lines) - 1, 8).round().astype(int)]
    sample += [("class", 0), ("class", 1), ("class", 2), ("riser", 0), ("riser", 1), ("mass", 0)]
    jobs = [(k, i, f) for k, i in sample for f in (1.0 + H, 1.0 - H, 1.0 + H_FINE, 1.0 - H_FINE)]
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        f32 = pool.map_async(f32_loss, [0])
        losses = pool.map(rollout_loss, jobs)
        loss_f32 = f32.get()[0]
    fd, fd_fine = [], []
    for n, (kind, index) in enumerate(sample):
        scale = 1.0
        if kind == "line":
            scale = float(np.sum(rest0[lines[index]]))       # per unit length of the line, as grad_lines
        elif kind == "riser":
            scale = seg_rest[index]
        elif kind == "mass":
            scale = segs.pilot_mass
        fd.append((losses[4 * n] - losses[4 * n + 1]) / (2.0 * H) / scale)
        fd_fine.append((losses[4 * n + 2] - losses[4 * n + 3]) / (2.0 * H_FINE) / scale)
    np.savez_compressed(OUT, state=state, payload=payload, target=target, loss=np.array(ref["loss"]),
                        grad_lines=grad_lines, grad_classes=grad_classes,
                        grad_riser_rest=ref["d_segment_rest"][: segs.segment_count],
                        grad_pilot_mass=np.array(ref["d_mass"]),
                        fd_kind=np.array([k for k, _ in sample]), fd_index=np.array([i for _, i in sample]),
                        fd_value=np.array(fd), fd_fine_value=np.array(fd_fine), loss_f32=np.array(loss_f32),
                        final=ref["final"].astype(np.float32),
                        order_hash=np.array(order_hash(do, ho)), settle=np.array(SETTLE), steps=np.array(STEPS))
    os.remove(OUT + ".partial.npz")
    print("wrote", OUT, "loss", ref["loss"], "FP32 loss", loss_f32,
          "fd", dict(zip([f"{k}{i}" for k, i in sample], np.round(fd, 8))))


if __name__ == "__main__":
    main()
