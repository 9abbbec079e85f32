"""swb_diagnostics_noalloc: the diagnostics reduction over caller-owned
device arrays with its scratch in a static device array.  Its output is
checked against swb_structure_diagnostics (the structure's own diagnostics,
scratch allocated at creation) on the same state, on two calls in a row.

Tolerances: counts, finiteness and the maxima are computed element by
element with the same arithmetic, so they must be equal; the sums (mass,
centre of mass, momentum, kinetic energy) are FP64 sums of the same FP32
terms in a different order, so they must agree to 1e-12 relative.

This file is named so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from tests.conftest import step_settings

SUM_RTOL = 1e-12
MAX_ITEMS = 524288  # SWB_NOALLOC_MAX_NODES == SWB_NOALLOC_MAX_CONSTRAINTS


def device_arrays(structure, definition):
    """The structure's current state as the caller-owned arrays the entry
    point takes (definition order, float4 with w = inverse mass)."""
    import torch

    states = structure.node_states()  # [N, 3 (position, previous, velocity), 3]
    nodes = definition.nodes()
    with np.errstate(divide="ignore"):
        inv_mass = np.where(nodes["fixed"] != 0, 0.0, (1.0 / nodes["mass"]).astype(np.float32)).astype(np.float32)
    packed = []
    for k in range(3):
        a = np.zeros((len(states), 4), dtype=np.float32)
        a[:, :3] = states[:, k, :].astype(np.float32)
        assert np.array_equal(a[:, :3].astype(np.float64), states[:, k, :])  # exact float state
        if k == 0:
            a[:, 3] = inv_mass
        packed.append(torch.from_numpy(a).cuda())
    cons = definition.constraints()
    first = torch.from_numpy(cons["first_node"].astype(np.uint32).view(np.int32)).cuda()
    second = torch.from_numpy(cons["second_node"].astype(np.uint32).view(np.int32)).cuda()
    rest = torch.from_numpy(cons["rest_length"].astype(np.float32)).cuda()
    kind = torch.from_numpy(cons["kind"].astype(np.uint8)).cuda()
    torch.cuda.synchronize()
    return packed, (first, second, rest, kind), len(states), len(cons)


def noalloc(arrays):
    (pos, prev, vel), (first, second, rest, kind), n, m = arrays
    out = abi.Diagnostics()
    status = abi.library().swb_diagnostics_noalloc(0, pos.data_ptr(), prev.data_ptr(), vel.data_ptr(), n,
                                                   first.data_ptr(), second.data_ptr(), rest.data_ptr(),
                                                   kind.data_ptr(), m, C.byref(out))
    return status, out


def assert_matches(got, ref):
    assert got.node_count == ref.node_count
    assert got.dynamic_node_count == ref.dynamic_node_count
    assert got.constraint_count == ref.constraint_count
    assert got.finite == ref.finite == 1
    assert got.maximum_distance_error == ref.maximum_distance_error
    assert got.maximum_cable_extension == ref.maximum_cable_extension
    assert got.total_dynamic_mass == pytest.approx(ref.total_dynamic_mass, rel=SUM_RTOL)
    assert got.kinetic_energy == pytest.approx(ref.kinetic_energy, rel=SUM_RTOL)
    for field in ("center_of_mass", "linear_momentum"):
        g, r = getattr(got, field), getattr(ref, field)
        scale = max(abs(r.x), abs(r.y), abs(r.z), 1e-30)
        for axis in "xyz":
            assert abs(getattr(g, axis) - getattr(r, axis)) <= SUM_RTOL * scale


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["patch", "wing"])
def test_noalloc_diagnostics_match_structure_diagnostics_twice(cuda_device, name):
    # the wing has no pilot here, and both definitions are moved so that
    # their bounding box is centred on the origin: the state's FP64 origin
    # (the box's centre on a 1/256 m grid) is then zero, and the node arrays
    # read back are the device's FP32 values exactly
    definition = sw.generate_patch() if name == "patch" else \
        sw.generate_wing(cells=8, chordwise=16, spanwise_per_cell=2, rib_layers=3, pilot=0)
    pos = definition.nodes()["position"]
    for axis in "xyz":
        pos[axis] -= 0.5 * (pos[axis].min() + pos[axis].max())
    with sw.Structure(definition) as structure:
        settings = step_settings()
        for call in range(2):
            structure.step(settings, diagnostics=False)
            ref = structure.diagnostics()
            arrays = device_arrays(structure, definition)
            status, got = noalloc(arrays)
            assert status == abi.OK, abi.library().swb_last_error()
            assert_matches(got, ref)
            if name == "wing":
                assert got.maximum_cable_extension >= 0.0 and got.maximum_distance_error > 0.0


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_maximum(cuda_device):
    out = abi.Diagnostics()
    lib = abi.library()
    status = lib.swb_diagnostics_noalloc(0, None, None, None, MAX_ITEMS + 1, None, None, None, None, 0,
                                         C.byref(out))
    assert status == abi.INVALID_ARGUMENT
    assert b"exceeds the no-alloc maximum" in lib.swb_last_error()
    status = lib.swb_diagnostics_noalloc(0, None, None, None, 0, None, None, None, None, MAX_ITEMS + 1,
                                         C.byref(out))
    assert status == abi.INVALID_ARGUMENT
    assert b"exceeds the no-alloc maximum" in lib.swb_last_error()
