"""Closed cell volumes on the device (swb_cell_volumes) against the
reference's estimateClosedCellVolume (cell_volume.cpp:161-306), compiled
into oracle/_ref, byte for byte: the device runs the geometric part in the
reference's order of operations, without FMA contraction.

A cell is a tube of skin triangles (an elliptic profile swept along the
span) closed by its two rib loops.  The cases cover both loop windings,
loops given as separate nodes (the geometric orientation fallback), jittered
shapes, and every early return: invalid loops, a bad or repeated face index,
a non-finite position part way through the faces, degenerate and
non-manifold faces, a flat (ambiguous) cell.
"""
import ctypes as C

import numpy as np
import pytest

import simwing_b200 as sw
import simwing_b200.abi as abi
from oracle import oracle as O


class CellDef(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("face_begin", "face_count", "low_begin", "low_count", "high_begin",
                                           "high_count")]


class CellVolume(C.Structure):
    _fields_ = [("signed_volume", C.c_double), ("volume", C.c_double)] + \
               [(n, C.c_uint64) for n in ("skin_boundary_edges", "cap_boundary_edges_matched",
                                          "non_manifold_skin_edges", "degenerate_skin_faces")] + \
               [(n, C.c_uint32) for n in ("valid", "watertight_after_capping", "used_geometric_orientation_fallback",
                                          "ambiguous_skin_orientation")]


def tube(m=12, k=6, rng=None, flat=False):
    """Nodes and triangles of one tube cell; returns (positions, triangles,
    low ring, high ring)."""
    pts, tris = [], []
    for j in range(k + 1):
        for i in range(m):
            a = 2 * np.pi * i / m
            x, z = 0.4 * np.cos(a), (0.0 if flat else 0.1 * np.sin(a))
            p = np.array([x, 0.25 * j, z])
            if rng is not None:
                p = p + rng.normal(scale=0.01, size=3)
            pts.append(p)
    for j in range(k):
        for i in range(m):
            a, b = j * m + i, j * m + (i + 1) % m
            c, d = a + m, b + m
            tris += [(a, b, d), (a, d, c)]
    return np.array(pts), tris, list(range(m)), [k * m + i for i in range(m)]


def build_cases():
    rng = np.random.default_rng(4)
    cells = []  # (positions, triangles, faces, low, high)
    for jitter in (None, rng, rng):
        p, t, lo, hi = tube(rng=jitter)
        faces = list(range(len(t)))
        cells.append((p, t, faces, lo, hi))                 # watertight
        cells.append((p, t, faces, lo[::-1], hi[::-1]))     # the other winding
        # loops as separate nodes at the same places: no shared edges, the
        # caps orient by geometry
        n = len(p)
        q = np.concatenate([p, p[lo], p[hi]])
        cells.append((q, t, faces, list(range(n, n + len(lo))), list(range(n + len(lo), n + 2 * len(lo)))))
    p, t, lo, hi = tube()
    faces = list(range(len(t)))
    cells.append((p, t, faces, lo[:2], hi))                        # loop too short
    cells.append((p, t, faces, [lo[0], lo[1], lo[1], lo[2]], hi))  # repeated loop node
    cells.append((p, t, faces[:10] + [len(t) + 5] + faces[10:], lo, hi))  # face index out of range
    cells.append((p, t, faces[:10] + [3] + faces[10:], lo, hi))    # repeated face
    bad = p.copy()
    bad[t[20][1]] = np.nan                                         # non-finite part way through
    cells.append((bad, t, faces, lo, hi))
    deg = p.copy()
    deg[t[7][2]] = deg[t[7][0]]                                    # degenerate faces
    cells.append((deg, t, faces, lo, hi))
    cells.append((p, t + [t[0]], faces + [len(t)], lo, hi))        # the same face twice: non-manifold edges
    pf, tf, lof, hif = tube(flat=True)                             # flat: ambiguous orientation
    n = len(pf)
    cells.append((np.concatenate([pf, pf[lof], pf[hif]]), tf, list(range(len(tf))),
                  list(range(n, n + len(lof))), list(range(n + len(lof), n + 2 * len(lof)))))
    return cells


def run(fn, case):
    p, t, faces, lo, hi = case
    d = sw.definition_from_arrays([(x, y, z, 1.0, 0) for x, y, z in np.nan_to_num(p)], t)
    cell = (CellDef * 1)(CellDef(0, len(faces), 0, len(lo), len(lo), len(hi)))
    f = np.array(faces, dtype=np.uint64)
    loops = np.array(list(lo) + list(hi), dtype=np.uint64)
    pos = np.ascontiguousarray(p, dtype=np.float64)
    out = (CellVolume * 1)()
    status = fn(d.pointer, f.ctypes.data, loops.ctypes.data, cell, 1, pos.ctypes.data, out)
    assert status == 0
    return out[0]


def bind(lib, name):
    fn = getattr(lib, name)
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    return fn


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")


@needs_ref
def test_reference_volume_of_a_closed_tube_is_the_polyhedron_volume():
    """Pins the fixture: the watertight tube's estimate is the volume of the
    polyhedron (skin plus the two fan-triangulated caps), by the divergence
    theorem in numpy."""
    p, t, lo, hi = tube()
    est = run(bind(O.ref_library(), "swref_cell_volumes"), (p, t, list(range(len(t))), lo, hi))
    assert est.valid and est.watertight_after_capping and not est.used_geometric_orientation_fallback
    ring = lambda r: p[r].mean(axis=0)
    tris = [p[list(x)] for x in t]
    cl, ch = ring(lo), ring(hi)
    for r, c in ((lo, cl), (hi, ch)):
        for i in range(len(r)):
            tris.append(np.array([c, p[r[i]], p[r[(i + 1) % len(r)]]]))
    vol = abs(sum(np.dot(a, np.cross(b, c)) for a, b, c in tris)) / 6.0  # |sum|: cap windings cancel in pairs
    assert est.volume == pytest.approx(vol, rel=0.05)
    assert est.volume == pytest.approx(0.4 * 0.1 * np.pi * 1.5 * 0.97, rel=0.05)


@pytest.mark.gpu
@needs_ref
def test_device_cell_volumes_equal_the_reference_bytewise(cuda_device):
    dev = bind(abi.library(), "swb_cell_volumes")
    ref = bind(O.ref_library(), "swref_cell_volumes")
    cases = build_cases()
    seen = set()
    for k, case in enumerate(cases):
        a, b = run(dev, case), run(ref, case)
        assert bytes(a) == bytes(b), f"case {k}"
        seen.add((b.valid, b.watertight_after_capping, b.used_geometric_orientation_fallback,
                  b.ambiguous_skin_orientation))
    # valid watertight, valid with fallback, invalid ambiguous, and the early returns
    assert (1, 1, 0, 0) in seen and (1, 0, 1, 0) in seen and (0, 0, 1, 1) in seen and (0, 0, 0, 0) in seen


def plan_for(case):
    p, t, faces, lo, hi = case
    d = sw.definition_from_arrays([(x, y, z, 1.0, 0) for x, y, z in np.nan_to_num(p)], t)
    cell = (CellDef * 1)(CellDef(0, len(faces), 0, len(lo), len(lo), len(hi)))
    f = np.array(faces, dtype=np.uint64)
    loops = np.array(list(lo) + list(hi), dtype=np.uint64)
    plan = C.c_void_p()
    sw._check(abi.library().swb_cell_volume_plan_create(d.pointer, f.ctypes.data, loops.ctypes.data,
                                                         C.cast(cell, C.c_void_p), 1, 0, C.byref(plan)))
    return d, plan


@pytest.mark.gpu
def test_device_resident_cell_volumes_equal_the_host_form(cuda_device):
    """swb_cell_volumes_device (tables uploaded once at plan creation,
    positions and results in device memory, one launch on the caller's
    stream) gives the host form's estimates byte for byte."""
    import torch

    lib = abi.library()
    host = bind(lib, "swb_cell_volumes")
    stream = torch.cuda.Stream()
    for k, case in enumerate(build_cases()):
        d, plan = plan_for(case)
        try:
            pos = torch.tensor(np.ascontiguousarray(case[0], dtype=np.float64), device="cuda")
            out = torch.zeros(C.sizeof(CellVolume), dtype=torch.uint8, device="cuda")
            for _ in range(2):  # the plan is reused
                sw._check(lib.swb_cell_volumes_device(plan, pos.data_ptr(), out.data_ptr(),
                                                      C.c_void_p(stream.cuda_stream)))
            stream.synchronize()
            got = CellVolume.from_buffer_copy(out.cpu().numpy().tobytes())
            assert bytes(got) == bytes(run(host, case)), f"case {k}"
        finally:
            lib.swb_cell_volume_plan_destroy(plan)


@pytest.mark.gpu
def test_structure_cell_volumes_at_the_device_state(cuda_device):
    """swb_structure_cell_volumes reads a structure's committed state where
    it lives: the estimates equal the host form's on the node states the
    structure reports (the same FP32 offsets widened to FP64 world
    positions)."""
    import torch

    lib = abi.library()
    p, t, lo, hi = tube(rng=np.random.default_rng(9))
    faces = list(range(len(t)))
    case = (p, t, faces, lo, hi)
    d, plan = plan_for(case)
    try:
        s = sw.Structure(d)
        st = sw.StepSettings(time_step=1.0 / 120.0, substeps=1, constraint_iterations=4, gravity=(0.0, 0.0, -9.81))
        out = torch.zeros(C.sizeof(CellVolume), dtype=torch.uint8, device="cuda")
        for _ in range(3):
            s.step(st, diagnostics=False)
            sw._check(lib.swb_structure_cell_volumes(s.handle, plan, out.data_ptr()))
            torch.cuda.synchronize()
            got = CellVolume.from_buffer_copy(out.cpu().numpy().tobytes())
            want = run(bind(lib, "swb_cell_volumes"), (s.positions(), t, faces, lo, hi))
            assert bytes(got) == bytes(want)
            assert got.valid and got.watertight_after_capping
        s.close()
    finally:
        lib.swb_cell_volume_plan_destroy(plan)
