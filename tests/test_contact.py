"""Contact building blocks on the device against the reference itself.

The reference's contact code (src/softwing/contact.cpp) is compiled into
oracle/_ref/libswref.so.  The device candidate list of a fabric self-contact
pair (swb_contact_candidates) is compared key for key with the list one
SoftBody contact iteration streams (read through the reference's own audit
hook), and the device closest-feature and swept-contact queries
(swb_contact_closest, swb_contact_sweep) with closestVertexTriangle,
closestEdgeEdge and sweptContact, byte for byte: the device runs these in
FP64 without FMA contraction, as the reference build does.

The CPU tests pin the candidate semantics (the eligible features whose
swept, expanded AABBs overlap on all three axes, in key order) with a numpy
restatement, and the host-side validation of the entry points.
"""
import ctypes as C

import numpy as np
import pytest

import simwing_b200 as sw
import simwing_b200.abi as abi
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")

EPS = np.finfo(np.float64).eps


def two_sheets():
    """The reference's contact fixture (simwing_structure_test.cpp:297-329):
    two disconnected triangles 1 cm apart."""
    nodes = [(-1, -1, 0, 1.0, 0), (1, -1, 0, 1.0, 0), (0, 1, 0, 1.0, 0),
             (-1, -1, 0.01, 1.0, 0), (0, 1, 0.01, 1.0, 0), (1, -1, 0.01, 1.0, 0)]
    d = sw.definition_from_arrays(nodes, [(0, 1, 2), (3, 4, 5)])
    p = np.array([n[:3] for n in nodes], dtype=np.float64)
    return d, p, p.copy(), 0.01


def folded_patch(n=12, gap=0.004):
    """A square sheet folded over itself along its mid-line during the
    substep: the upper half lands `gap` above the lower half."""
    d = sw.generate_patch(nx=n, ny=n, seed=7)
    prev = d.positions()
    cur = prev.copy()
    axis = 2 if np.ptp(prev[:, 2]) > np.ptp(prev[:, 1]) else 1
    mid = 0.5 * (prev[:, axis].min() + prev[:, axis].max())
    up = prev[:, axis] > mid
    cur[up, axis] = 2 * mid - prev[up, axis]
    normal = 1 if axis == 2 else 2
    cur[up, normal] += gap
    return d, prev, cur, 0.75 * gap


def crumpled_patch(n=16, seed=11):
    """A sheet crumpled by smooth random displacements of about its own
    edge length, so that many non-adjacent features come close."""
    d = sw.generate_patch(nx=n, ny=n, seed=seed)
    prev = d.positions()
    rng = np.random.default_rng(seed)
    k = rng.normal(size=(3, 3, 2))
    u = (prev - prev.min(0)) / np.ptp(prev, axis=0).clip(1e-9)
    disp = np.zeros_like(prev)
    for c in range(3):
        disp[:, c] = 0.15 * (np.sin(6.0 * (k[c, 0, 0] * u[:, 0] + k[c, 0, 1] * u[:, 2]) + k[c, 1, 0]) +
                             np.cos(5.0 * (k[c, 2, 0] * u[:, 1] + k[c, 2, 1] * u[:, 2])))
    return d, prev, prev + disp, 0.01


FIXTURES = {"two_sheets": two_sheets, "folded_patch": folded_patch, "crumpled_patch": crumpled_patch}


def key_tuple(k):
    return (k.pair, k.kind, tuple(k.first), tuple(k.second))


def restated_candidates(d, half_thickness, prev, cur):
    """Candidate keys as the exhaustive overlap predicate over eligible
    features, with the swept AABB of contact.cpp:488-526 (numpy FP64)."""
    tri = np.asarray(d.triangles()["nodes"], dtype=np.int64).reshape(-1, 3)
    verts = np.unique(tri)
    edges = sorted({(min(a, b), max(a, b)) for t in tri for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0]))})
    sep = 2.0 * half_thickness

    def box(ids):
        pts = np.concatenate([prev[ids], cur[ids]])
        lo, hi = pts.min(0), pts.max(0)
        scale = max(1.0, float(np.abs(pts).max()))
        total = sep + 64.0 * EPS * max(scale, sep)
        return lo - total, hi + total

    def overlap(a, b):
        return bool(np.all(a[0] <= b[1]) and np.all(b[0] <= a[1]))

    vb = {v: box([v]) for v in verts}
    tb = [box(list(t)) for t in tri]
    eb = [box(list(e)) for e in edges]
    keys = []
    for v in verts:
        for t, nodes in enumerate(tri):
            if v not in nodes and overlap(vb[v], tb[t]):
                keys.append((0, 0, (int(v), 0, 0), (t, 0, 0)))
    for i, e in enumerate(edges):
        for j in range(i + 1, len(edges)):
            f = edges[j]
            if len({e[0], e[1], f[0], f[1]}) == 4 and overlap(eb[i], eb[j]):
                keys.append((0, 1, (e[0], e[1], 0), (f[0], f[1], 0)))
    return keys


@needs_ref
@pytest.mark.parametrize("name", ["two_sheets", "folded_patch"])
def test_reference_candidates_are_the_overlapping_eligible_features(name):
    d, prev, cur, h = FIXTURES[name]()
    keys, possible, excluded = O.ref_contact_candidates(d, h, prev, cur)
    assert [key_tuple(k) for k in keys] == restated_candidates(d, h, prev, cur)
    assert len(keys) > 0


def test_contact_entry_points_validate_on_the_host():
    d, prev, cur, h = two_sheets()
    lib = abi.library()
    n = C.c_uint64()
    for bad_h in (0.0, -1.0, float("nan")):
        assert lib.swb_contact_candidates(d.pointer, bad_h, prev.ctypes.data, cur.ctypes.data, None, 0,
                                          C.byref(n), None, None) == abi.INVALID_ARGUMENT
    degenerate = sw.definition_from_arrays([(0, 0, 0, 1.0, 0), (1, 0, 0, 1.0, 0), (2, 0, 0, 1.0, 0)], [(0, 1, 2)])
    p = np.zeros((3, 3))
    assert lib.swb_contact_candidates(degenerate.pointer, 0.01, p.ctypes.data, p.ctypes.data, None, 0,
                                      C.byref(n), None, None) == abi.INVALID_ARGUMENT
    repeated = sw.definition_from_arrays([(0, 0, 0, 1.0, 0), (1, 0, 0, 1.0, 0), (0, 1, 0, 1.0, 0)], [(0, 1, 1)])
    assert lib.swb_contact_candidates(repeated.pointer, 0.01, p.ctypes.data, p.ctypes.data, None, 0,
                                      C.byref(n), None, None) == abi.INVALID_ARGUMENT
    q = np.zeros((1, 9))
    out = (abi.CcdResult * 1)()
    assert lib.swb_contact_sweep(abi.FEATURE_SEGMENT_TRIANGLE, 1, *[q.ctypes.data] * 4, 0.0,
                                 C.byref(sw.CcdSettings()), out) == abi.UNSUPPORTED
    assert lib.swb_contact_sweep(abi.FEATURE_EDGE_EDGE, 1, *[q.ctypes.data] * 4, 0.0,
                                 C.byref(sw.CcdSettings(interval_subdivisions=abi.CCD_MAX_SUBDIVISIONS + 1)),
                                 out) == abi.INVALID_ARGUMENT
    assert lib.swb_contact_closest(7, 1, q.ctypes.data, q.ctypes.data, 0.0, (abi.ClosestResult * 1)()) == \
        abi.INVALID_ARGUMENT


def test_default_ccd_settings_are_the_reference_defaults():
    s = sw.CcdSettings()
    assert (s.conservative_iterations, s.interval_subdivisions, s.time_tolerance, s.distance_tolerance) == \
        (32, 256, 1.0e-8, 1.0e-10)


# ---- device against the reference (GPU) ------------------------------------

@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_device_candidates_equal_the_reference(cuda_device, name):
    d, prev, cur, h = FIXTURES[name]()
    ref_keys, ref_possible, ref_excluded = O.ref_contact_candidates(d, h, prev, cur)
    keys, possible, excluded = sw.contact_candidates(d, h, prev, cur)
    assert (possible, excluded) == (ref_possible, ref_excluded)
    assert [key_tuple(k) for k in keys] == [key_tuple(k) for k in ref_keys]
    assert len(keys) > 0


@pytest.mark.gpu
def test_device_candidates_of_an_empty_surface(cuda_device):
    d = sw.definition_from_arrays([(0, 0, 0, 1.0, 0)])
    p = np.zeros((1, 3))
    keys, possible, excluded = sw.contact_candidates(d, 0.01, p, p)
    assert (keys, possible, excluded) == ([], 0, 0)


def random_features(rng, n, kind):
    """Random features around the origin plus the degenerate and boundary
    cases the queries branch on."""
    first = rng.normal(scale=0.3, size=(n, 9))
    second = rng.normal(scale=0.3, size=(n, 9))
    special_first, special_second = [], []
    if kind == abi.FEATURE_VERTEX_TRIANGLE:
        tri = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], dtype=float)
        for p in ([0.2, 0.2, 0.1], [-1, -1, 0.3], [2, -0.5, 0], [-0.5, 2, 0], [0.6, 0.6, 0.0], [0.5, -0.2, 0.0],
                  [-0.2, 0.5, 0.0], [0.25, 0.25, 0.0], [0, 0, 0], [1, 0, 0]):
            special_first.append(p + [0] * 6)
            special_second.append(tri)
        special_first.append([0.3, 0.3, 0.3] + [0] * 6)   # collinear triangle: degenerate
        special_second.append([0, 0, 0, 1, 1, 1, 2, 2, 2])
        special_first.append([np.inf, 0, 0] + [0] * 6)    # non-finite
        special_second.append(tri)
    else:
        for f, s in (([0, 0, 0, 1, 0, 0], [0, 1, 0, 1, 1, 0]),       # parallel
                     ([0, 0, 0, 1, 0, 0], [0.5, -1, 0, 0.5, 1, 0]),   # crossing: zero distance
                     ([0, 0, 0, 1, 0, 0], [2, 1, 0, 2, -1, 1]),       # clamped ends
                     ([0, 0, 0, 1, 0, 0], [-1, 0, 1, -1, 0, 1]),      # degenerate second edge
                     ([0, 0, 0, 1, 0, 0], [0, 0, 0, 1, 0, 0]),        # coincident
                     ([0, 0, 0, 1, 0, 0], [3, 0, 0, 4, 0, 0])):       # collinear, apart
            special_first.append(f + [0, 0, 0])
            special_second.append(s + [0, 0, 0])
    return (np.concatenate([first, np.array(special_first, dtype=float)]),
            np.concatenate([second, np.array(special_second, dtype=float)]))


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("kind", [abi.FEATURE_VERTEX_TRIANGLE, abi.FEATURE_EDGE_EDGE])
@pytest.mark.parametrize("separation", [0.0, 0.02, -1.0])
def test_device_closest_features_equal_the_reference_bytewise(cuda_device, kind, separation):
    rng = np.random.default_rng(100 + kind)
    first, second = random_features(rng, 3000, kind)
    dev = sw.contact_closest(kind, first, second, separation)
    ref = O.ref_contact_closest(kind, first, second, separation)
    mismatched = [i for i, (a, b) in enumerate(zip(dev, ref)) if bytes(a) != bytes(b)]
    assert not mismatched, f"{len(mismatched)} results differ, first at {mismatched[:5]}"
    statuses = {r.status for r in ref}
    if separation >= 0.0:
        assert abi.GEOMETRY_CERTIFIED in statuses and abi.GEOMETRY_DEGENERATE in statuses


def random_motions(rng, n, kind, speed):
    """Primitives moving linearly: approach, crossing, grazing and resting
    motions at several speeds."""
    fp, sp = random_features(rng, n, kind)
    fp, sp = fp[:n], sp[:n]
    fc = fp + speed * rng.normal(size=fp.shape)
    sc = sp + speed * rng.normal(size=sp.shape)
    # a quarter of the features rest; a quarter move rigidly together
    fc[: n // 4], sc[: n // 4] = fp[: n // 4], sp[: n // 4]
    shift = speed * rng.normal(size=(n // 4, 3))
    lo, hi = n // 4, n // 2
    fc[lo:hi] = fp[lo:hi] + np.tile(shift, 3)
    sc[lo:hi] = sp[lo:hi] + np.tile(shift, 3)
    return fp, fc, sp, sc


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("kind", [abi.FEATURE_VERTEX_TRIANGLE, abi.FEATURE_EDGE_EDGE])
@pytest.mark.parametrize("settings", [
    {}, {"conservative_iterations": 0}, {"interval_subdivisions": 0},
    {"conservative_iterations": 0, "interval_subdivisions": 0}, {"conservative_iterations": 2, "interval_subdivisions": 3},
    {"time_tolerance": -1.0}])
def test_device_swept_contact_equals_the_reference_bytewise(cuda_device, kind, settings):
    rng = np.random.default_rng(7 + kind)
    cs = sw.CcdSettings(**settings)
    parts = [random_motions(rng, 600, kind, s) for s in (0.01, 0.2, 1.0)]
    fp, fc, sp, sc = (np.concatenate([p[i] for p in parts]) for i in range(4))
    for separation in (0.0, 0.05):
        dev = sw.contact_sweep(kind, fp, fc, sp, sc, separation, cs)
        ref = O.ref_contact_sweep(kind, fp, fc, sp, sc, separation, cs)
        mismatched = [i for i, (a, b) in enumerate(zip(dev, ref)) if bytes(a) != bytes(b)]
        assert not mismatched, f"{len(mismatched)} results differ, first at {mismatched[:5]}"
    if not settings:
        states = {r.state for r in ref}
        assert {abi.CCD_NO_IMPACT, abi.CCD_IMPACT, abi.CCD_INITIALLY_PROXIMATE} <= states
        assert any(r.used_interval_fallback for r in ref)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [abi.FEATURE_VERTEX_TRIANGLE, abi.FEATURE_EDGE_EDGE])
def test_swept_contact_with_a_tolerance_below_double_spacing_returns(cuda_device, kind):
    """A time tolerance finer than the spacing of doubles near the impact
    time: the bisection of sweptContact (contact.cpp:778-804) reaches an
    interval whose midpoint rounds onto one of its ends, where the
    reference's loop would never end.  The device stops there with the
    interval refined to double resolution; the states are those of a
    tolerance the reference handles."""
    rng = np.random.default_rng(31 + kind)
    parts = [random_motions(rng, 400, kind, s) for s in (0.05, 0.3)]
    fp, fc, sp, sc = (np.concatenate([p[i] for p in parts]) for i in range(4))
    fine = sw.contact_sweep(kind, fp, fc, sp, sc, 0.05, sw.CcdSettings(time_tolerance=1e-300))
    coarse = sw.contact_sweep(kind, fp, fc, sp, sc, 0.05, sw.CcdSettings(time_tolerance=1e-12))
    impacts = 0
    for a, b in zip(fine, coarse):
        assert a.state == b.state
        if a.state == abi.CCD_IMPACT:
            impacts += 1
            assert a.bracket_lower <= a.time_of_impact <= a.bracket_upper
            assert a.bracket_upper - a.bracket_lower <= 1e-12
            assert abs(a.time_of_impact - b.time_of_impact) <= 2e-12
    assert impacts > 0
