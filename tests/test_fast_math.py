"""fast_atan2 / fast_rcp (simwing_b200/csrc/fast_math.h), the short forms the
projection kernels use, against the C++ library on the host: fast_atan2
within 4e-7 rad over every octant, near the octant boundaries and at the
special points.  The checks live in tests/cpp/fast_math_test.cpp."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fast_math_against_the_library(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "fast_math_test"
    subprocess.run([cxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror",
                    os.path.join(ROOT, "tests", "cpp", "fast_math_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


def device_eval(which, a, b=None):
    import ctypes as C

    import numpy as np

    import simwing_b200 as sw
    from simwing_b200 import abi

    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(a if b is None else b, dtype=np.float32)
    out = np.zeros_like(a)
    sw._check(abi.library().swb_fast_math_eval(which, a.ctypes.data, b.ctypes.data, out.ctypes.data, a.size))
    return out


@pytest.mark.gpu
def test_device_fast_math(cuda_device):
    """The device forms on the GPU: fast_atan2 within 7e-7 rad of atan2
    (4e-7 for the polynomial and its reflections, plus the approximate
    division's 2 ulp of the reduced argument) over every octant, the octant
    boundaries, the axes and magnitudes from 1e-30 to 1e30; fast_rcp within
    2 ulp over normal magnitudes below 2^126."""
    import numpy as np

    from simwing_b200 import abi

    rng = np.random.default_rng(11)
    n = 1 << 20
    mag = 10.0 ** rng.uniform(-30, 30, n)
    ang = rng.uniform(-np.pi, np.pi, n)
    ang[: n // 8] = np.round(ang[: n // 8] / (np.pi / 4)) * (np.pi / 4) + rng.normal(0, 1e-6, n // 8)
    y = (mag * np.sin(ang)).astype(np.float32)
    x = (mag * np.cos(ang)).astype(np.float32)
    special = np.array([0.0, 1.0, -1.0, 1e-30, -1e-30], dtype=np.float32)
    y = np.concatenate([y, np.repeat(special, special.size)])
    x = np.concatenate([x, np.tile(special, special.size)])
    got = device_eval(abi.FAST_ATAN2, y, x).astype(np.float64)
    want = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    err = np.abs(got - want)
    err = np.minimum(err, 2 * np.pi - err)  # +pi and -pi are the same angle
    assert float(err.max()) <= 7e-7, (float(err.max()), y[err.argmax()], x[err.argmax()])
    v = (10.0 ** rng.uniform(-37, 37, n) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    r = device_eval(abi.FAST_RCP, v).astype(np.float64)
    rel = np.abs(r * v.astype(np.float64) - 1.0)
    assert float(rel.max()) <= 2.0 * 2.0 ** -23, float(rel.max())
