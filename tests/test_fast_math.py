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
