"""Adjoint arithmetic of the device step (simwing_b200/csrc/adjoint_math.h),
compiled for the host and checked against central finite differences in
double precision: the hand-written reverse of the distance-type and dihedral
projections (every input, every regime), and the dual-number Jacobians of the
rigid-pilot functions.  The checks live in tests/cpp/adjoint_math_test.cpp."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_adjoint_math_matches_finite_differences(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "adjoint_math_test"
    subprocess.run([cxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror",
                    os.path.join(ROOT, "tests", "cpp", "adjoint_math_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("ok  ") == 11
