"""The C++ mirror of simwing::fsi::Structure (include/simwing_b200_structure.hpp)
compiles against the C-ABI with the reference's type and member names and
throws the reference's exception types (src/fsi/structure.cpp:102-455,
778-831, 961-1027).  The checks live in tests/cpp/structure_mirror_test.cpp."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def mirror_binary(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("mirror") / "structure_mirror_test"
    lib_dir = os.path.join(ROOT, "simwing_b200")
    subprocess.run([cxx, "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "structure_mirror_test.cpp"), "-L", lib_dir,
                    "-lsimwing_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(out)], check=True)
    return str(out)


def run(binary, mode):
    r = subprocess.run([binary, mode], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
    return r.stdout


def test_mirror_validation_and_exception_mapping(mirror_binary):
    out = run(mirror_binary, "cpu")
    assert out.count("ok  ") == 8


@pytest.mark.gpu
def test_mirror_steps_checkpoints_and_throws_like_the_reference(mirror_binary, cuda_device):
    out = run(mirror_binary, "gpu")
    assert out.count("ok  ") == 19
