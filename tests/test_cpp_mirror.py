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


def reference_details():
    """The details the reference build's exceptions carry on the mirror
    test's two failing definitions: a wing whose line residual bound is
    zero, and two pinned sheets inside each other's contact envelope."""
    import simwing_b200 as sw
    from oracle import oracle as O
    from tests.conftest import step_settings

    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, pressure=0.0)
    d.view.suspension.contents.maximum_line_residual = 0.0
    ref = O.RefStructure(d)
    with pytest.raises(O.OracleError) as susp:
        for _ in range(20):
            ref.step(step_settings())
    nodes = [(-1, -1, 0, 1.0, 1), (1, -1, 0, 1.0, 1), (0, 1, 0, 1.0, 1),
             (-1, -1, 0.005, 1.0, 1), (0, 1, 0.005, 1.0, 1), (1, -1, 0.005, 1.0, 1), (3, 3, 3, 1.0, 0)]
    ref = O.RefStructure(sw.definition_from_arrays(nodes, [(0, 1, 2), (3, 4, 5)], contact=(0.01, 0.0, 0.0, 0.0)))
    with pytest.raises(O.OracleError) as contact:
        ref.step(step_settings(iterations=4))
    return susp.value, contact.value


@pytest.mark.gpu
def test_mirror_steps_checkpoints_and_throws_like_the_reference(mirror_binary, cuda_device):
    from simwing_b200 import abi
    from oracle import oracle as O

    out = run(mirror_binary, "gpu")
    assert out.count("ok  ") == 21
    if not O.ref_available():
        pytest.skip("reference build not present")
    susp, contact = reference_details()
    lines = {ln.split()[1]: ln.split()[2:] for ln in out.splitlines() if ln.startswith("detail ")}
    assert abi.SUSPENSION_PHASES[int(lines["suspension"][0])] == susp.phase
    assert lines["suspension"][1] == susp.entity
    pair, kind, *prims = (int(x) for x in lines["contact"])
    assert (pair, kind, tuple(prims[:3]), tuple(prims[3:])) == contact.key
