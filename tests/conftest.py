"""Test configuration: the `gpu` marker, repository imports and the in-tree
builds (product library and the C oracle port) when they are missing."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C-ABI")


def _ensure_built():
    lib = os.path.join(ROOT, "simwing_b200", "libsimwing_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "simwing_b200"), "-j8"], check=True)
    for target, lib in (("port", "liboracle.so"), ("adjoint", "libadjoint.so")):
        if not os.path.exists(os.path.join(ROOT, "oracle", lib)):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), target], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.cuda.get_device_properties(0)


def step_settings(iterations=48, substeps=1, dt=1.0 / 120.0, gravity=(0.0, 0.0, -9.81), damping=0.25):
    import simwing_b200 as sw

    return sw.StepSettings(time_step=dt, substeps=substeps, constraint_iterations=iterations, gravity=gravity,
                           velocity_damping=damping)
