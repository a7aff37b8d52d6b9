"""Shared fixtures: the CPU oracle (checker), the CUDA product and test problems."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_testfiles.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def gpt():
    return importlib.import_module("gpu-pcg-tracking_b200")


@pytest.fixture(scope="session")
def problem_mod():
    return importlib.import_module("gpu-pcg-tracking_b200.problem")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def ref_problem(golden, N, start=1):
    """Reference-compatible instance: rows of testfiles/0_0_traj.csv as xu and its
    FK golden file as the goal (runme.cu:145-161), dt = 1/64, explicit Euler."""
    tr = golden["traj_0_0"][start:start + N].astype(np.float32)
    ee = golden["eepos_0_0"][start:start + N].astype(np.float32)
    xu = tr.reshape(-1)[:21 * N - 7].copy()
    return {"xu": xu, "goal": ee.reshape(-1).copy(), "xs": xu[:14].copy(), "lam": np.zeros(14 * N, np.float32)}
