"""The FP64 yardstick of the accuracy reports (gpu-pcg-tracking_b200/fp64check.py) against the
oracle's FP64 Schur complement, banded Cholesky and dz recovery (no GPU needed)."""
import importlib

import numpy as np
import pytest

from conftest import ref_problem


@pytest.fixture(scope="module")
def fp64check():
    return importlib.import_module("gpu-pcg-tracking_b200.fp64check")


@pytest.mark.parametrize("N,rho", [(2, 1e-3), (7, 1e-2), (32, 1e-3)])
def test_fp64check_matches_oracle_fp64_solve(oracle, problem_mod, fp64check, N, rho):
    par = oracle.make_params(dt=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)
    p = problem_mod.make_problem(N, 3, dt=0.01)
    G, Cm, g, c = oracle.form_kkt(par, N, p["xu"], p["goal"], p["xs"], "f32")
    S, _, gam, Gi = oracle.form_schur(N, rho, G, Cm, g, c, "f64")
    lam_o = oracle.banded_cholesky(N, S, gam, "f64")
    dz_o = oracle.compute_dz(N, Gi, Cm, g, lam_o, "f64")
    lam, dz = fp64check.solve_step(N, rho, G, Cm, g, c)
    assert fp64check.rel_err(lam, lam_o) < 1e-8
    assert fp64check.rel_err(dz, dz_o) < 1e-8


def test_fp64check_on_reference_trajectory(oracle, golden, fp64check):
    N = 32
    par = oracle.make_params()  # dt 1/64, explicit Euler, QD = R = 1e-4
    p = ref_problem(golden, N)
    G, Cm, g, c = oracle.form_kkt(par, N, p["xu"], p["goal"], p["xs"], "f32")
    S, _, gam, Gi = oracle.form_schur(N, 1e-3, G, Cm, g, c, "f64")
    lam_o = oracle.banded_cholesky(N, S, gam, "f64")
    dz_o = oracle.compute_dz(N, Gi, Cm, g, lam_o, "f64")
    lam, dz = fp64check.solve_step(N, 1e-3, G, Cm, g, c)
    assert fp64check.rel_err(lam, lam_o) < 1e-7
    assert fp64check.rel_err(dz, dz_o) < 1e-7


def test_rel_err_definition(fp64check):
    assert fp64check.rel_err([1.0, 2.0], [1.0, 2.0]) == 0.0
    assert abs(fp64check.rel_err([1.0, 2.5], [1.0, 2.0]) - 0.25) < 1e-15
    assert fp64check.rel_err([], []) == 0.0
