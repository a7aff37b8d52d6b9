"""Pins the CPU oracle to the reference's own known-answer data and to the
mathematics it restates (no GPU needed)."""
import numpy as np
import pytest

from conftest import ref_problem


def test_fk_matches_reference_golden_file(oracle, golden):
    # testfiles/0_0_eepos.traj = reference FK of every row of 0_0_traj.csv, 6 digits (generateeepos.cu:101-107)
    tr, ee = golden["traj_0_0"], golden["eepos_0_0"]
    for prec, tol in (("f64", 2e-5), ("f32", 3e-5)):
        err = max(np.abs(oracle.fk(tr[i, :7].astype(np.float64), prec) - ee[i]).max() for i in range(len(tr)))
        assert err < tol, (prec, err)


def test_forward_dynamics_reproduces_reference_trajectories(oracle, golden):
    # testfiles/*_traj.csv are explicit-Euler rollouts at dt = 1/64 with the reference plant (gravity 0)
    dt = 1.0 / 64
    for name in ("traj_0_1", "traj_1_2", "traj_2_3", "traj_3_4", "traj_4_0"):
        tr = golden[name].astype(np.float64)
        for k in range(1, len(tr) - 1):
            x, xn = tr[k], tr[k + 1]
            qdd = oracle.fd(x[:7], x[7:14], x[14:])
            assert np.abs(xn[:7] - (x[:7] + dt * x[7:14])).max() < 1e-6
            assert np.abs(xn[7:14] - (x[7:14] + dt * qdd)).max() < 2e-5, (name, k)


def test_dynamics_gradient_matches_finite_differences(oracle):
    rng = np.random.default_rng(3)
    for _ in range(3):
        x = np.concatenate([rng.uniform(-2, 2, 7), rng.normal(0, 2, 7), rng.normal(0, 20, 7)])
        qdd, dfdu = oracle.fd_grad(x[:7], x[7:14], x[14:])
        np.testing.assert_allclose(qdd, oracle.fd(x[:7], x[7:14], x[14:]), rtol=1e-12, atol=1e-10)
        h = 1e-6
        num = np.zeros((7, 21))
        for j in range(21):
            xp, xm = x.copy(), x.copy()
            xp[j] += h
            xm[j] -= h
            num[:, j] = (oracle.fd(xp[:7], xp[7:14], xp[14:]) - oracle.fd(xm[:7], xm[7:14], xm[14:])) / (2 * h)
        ana = dfdu.reshape(21, 7).T
        assert np.abs(num - ana).max() <= 1e-6 * max(1.0, np.abs(num).max())


def test_minv_and_rnea_are_consistent(oracle):
    rng = np.random.default_rng(4)
    q, qd, qdd = rng.uniform(-2, 2, 7), rng.normal(0, 1, 7), rng.normal(0, 1, 7)
    Minv = oracle.minv(q)
    M = np.stack([oracle.rnea(q, np.zeros(7), e) for e in np.eye(7)], axis=1)
    np.testing.assert_allclose(M, M.T, atol=1e-12)
    np.testing.assert_allclose(Minv @ M, np.eye(7), atol=1e-10)
    tau = oracle.rnea(q, qd, qdd)
    np.testing.assert_allclose(oracle.fd(q, qd, tau), qdd, atol=1e-9)


def test_fk_gradient_matches_finite_differences(oracle):
    rng = np.random.default_rng(5)
    q = rng.uniform(-2, 2, 7)
    J = oracle.fk_grad(q).reshape(7, 6)[:, :3].T
    h = 1e-6
    num = np.stack([(oracle.fk(q + h * e)[:3] - oracle.fk(q - h * e)[:3]) / (2 * h) for e in np.eye(7)], axis=1)
    np.testing.assert_allclose(J, num, atol=1e-8)


def dense_from_blocks(N, S):
    n = 14 * N
    M = np.zeros((n, n))
    for k in range(N):
        row = S[588 * k:588 * k + 588]
        for b, kk in ((0, k - 1), (1, k), (2, k + 1)):
            if 0 <= kk < N:
                M[14 * k:14 * k + 14, 14 * kk:14 * kk + 14] = row[196 * b:196 * b + 196].reshape(14, 14, order="F")
    return M


def kkt_dense(N, G, Cm, g, c, rho):
    """Dense KKT pieces: Gt = blockdiag(Q + rho I, R + rho I), constraint matrix Cc, so the
    reference's linear system is [Gt Cc^T; Cc 0][dz; lambda] = [g; c] (oldschur.cuh:966-1092)."""
    nz = 21 * N - 7
    Gt = np.zeros((nz, nz))
    for k in range(N):
        Q = G[245 * k:245 * k + 196].reshape(14, 14, order="F")
        Gt[21 * k:21 * k + 14, 21 * k:21 * k + 14] = Q + rho * np.eye(14)
        if k < N - 1:
            Rm = G[245 * k + 196:245 * k + 245].reshape(7, 7, order="F")
            Gt[21 * k + 14:21 * k + 21, 21 * k + 14:21 * k + 21] = Rm + rho * np.eye(7)
    Cc = np.zeros((14 * N, nz))
    Cc[0:14, 0:14] = np.eye(14)
    for k in range(N - 1):
        mA = Cm[294 * k:294 * k + 196].reshape(14, 14, order="F")
        mB = Cm[294 * k + 196:294 * k + 294].reshape(14, 7, order="F")
        Cc[14 * (k + 1):14 * (k + 2), 21 * k:21 * k + 14] = mA
        Cc[14 * (k + 1):14 * (k + 2), 21 * k + 14:21 * k + 21] = mB
        Cc[14 * (k + 1):14 * (k + 2), 21 * (k + 1):21 * (k + 1) + 14] = np.eye(14)
    return Gt, Cc


@pytest.mark.parametrize("N", [2, 3, 6])
def test_schur_restatement_is_the_schur_complement(oracle, golden, N):
    p = ref_problem(golden, N)
    par = oracle.make_params()
    rho = 1e-2
    G, Cm, g, c = oracle.form_kkt(par, N, p["xu"], p["goal"], p["xs"])
    S, Pv, gam, Gi = oracle.form_schur(N, rho, G, Cm, g, c)
    Gt, Cc = kkt_dense(N, G, Cm, g, c, rho)
    Gti = np.linalg.inv(Gt)
    M = Cc @ Gti @ Cc.T
    np.testing.assert_allclose(dense_from_blocks(N, S), -M, rtol=1e-9, atol=1e-9 * np.abs(M).max())
    np.testing.assert_allclose(gam, -(Cc @ Gti @ g - c), rtol=1e-9, atol=1e-9 * np.abs(gam).max())
    # block-Jacobi preconditioner: Pinv diag blocks invert S diag blocks
    for k in range(N):
        Sd = S[588 * k + 196:588 * k + 392].reshape(14, 14, order="F")
        Pd = Pv[588 * k + 196:588 * k + 392].reshape(14, 14, order="F")
        np.testing.assert_allclose(Sd @ Pd, np.eye(14), atol=1e-8)
    # dz from the exact lambda solves the full KKT system
    lam = oracle.banded_cholesky(N, S, gam)
    dz = oracle.compute_dz(N, Gi, Cm, g, lam)
    np.testing.assert_allclose(Gt @ dz + Cc.T @ lam, g, atol=1e-8 * max(1, np.abs(g).max()))
    np.testing.assert_allclose(Cc @ dz, c, atol=1e-8 * max(1, np.abs(c).max()))


@pytest.mark.parametrize("N", [2, 5, 16])
def test_linear_solvers_agree_with_dense_solve(oracle, golden, N):
    p = ref_problem(golden, N)
    par = oracle.make_params()
    G, Cm, g, c = oracle.form_kkt(par, N, p["xu"], p["goal"], p["xs"])
    S, Pv, gam, Gi = oracle.form_schur(N, 0.1, G, Cm, g, c)
    lam = np.linalg.solve(dense_from_blocks(N, S), gam)
    np.testing.assert_allclose(oracle.banded_cholesky(N, S, gam), lam, rtol=1e-8, atol=1e-10 * np.abs(lam).max())
    ldl = oracle.ldl_solve(N, S, gam)
    assert np.linalg.norm(ldl - lam) <= 1e-3 * np.linalg.norm(lam)
    lp, it, mx = oracle.pcg(N, S, Pv, gam, np.zeros(14 * N), 20000, 1e-10)
    assert not mx
    assert np.linalg.norm(lp - lam) <= 1e-6 * np.linalg.norm(lam)


def test_csc_pattern_is_upper_triangle_of_block_tridiagonal(oracle):
    for N in (1, 2, 4):
        cp, ri = oracle.csc_pattern(N)
        assert cp[-1] == 196 * (N - 1) + 105 * N
        for j in range(14 * N):
            rows = ri[cp[j]:cp[j + 1]]
            assert (rows <= j).all() and (np.diff(rows) > 0).all()
            assert rows[-1] == j and rows[0] == max(0, (j // 14 - 1) * 14)


def test_sqp_oracle_reduces_merit(oracle, golden):
    N = 16
    p = ref_problem(golden, N)
    par = oracle.make_params()
    sv = oracle.make_solver(linsys=2, sqp_max_iter=10)
    m0, _ = oracle.merit(par, N, p["xu"], None, 0.0, p["goal"], p["xs"], 0)
    xu, lam, rho, st, _ = oracle.sqp_solve(par, sv, N, p["goal"], p["lam"], p["xu"], 1e-3)
    assert st.sqp_iters >= 1 and st.merit_final < m0


def test_stair_preconditioner_cuts_block_jacobi_iterations(oracle, problem_mod):
    """The stair ("SS") preconditioner (gato_form_ss_inner, oldschur.cuh:334-494; shipped but
    never called by the reference) on a seeded N = 32 Schur system in FP64: the PCG reaches the same
    relative residual 1e-8 in fewer iterations than with the block-Jacobi Pinv it extends, and both
    solutions agree with the banded Cholesky."""
    N = 32
    p = problem_mod.make_problem(N, 5, dt=0.01)
    par = oracle.make_params(dt=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)
    G, Cm, g, c = oracle.form_kkt(par, N, p["xu"], p["goal"], p["xs"])
    S, P, gam, _ = oracle.form_schur(N, 1e-3, G, Cm, g, c)
    Pss = oracle.form_ss(N, S, P)
    assert np.abs(Pss[:196]).max() == 0 and np.abs(Pss[-196:]).max() == 0
    ref = oracle.banded_cholesky(N, S, gam)
    lam_bj, it_bj, mx_bj = oracle.pcg(N, S, P, gam, np.zeros(14 * N), 20000, 1e-8)
    lam_ss, it_ss, mx_ss = oracle.pcg(N, S, Pss, gam, np.zeros(14 * N), 20000, 1e-8)
    assert not mx_bj and not mx_ss
    assert it_ss < it_bj, (it_ss, it_bj)
    for lam in (lam_bj, lam_ss):
        assert np.abs(lam - ref).max() <= 1e-4 * np.abs(ref).max()
