"""Failure paths of the solve, driven from the host (SURVEY's status and exit-flag contract).

Every failure here comes from the inputs or the settings -- a NaN in xu, a PCG budget of one
iteration, a problem on which no line-search step can lower the merit, rho = 0 with a rank-deficient
cost -- never from a GPU fault: the kernels run to completion and report through gpt_sqp_stats and the
returned gpt_status (the reference reports only through its tuple: pcg_exit_vec, sqp_time_exit,
toplevel.cuh:293-306,396-407,502).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SPEC_CFG = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)


def raw_solve(gpt, sv, N, goal, lam, xu, rho, rho_reset=1e-3):
    """gpt_sqp_solve through the C ABI: (status, stats dict, rho out, pcg iters, pcg exit flags)."""
    L = gpt.lib()
    r = C.c_float(rho)
    st = gpt.SqpStats()
    n = sv.solver.sqp_max_iter
    iters = (C.c_uint32 * n)()
    ex = (C.c_uint8 * n)()
    status = L.gpt_sqp_solve(sv._h, N, gpt._ptr(goal), gpt._ptr(lam), gpt._ptr(xu), C.byref(r), rho_reset,
                             C.byref(st), C.cast(iters, C.c_void_p), C.cast(ex, C.c_void_p),
                             gpt._stream(None))
    torch.cuda.synchronize()
    return status, st.as_dict(), r.value, list(iters), list(ex)


def tensors(p):
    return (torch.as_tensor(p[k], device="cuda") for k in ("goal", "lam", "xu"))


def static_problem(N, q0):
    """Every knot at rest in joint configuration q0 (zero velocity and control); x_s = x_0."""
    xu = np.zeros(21 * N, np.float32)
    for k in range(N):
        xu[21 * k:21 * k + 7] = q0
    goal = np.zeros(6 * N, np.float32)
    return {"xu": xu[:21 * N - 7].copy(), "goal": goal, "lam": np.zeros(14 * N, np.float32)}


def test_nan_in_xu_reports_nonfinite(gpt, problem_mod):
    N = 32
    sv = gpt.Solver(max_knot_points=N, **SPEC_CFG)
    try:
        for graph in (1, 0):
            sv.set_solver(sqp_max_iter=10, pcg_max_iter=10000, pcg_exit_tol=1e-5, sqp_graph=graph)
            p = problem_mod.make_problem(N, 2, dt=0.01)
            p["xu"][21 * 5 + 3] = np.nan
            goal, lam, xu = tensors(p)
            status, st, _, _, _ = raw_solve(gpt, sv, N, goal, lam, xu, 1e-3)
            assert status == 5, status  # GPT_ERR_NONFINITE
            assert st["exit_flags"] & gpt.EXIT_NONFINITE
            assert "non-finite" in gpt.lib().gpt_last_error().decode()
            with pytest.raises(gpt.GptError) as ei:
                sv.sqp_solve(N, goal, lam, xu, 1e-3)
            assert ei.value.status == 5
    finally:
        sv.close()


def test_nan_in_one_instance_leaves_the_batch_intact(gpt, problem_mod):
    """Instances are independent: a NaN in one flags that instance only; the others' results equal a
    batch solved without it."""
    Ns = [24, 40, 32]
    batch = problem_mod.make_batch(Ns, seed0=60, dt=0.01)
    sv = gpt.Solver(max_knot_points=64, max_batch=3, **SPEC_CFG)
    try:
        sv.set_solver(sqp_max_iter=8, pcg_max_iter=10000, pcg_exit_tol=1e-5, pcg_cluster_size=gpt.PCG_WARP_PAIR)
        outs = []
        for poison in (False, True):
            xu_h = batch["xu"].copy()
            if poison:
                xu_h[21 * 24 + 21 * 3 + 1] = np.nan  # instance 1, knot 3
            xu = torch.as_tensor(xu_h, device="cuda")
            lam = torch.as_tensor(batch["lam"], device="cuda")
            goal = torch.as_tensor(batch["goal"], device="cuda")
            B = len(Ns)
            Nsc = (C.c_uint32 * B)(*Ns)
            rr = (C.c_float * B)(*([1e-3] * B))
            sts = (gpt.SqpStats * B)()
            status = gpt.lib().gpt_sqp_solve_batched(sv._h, B, C.cast(Nsc, C.c_void_p), gpt._ptr(goal), gpt._ptr(lam),
                                                     gpt._ptr(xu), C.cast(rr, C.c_void_p), 1e-3,
                                                     C.cast(sts, C.c_void_p), gpt._stream(None))
            torch.cuda.synchronize()
            outs.append((status, [s.as_dict() for s in sts], xu.cpu().numpy(), lam.cpu().numpy()))
        assert outs[0][0] == 0 and outs[1][0] == 5
        flags = [s["exit_flags"] & gpt.EXIT_NONFINITE for s in outs[1][1]]
        assert flags[1] and not flags[0] and not flags[2]
        for a, b in ((0, 24), (64, 96)):  # instances 0 and 2
            assert np.array_equal(outs[0][2][21 * a:21 * b], outs[1][2][21 * a:21 * b])
            assert np.array_equal(outs[0][3][14 * a:14 * b], outs[1][3][14 * a:14 * b])
    finally:
        sv.close()


def test_pcg_budget_of_one_iteration_sets_the_maxiter_flags(gpt, problem_mod):
    """Block-Jacobi PCG (the reference's preconditioner) limited to one iteration cannot reach the
    tolerance: every linear solve reports the max-iteration exit (pcg_exit_vec, toplevel.cuh:293-306)."""
    N = 32
    sv = gpt.Solver(max_knot_points=N, **SPEC_CFG)
    try:
        sv.set_solver(sqp_max_iter=5, pcg_max_iter=1, pcg_exit_tol=1e-5, pcg_precond=0, pcg_cluster_size=1,
                      sqp_graph=0)
        goal, lam, xu = tensors(problem_mod.make_problem(N, 4, dt=0.01))
        status, st, _, iters, ex = raw_solve(gpt, sv, N, goal, lam, xu, 1e-3)
        assert status == 0, gpt.lib().gpt_last_error()
        n = st["sqp_iters"]
        assert n >= 1
        assert st["exit_flags"] & gpt.EXIT_PCG_MAXITER
        assert st["pcg_maxiter_count"] == n
        assert iters[:n] == [1] * n and ex[:n] == [1] * n
        # the exact preconditioner meets the same tolerance in one iteration: no flag
        sv.set_solver(pcg_precond=1, pcg_cluster_size=0, pcg_max_iter=1)
        goal, lam, xu = tensors(problem_mod.make_problem(N, 4, dt=0.01))
        status, st, _, iters, ex = raw_solve(gpt, sv, N, goal, lam, xu, 1e-3)
        assert status == 0 and not (st["exit_flags"] & gpt.EXIT_PCG_MAXITER) and st["pcg_maxiter_count"] == 0
    finally:
        sv.close()


def test_line_search_failure_until_rho_max_resets_rho(gpt):
    """A problem at rest with no end-effector weight has merit 0 and dz = 0: no step lowers the merit,
    the line search fails every iteration, rho grows by the schedule (toplevel.cuh:396-407) until it
    passes rho_max, then the solve exits with rho reset to rho_reset."""
    N = 16
    sv = gpt.Solver(max_knot_points=N, **SPEC_CFG)
    try:
        sv.set_cost_weights(0.0, 1e-2, 1e-4)
        for graph in (1, 0):
            sv.set_solver(sqp_max_iter=40, pcg_max_iter=10000, pcg_exit_tol=1e-5, sqp_graph=graph)
            q0 = np.array([0.3, -0.5, 0.2, 1.0, -0.4, 0.6, 0.1], np.float32)
            goal, lam, xu = tensors(static_problem(N, q0))
            status, st, rho, _, _ = raw_solve(gpt, sv, N, goal, lam, xu, 1e-3, rho_reset=5e-3)
            assert status == 0, gpt.lib().gpt_last_error()
            # the float32 schedule from rho = 1e-3, drho = 1: fails until rho > 10
            f, r, d, n = np.float32(1.2), np.float32(1e-3), np.float32(1.0), 0
            while True:
                d = max(np.float32(d * f), f)
                r = max(np.float32(r * d), np.float32(1e-3))
                n += 1
                if r > np.float32(10.0):
                    break
            assert st["exit_flags"] & gpt.EXIT_RHO_MAX
            assert st["sqp_iters"] == n and st["ls_fail_count"] == n, (st, n)
            assert rho == np.float32(5e-3) and st["rho_final"] == np.float32(5e-3)
            assert st["merit_initial"] == 0.0 and st["merit_final"] == 0.0
    finally:
        sv.close()


def test_rho_zero_with_singular_cost_reports_factor(gpt, problem_mod):
    """rho = 0 leaves (Q + rho I) with the rank-one end-effector block and, with R_COST = 0, (R + rho I)
    = 0: the Schur complement's inverses meet vanishing pivots and the call returns GPT_ERR_FACTOR with
    GPT_EXIT_FACTOR set, instead of a solve on garbage."""
    N = 16
    sv = gpt.Solver(max_knot_points=N, timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=0.0)
    try:
        for graph in (1, 0):
            sv.set_solver(sqp_max_iter=5, pcg_max_iter=10000, pcg_exit_tol=1e-5, sqp_graph=graph)
            goal, lam, xu = tensors(problem_mod.make_problem(N, 1, dt=0.01))
            status, st, _, _, _ = raw_solve(gpt, sv, N, goal, lam, xu, 0.0)
            assert status == 6, (status, gpt.lib().gpt_last_error())  # GPT_ERR_FACTOR
            assert st["exit_flags"] & gpt.EXIT_FACTOR
            assert st["sqp_iters"] == 1  # the instance stops after the failed iteration
        # the same problem with rho > 0 solves
        sv.set_solver(sqp_max_iter=5, sqp_graph=1)
        goal, lam, xu = tensors(problem_mod.make_problem(N, 1, dt=0.01))
        status, st, _, _, _ = raw_solve(gpt, sv, N, goal, lam, xu, 1e-3)
        assert status == 0 and not (st["exit_flags"] & gpt.EXIT_FACTOR)
    finally:
        sv.close()
