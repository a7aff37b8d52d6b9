"""Adjoint of the SQP step (gpt_sqp_adjoint) against FP64 central finite
differences of the same map on the oracle.

The map: at an iterate xu, xu+ = xu - dz(theta), dz from the KKT system formed
at xu with cost weights theta (per-joint velocity weights qd, per-joint control
weights r, the end-effector weight q_ee) and goal trajectory p*.  The loss is a
seeded linear functional l = w . xu+, so dl/dxu+ = w.  The oracle evaluates the
map in FP64 (its KKT formation, Schur complement, banded Cholesky, dz), with
per-joint weights applied to its KKT blocks; central differences with relative
step 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SPEC = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def step_map(oracle, N, xu, goal, xs, rho, qd, r, q_ee, ref_terminal):
    """FP64 xu+ = xu - dz with per-joint weights qd (7), r (7) and q_ee."""
    par = oracle.make_params(dt=SPEC["timestep"], integrator=SPEC["integrator"], qd_cost=0.0, r_cost=0.0, q_ee=q_ee,
                             ref_terminal=ref_terminal)
    G, Cm, g, c = (np.array(a, np.float64) for a in oracle.form_kkt(par, N, xu, goal, xs))
    x = lambda k: xu[21 * k:21 * k + 14]
    for k in range(N):
        xt = x(k) if k < N - 1 else (x(N - 2) if ref_terminal else x(N - 1))
        for i in range(7):
            G[245 * k + (7 + i) * 14 + 7 + i] += qd[i]
            g[21 * k + 7 + i] += qd[i] * xt[7 + i]
            if k < N - 1:
                G[245 * k + 196 + i * 7 + i] += r[i]
                g[21 * k + 14 + i] += r[i] * xu[21 * k + 14 + i]
    S, _, gam, Gi = oracle.form_schur(N, rho, G, Cm, g, c)
    lam = oracle.banded_cholesky(N, S, gam)
    dz = oracle.compute_dz(N, Gi, Cm, g, lam)
    return np.asarray(xu, np.float64) - np.asarray(dz)


def fd(f, theta, rel=1e-4, floor=1e-6):
    out = np.zeros(len(theta))
    for i in range(len(theta)):
        h = rel * max(abs(theta[i]), floor)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        out[i] = (f(tp) - f(tm)) / (2 * h)
    return out


@pytest.mark.parametrize("ref_terminal,N,rho", [(1, 12, 1e-2), (0, 12, 1e-2), (1, 32, 1e-2), (1, 12, 1e-3), (1, 128, 1e-3)])
def test_adjoint_matches_fd(gpt, oracle, problem_mod, ref_terminal, N, rho):
    """Gradients of w . xu+ w.r.t. qd (7), r (7), q_ee and the goal (xyz per
    knot) match FP64 central differences to 1e-3 relative (per group), also at
    longer horizons and a smaller regularisation, up to the bench's horizon
    N = 128 at rho = 1e-3."""
    p = problem_mod.make_problem(N, 3, dt=SPEC["timestep"])
    xu, goal, xs = (p[k].astype(np.float64) for k in ("xu", "goal", "xs"))
    # an iterate off the goal (the initial guess tracks it to rounding), rounded to FP32 as the GPU sees it
    xu = (xu + np.random.default_rng(9).normal(0, 0.05, xu.shape)).astype(np.float32).astype(np.float64)
    w = np.random.default_rng(5).normal(0, 1, 21 * N - 7)
    sv = gpt.Solver(max_knot_points=N, ref_terminal=ref_terminal, **SPEC)
    sv.set_solver(pcg_exit_tol=1e-9, pcg_max_iter=100000)
    xnext = torch.zeros(21 * N - 7, device="cuda")
    out = sv.sqp_adjoint([N], dev(goal), dev(xs), dev(xu), [rho], dev(w), xu_next=xnext)
    sv.close()
    qd0, r0, qee0 = np.full(7, SPEC["qd_cost"]), np.full(7, SPEC["r_cost"]), 1.0
    loss = lambda qd, r, qee, gl: float(w @ step_map(oracle, N, xu, gl, xs, rho, qd, r, qee, ref_terminal))
    # the step itself: the GPU's xu+ against the FP64 map (FP32 KKT data, small cond(S) here)
    xp = step_map(oracle, N, xu, goal, xs, rho, qd0, r0, qee0, ref_terminal)
    e_fwd = np.linalg.norm(host(xnext) - xp) / np.linalg.norm(xp - xu)
    assert e_fwd <= 1e-3, e_fwd
    want = {
        "qd": fd(lambda t: loss(t, r0, qee0, goal), qd0),
        "r": fd(lambda t: loss(qd0, t, qee0, goal), r0),
        "q_ee": fd(lambda t: loss(qd0, r0, t[0], goal), np.array([qee0])),
    }
    xyz = np.array([6 * k + d for k in range(N) for d in range(3)])

    def loss_goal(t):
        gl = goal.copy()
        gl[xyz] = t
        return loss(qd0, r0, qee0, gl)
    want["goal"] = fd(loss_goal, goal[xyz], rel=1e-4, floor=1e-2)
    got = {"qd": host(out["qd"])[0], "r": host(out["r"])[0], "q_ee": host(out["q_ee"]),
           "goal": host(out["goal"])[xyz]}
    errs = {k: np.linalg.norm(got[k] - want[k]) / max(np.linalg.norm(want[k]), 1e-12) for k in want}
    assert max(errs.values()) <= 1e-3, (ref_terminal, e_fwd, errs)
    # rpy entries of the goal carry no gradient
    rpy = np.array([6 * k + d for k in range(N) for d in range(3, 6)])
    assert np.all(host(out["goal"])[rpy] == 0)
    if ref_terminal:
        # the reference's terminal block never reads goal_{N-1}
        assert np.all(host(out["goal"])[6 * (N - 1):6 * N] == 0)


def test_adjoint_batched_equals_single(gpt, problem_mod):
    """Two instances of different horizon in one call give the same gradients
    as each instance alone (per-instance weight gradients, per-knot goal)."""
    Ns = [8, 12]
    ps = [problem_mod.make_problem(n, 10 + i, dt=SPEC["timestep"]) for i, n in enumerate(Ns)]
    sv = gpt.Solver(max_knot_points=12, max_batch=2, **SPEC)
    sv.set_solver(pcg_exit_tol=1e-9, pcg_max_iter=100000, pcg_cluster_size=1)
    rng = np.random.default_rng(1)
    ws = [rng.normal(0, 1, 21 * n - 7).astype(np.float32) for n in Ns]
    cat = lambda key, pad: np.concatenate([np.concatenate([p[key], np.zeros(pad(n), np.float32)])
                                           for p, n in zip(ps, Ns)])
    xu = cat("xu", lambda n: 7)
    goal = cat("goal", lambda n: 0)
    xs = np.concatenate([p["xs"] for p in ps])
    w = np.concatenate([np.concatenate([wi, np.zeros(7, np.float32)]) for wi in ws])
    both = sv.sqp_adjoint(Ns, dev(goal), dev(xs), dev(xu), [1e-2, 1e-2], dev(w))
    off = 0
    for i, (n, p) in enumerate(zip(Ns, ps)):
        one = sv.sqp_adjoint([n], dev(p["goal"]), dev(p["xs"]), dev(p["xu"]), [1e-2], dev(ws[i]))
        np.testing.assert_allclose(host(both["qd"])[i], host(one["qd"])[0], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(host(both["r"])[i], host(one["r"])[0], rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(host(both["q_ee"])[i], host(one["q_ee"])[0], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(host(both["goal"])[6 * off:6 * (off + n)], host(one["goal"]), rtol=1e-5, atol=1e-6)
        off += n
    sv.close()


def test_autograd_function_uses_the_adjoint(gpt, problem_mod):
    """sqp_solve under torch.autograd: the forward pass is gpt_sqp_solve_batched,
    the backward pass returns gpt_sqp_adjoint's gradients at the returned solution
    (goal per knot; the three shared weights as sums of the per-joint,
    per-instance gradients)."""
    import importlib
    ag = importlib.import_module("gpu-pcg-tracking_b200.autograd")
    Ns = [8, 12]
    ps = [problem_mod.make_problem(n, 20 + i, dt=SPEC["timestep"]) for i, n in enumerate(Ns)]
    cat = lambda key, pad: np.concatenate([np.concatenate([p[key], np.zeros(pad, np.float32)]) for p in ps])
    sv = gpt.Solver(max_knot_points=12, max_batch=2, **SPEC)
    sv.set_solver(sqp_max_iter=5, pcg_exit_tol=1e-8, pcg_max_iter=100000, pcg_cluster_size=1)
    goal0 = dev(cat("goal", 0))
    xu0, lam0 = dev(cat("xu", 7)), dev(cat("lam", 0))
    w = torch.as_tensor(np.random.default_rng(3).normal(0, 1, xu0.numel()).astype(np.float32), device="cuda")
    # plain calls: solve, then the adjoint at the solution with the final rho
    xu_r, lam_r = xu0.clone(), lam0.clone()
    rho_r, _ = sv.sqp_solve_batched(Ns, goal0, lam_r, xu_r, [1e-3, 1e-3])
    xs = torch.cat([xu0[0:14], xu0[21 * 8:21 * 8 + 14]])
    ref = sv.sqp_adjoint(Ns, goal0, xs, xu_r, rho_r, w)
    # the same through autograd
    goal = goal0.clone().requires_grad_(True)
    weights = torch.tensor([1.0, SPEC["qd_cost"], SPEC["r_cost"]], device="cuda", requires_grad=True)
    xu, lam = ag.sqp_solve(sv, Ns, goal, weights, xu0, lam0, [1e-3, 1e-3])
    assert torch.equal(xu, xu_r)
    (w * xu).sum().backward()
    assert torch.equal(goal.grad, ref["goal"])
    want_w = torch.stack([ref["q_ee"].sum(), ref["qd"].sum(), ref["r"].sum()])
    assert torch.allclose(weights.grad, want_w, rtol=1e-6, atol=0)
    sv.close()
