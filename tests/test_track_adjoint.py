"""gpt_track_batched_adjoint: the MPC tracking loop (toplevel.cuh:507-796) with the one-step adjoint
of every control update's solve, on the update's horizon tracking loss
l = 1/2 sum_k |p(q_k+) - p*_k|^2 at xu+ = xu - dz (no reference counterpart).

* The forward run equals gpt_track_batched's bit for bit.
* With one control update, the returned weight gradient equals gpt_sqp_adjoint at the same
  solution with dl/dxu+ formed on the host from the oracle's FP64 forward kinematics and position
  Jacobian, and the returned loss equals l evaluated the same way.

Workload: prefixes of the reference's trajectory testfiles/0_0_traj.csv and its end-effector file,
dt = 1/64, explicit Euler, QD = R = 1e-4 (the reference's settings)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

REF_CFG = dict(timestep=1.0 / 64, integrator=0, qd_cost=1e-4, r_cost=1e-4)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def batch(golden, specs):
    tr = np.concatenate([golden["traj_0_0"][st:st + S] for _, S, st in specs]).astype(np.float32)
    ee = np.concatenate([golden["eepos_0_0"][st:st + S] for _, S, st in specs]).astype(np.float32)
    xs = np.concatenate([golden["traj_0_0"][st, :14] for _, _, st in specs]).astype(np.float32)
    return tr, ee, xs


def test_track_adjoint_forward_equals_track_batched(gpt, golden):
    """Three instances of uneven horizon and trajectory length: errors, statistics and the final
    plant states of the adjoint run are those of gpt_track_batched; the weight gradients and the
    losses are finite, the losses positive, no adjoint solve fails."""
    specs = [(12, 20, 0), (16, 26, 3), (8, 14, 7)]
    Ns, Ss = [s[0] for s in specs], [s[1] for s in specs]
    tr, ee, xs0 = batch(golden, specs)
    cfg = gpt.default_track_config(sim_period_us=4000.0)
    sv = gpt.Solver(max_knot_points=16, max_batch=3, sqp_max_iter=3, **REF_CFG)
    try:
        xs_a = dev(xs0)
        err_a, st_a = sv.track_batched(Ns, Ss, dev(ee), dev(tr), xs_a, cfg)
        xs_b = dev(xs0)
        err_b, st_b, wgrad, loss, fails = sv.track_batched_adjoint(Ns, Ss, dev(ee), dev(tr), xs_b, cfg)
        torch.cuda.synchronize()
    finally:
        sv.close()
    assert np.array_equal(err_a.cpu().numpy(), err_b.cpu().numpy())
    assert np.array_equal(xs_a.cpu().numpy(), xs_b.cpu().numpy())
    for b in range(len(specs)):
        assert st_a[b] == st_b[b], b
    w, lo = wgrad.cpu().numpy(), loss.cpu().numpy()
    assert np.all(np.isfinite(w)) and np.all(np.isfinite(lo)), (w, lo)
    assert np.all(lo > 0), lo
    assert np.all(np.abs(w).max(axis=1) > 0), w
    assert fails == [0, 0, 0], fails


@pytest.mark.parametrize("N,start", [(16, 0), (24, 5)])
def test_track_adjoint_one_update_equals_sqp_adjoint(gpt, golden, oracle, N, start):
    """One control update: the solve from the trajectory's first N rows, then the adjoint at its
    solution.  The same solve through gpt_sqp_solve_batched and gpt_sqp_adjoint (first with a zero
    loss gradient for xu+, then with dl/dxu+ = J(q+)^T (p(q+) - p*) from the oracle's FP64
    kinematics) gives the same 15 weight gradients (relative 2e-3 of their largest magnitude:
    FP32 kinematics on the GPU) and the same loss (relative 1e-5)."""
    S = N + 4
    tr, ee, xs0 = batch(golden, [(N, S, start)])
    cfg = gpt.default_track_config(sim_period_us=4000.0, max_control_updates=1)
    kw = dict(max_knot_points=N, sqp_max_iter=4, **REF_CFG)
    sv = gpt.Solver(**kw)
    try:
        _, st, wgrad, loss, fails = sv.track_batched_adjoint([N], [S], dev(ee), dev(tr), dev(xs0), cfg)
        torch.cuda.synchronize()
        assert st[0]["control_updates"] == 1 and fails == [0]
        w_track, l_track = wgrad.cpu().numpy()[0].astype(np.float64), float(loss.cpu().numpy()[0])
    finally:
        sv.close()

    xu0 = tr[:N].reshape(-1)[:21 * N - 7].copy()
    goal = ee[:N].reshape(-1).copy()
    sv = gpt.Solver(**kw)
    try:
        xu = dev(xu0)
        rho, _ = sv.sqp_solve_batched([N], dev(goal), torch.zeros(14 * N, device="cuda"), xu, [1e-3])
        xs = dev(xu0[:14])
        xu_next = torch.zeros(21 * N - 7, device="cuda")
        sv.sqp_adjoint([N], dev(goal), xs, xu, rho, torch.zeros(21 * N - 7, device="cuda"), xu_next=xu_next)
        xn = xu_next.cpu().numpy().astype(np.float64)
        grad = np.zeros(21 * N - 7)
        l_host = 0.0
        for k in range(N):
            q = xn[21 * k:21 * k + 7]
            e = oracle.fk(q)[:3] - goal[6 * k:6 * k + 3].astype(np.float64)
            l_host += 0.5 * float(e @ e)
            J = oracle.fk_grad(q).reshape(7, 6)[:, :3]
            grad[21 * k:21 * k + 7] = J @ e
        out = sv.sqp_adjoint([N], dev(goal), xs, xu, rho, dev(grad))
        torch.cuda.synchronize()
        w_ref = np.concatenate([out["qd"].cpu().numpy()[0], out["r"].cpu().numpy()[0],
                                out["q_ee"].cpu().numpy()[:1]]).astype(np.float64)
    finally:
        sv.close()
    scale = np.abs(w_ref).max()
    assert scale > 0
    assert np.abs(w_track - w_ref).max() <= 2e-3 * scale, (w_track, w_ref)
    assert abs(l_track - l_host) <= 1e-5 * abs(l_host) + 1e-9, (l_track, l_host)
