"""The MPC tracking loop (track, toplevel.cuh:507-796) and the plant simulator
(simple_simulate, integrator.cuh:365-398): the oracle's restatement on the CPU,
and gpt_track / gpt_track_batched / gpt_simulate against it on the GPU.

Workload: a prefix of the reference's own trajectory testfiles/0_0_traj.csv and
its end-effector file (the rows runme.cu:145-161 loads), dt = 1/64, explicit
Euler, QD = R = 1e-4, plant state x_s = the first row's state (runme.cu:165)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

REF_CFG = dict(timestep=1.0 / 64, integrator=0, qd_cost=1e-4, r_cost=1e-4)


def traj(golden, S, start=0, name="0_0"):
    tr = golden[f"traj_{name}"][start:start + S].astype(np.float32)
    ee = golden["eepos_0_0"][start:start + S].astype(np.float32) if name == "0_0" else None
    return tr, ee


def oracle_track(oracle, N, tr, ee, sim_us, sqp_iters, precision, jitter=0, linsys=2):
    P = oracle.make_params()
    SV = oracle.make_solver(linsys=linsys, sqp_max_iter=sqp_iters)
    cfg = oracle.make_track_cfg(sim_period_us=sim_us, jitter_solves=jitter)
    return oracle.track(P, SV, cfg, N, ee, tr, tr[0, :14].copy(), precision=precision)


# ---------------------------------------------------------------------------
# CPU: the oracle
# ---------------------------------------------------------------------------

def test_oracle_simulate_is_euler_steps_of_forward_dynamics(oracle):
    """simple_simulate = floor(T / h) explicit-Euler steps of FD (control of knot
    floor(t / dt)) plus one step of the remainder fmod(T, h) (integrator.cuh:365-398)."""
    rng = np.random.default_rng(5)
    N, dt = 8, 1.0 / 64
    xu = rng.normal(0, 0.3, 21 * N - 7)
    xs = rng.normal(0, 0.3, 14)
    for t0_us, sim_us in ((0.0, 2000.0), (2000.0, 2000.0), (8000.0, 9100.0)):
        got = oracle.simulate(N, xs, xu, dt, t0_us, sim_us)
        h = np.float32(2e-4)
        x = xs.copy()
        n = int((sim_us * 1e-6) / float(h))
        co = min(int((t0_us * 1e-6) / dt), N - 2)
        for step in range(n):
            co = min(int((t0_us * 1e-6 + float(np.float32(step) * h)) / dt), N - 2)
            qdd = oracle.fd(x[:7], x[7:], xu[21 * co + 14:21 * co + 21])
            x = np.concatenate([x[:7] + float(h) * x[7:], x[7:] + float(h) * qdd])
        hl = float(np.float32(np.fmod(sim_us * 1e-6, float(h))))
        qdd = oracle.fd(x[:7], x[7:], xu[21 * co + 14:21 * co + 21])
        x = np.concatenate([x[:7] + hl * x[7:], x[7:] + hl * qdd])
        assert np.allclose(got, x, rtol=1e-12, atol=1e-12), (t0_us, sim_us)


def test_oracle_track_runs_the_reference_schedule(oracle, golden):
    """One error per shift, traj_steps shifts; the update count follows the loop's clock
    (shift once time_since > timestep, then wrap by fmod, toplevel.cuh:668-724): at 8 ms per
    update and dt = 1/64 s the clock shifts on every second update."""
    N, S = 12, 20
    tr, ee = traj(golden, S)
    x, err, ts = oracle_track(oracle, N, tr, ee, 8000.0, 2, "f64")
    assert ts.shifts == S and len(err) == S
    assert ts.control_updates == 2 * S  # the 20th shift falls on update 40; the next update exits
    assert np.all(np.isfinite(err)) and np.all(err >= 0)
    assert err[0] < 0.01  # the run starts on the trajectory


def test_oracle_track_f32_agrees_with_f64(oracle, golden):
    """The FP32 restatement (the reference's precision, qdldl-path LDL^T) and the FP64 one
    (banded Cholesky) trace the same closed loop: end-effector errors agree to 2e-3 m; the joint
    states only to 0.1, since the position-only cost leaves 4 of the 7 joint directions to the
    weak velocity and control weights (1e-4), where rounding differences drift freely."""
    N, S = 16, 24
    tr, ee = traj(golden, S)
    x64, e64, t64 = oracle_track(oracle, N, tr, ee, 8000.0, 4, "f64")
    x32, e32, t32 = oracle_track(oracle, N, tr, ee, 8000.0, 4, "f32", linsys=1)
    assert t64.control_updates == t32.control_updates and t64.shifts == t32.shifts
    assert np.max(np.abs(e64 - e32)) < 2e-3
    assert abs(t64.final_error - t32.final_error) < 2e-3
    assert np.max(np.abs(x64 - x32)) < 0.1


# ---------------------------------------------------------------------------
# GPU: gpt_simulate / gpt_track / gpt_track_batched through the C ABI
# ---------------------------------------------------------------------------

def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


@pytest.mark.gpu
def test_simulate_matches_oracle(gpt, oracle):
    """gpt_simulate against the FP64 oracle: relative 2e-5 of the state scale over up to
    46 FP32 plant steps (control offsets 0 and 1, partial last step)."""
    rng = np.random.default_rng(7)
    N = 8
    sv = gpt.Solver(max_knot_points=N, **REF_CFG)
    try:
        for t0_us, sim_us in ((0.0, 2000.0), (2000.0, 2000.0), (8000.0, 9100.0)):
            xu = rng.normal(0, 0.3, 21 * N - 7).astype(np.float32)
            xs = rng.normal(0, 0.3, 14).astype(np.float32)
            want = oracle.simulate(N, xs.astype(np.float64), xu.astype(np.float64), 1.0 / 64, t0_us, sim_us)
            d_xs = dev(xs)
            sv.simulate(N, d_xs, dev(xu), t0_us, sim_us)
            got = d_xs.cpu().numpy().astype(np.float64)
            scale = np.max(np.abs(want))
            assert np.max(np.abs(got - want)) <= 2e-5 * scale, (t0_us, sim_us, got, want)
    finally:
        sv.close()


def _gpu_track(gpt, N, tr, ee, sim_us, sqp_iters, jitter=0, **solver_kw):
    sv = gpt.Solver(max_knot_points=N, sqp_max_iter=sqp_iters, **REF_CFG, **solver_kw)
    try:
        cfg = gpt.default_track_config(sim_period_us=sim_us, jitter_solves=jitter)
        xs = dev(tr[0, :14])
        log = torch.zeros(256, dtype=torch.int32, device="cuda")
        err, st = sv.track(N, dev(ee), dev(tr), xs, cfg, sqp_iters_log=log)
        torch.cuda.synchronize()
        return xs.cpu().numpy().astype(np.float64), err.cpu().numpy().astype(np.float64), st, log.cpu().numpy()
    finally:
        sv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("jitter", [0, 2])
def test_track_matches_oracle(gpt, oracle, golden, jitter):
    """gpt_track against the FP64 oracle loop on the reference trajectory prefix: the same
    schedule (updates, shifts), and per-shift tracking errors and the final plant state within
    three times the FP32-vs-FP64 oracle gap of the same run (floor 1e-4): the closed loop
    amplifies per-solve rounding alike in every FP32 implementation (the joint state most, along
    the null space of the position-only cost)."""
    N, S, sim_us, iters = 16, 24, 8000.0, 4
    tr, ee = traj(golden, S)
    x64, e64, t64 = oracle_track(oracle, N, tr, ee, sim_us, iters, "f64", jitter=jitter)
    x32, e32, _ = oracle_track(oracle, N, tr, ee, sim_us, iters, "f32", jitter=jitter, linsys=1)
    tol_e = max(3 * np.max(np.abs(e64 - e32)), 1e-4)
    tol_x = max(3 * np.max(np.abs(x64 - x32)), 1e-4)
    xg, eg, st, log = _gpu_track(gpt, N, tr, ee, sim_us, iters, jitter=jitter)
    assert st["control_updates"] == t64.control_updates and st["shifts"] == t64.shifts == S
    assert st["nonfinite"] == 0
    assert np.max(np.abs(eg - e64)) <= tol_e, (np.max(np.abs(eg - e64)), tol_e)
    assert np.max(np.abs(xg - x64)) <= tol_x, (np.max(np.abs(xg - x64)), tol_x)
    assert abs(st["final_tracking_error"] - t64.final_error) <= tol_e
    assert st["sqp_iters_total"] == int(log[:st["control_updates"]].sum())
    assert abs(st["tracking_error_mean"] - np.mean(e64)) <= tol_e


@pytest.mark.gpu
def test_track_batched_equals_single_runs(gpt, golden):
    """Three instances of uneven horizon and trajectory length in one gpt_track_batched call give
    the same bits as three gpt_track calls (fixed PCG kernel); the shorter runs stop at their own
    traj_steps while the batch goes on.  The graph and host-loop solves agree bit for bit."""
    specs = [(12, 20, 0), (16, 26, 3), (8, 14, 7)]
    kw = dict(pcg_cluster_size=gpt.PCG_WARP_PAIR)
    singles = []
    for N, S, start in specs:
        tr, _ = traj(golden, S, start)
        ee = golden["eepos_0_0"][start:start + S].astype(np.float32)
        singles.append(_gpu_track(gpt, N, tr, ee, 4000.0, 3, **kw))
    Ns = [s[0] for s in specs]
    Ss = [s[1] for s in specs]
    tr_all = np.concatenate([golden["traj_0_0"][st:st + S] for _, S, st in specs]).astype(np.float32)
    ee_all = np.concatenate([golden["eepos_0_0"][st:st + S] for _, S, st in specs]).astype(np.float32)
    xs0 = np.concatenate([golden["traj_0_0"][st, :14] for _, _, st in specs]).astype(np.float32)
    for graph in (1, 2, 3, 0):
        sv = gpt.Solver(max_knot_points=16, max_batch=3, sqp_max_iter=3, sqp_graph=graph, **REF_CFG, **kw)
        try:
            xs = dev(xs0)
            err, stats = sv.track_batched(Ns, Ss, dev(ee_all), dev(tr_all), xs,
                                          gpt.default_track_config(sim_period_us=4000.0))
            torch.cuda.synchronize()
            xs_h, err_h = xs.cpu().numpy(), err.cpu().numpy()
        finally:
            sv.close()
        row = 0
        for b, (N, S, _) in enumerate(specs):
            xg, eg, st, _ = singles[b]
            assert stats[b]["shifts"] == S == st["shifts"]
            assert stats[b]["control_updates"] == st["control_updates"]
            assert np.array_equal(xs_h[14 * b:14 * b + 14], xg.astype(np.float32)), (graph, b)
            assert np.array_equal(err_h[row:row + S], eg.astype(np.float32)), (graph, b)
            row += S


@pytest.mark.gpu
def test_track_rejects_short_trajectories(gpt, golden):
    N = 16
    tr, ee = traj(golden, N - 1)
    sv = gpt.Solver(max_knot_points=N, **REF_CFG)
    try:
        with pytest.raises(gpt.GptError):
            sv.track(N, dev(ee), dev(tr), dev(tr[0, :14]))
    finally:
        sv.close()


def test_oracle_track_loop_matches_restated_host_logic(oracle, golden):
    """The oracle's track loop against a line-by-line restatement of the reference's host logic
    (toplevel.cuh:600-726: the clock, just_shift's knot-by-knot copies, the fills -- inside the
    trajectory from row traj_offset, past it the last q with zero velocity and zero control -- the
    goal-window shift and x_0 <- x_s), with the SQP solve switched off (sqp_max_iter 0) so that
    only the loop's bookkeeping and the plant act: identical errors and final state in FP64."""
    N, S, dt, sim = 6, 14, 1.0 / 64, 6000.0
    tr = golden["traj_0_0"][:S].astype(np.float64)
    ee = golden["eepos_0_0"][:S].astype(np.float64)
    P = oracle.make_params()
    SV = oracle.make_solver(linsys=2, sqp_max_iter=0)
    cfg = oracle.make_track_cfg(sim_period_us=sim)
    xs_o, err_o, ts = oracle.track(P, SV, cfg, N, ee, tr, tr[0, :14].copy())

    L = 21 * N - 7
    trf, eef = tr.reshape(-1), ee.reshape(-1)
    xu = trf[:L].copy()
    xu_old = xu.copy()
    goal = eef[:6 * N].copy()
    xs = tr[0, :14].copy()
    errs = []
    time_since, prev, shifted, off = 0.0, 0.0, False, 0
    for _ in range(100000):
        if off == S:
            break
        xs = oracle.simulate(N, xs, xu_old, dt, prev, sim)
        xu_old = xu.copy()
        time_since += sim * 1e-6
        if not shifted and time_since > dt:
            p = oracle.fk(xs[:7])
            errs.append(abs(p[0] - goal[0]) + abs(p[1] - goal[1]) + abs(p[2] - goal[2]))
            off += 1
            for k in range(N - 1):  # just_shift: knot k <- knot k+1, the last step copies the state only
                n = 14 + (7 if k < N - 2 else 0)
                xu[21 * k:21 * k + n] = xu[21 * (k + 1):21 * (k + 1) + n]
            if off + N < S:
                xu[L - 21:L] = trf[21 * off - 7:21 * off + 14]
            else:
                xu[L - 14:L - 7] = trf[21 * (S - 1):21 * (S - 1) + 7]
                xu[L - 7:L] = 0.0
                xu[L - 21:L - 14] = 0.0
            for k in range(N - 1):
                goal[6 * k:6 * k + 6] = goal[6 * (k + 1):6 * (k + 1) + 6]
            row = off + N - 1 if off + N < S else S - 1
            goal[6 * (N - 1):] = eef[6 * row:6 * row + 6]
            shifted = True
        if time_since > dt:
            shifted = False
            time_since = np.fmod(time_since, dt)
        xu[:14] = xs
        prev = sim
    assert ts.shifts == S == len(errs)
    np.testing.assert_array_equal(err_o, np.array(errs))
    np.testing.assert_array_equal(xs_o, xs)
