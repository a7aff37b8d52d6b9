"""The default product path, pinned per SQP iterate to the oracle.

The batched solve runs exactly as the bench runs it (FP64 Schur rows, the autotuned PCG --
the warp-pair kernel for a 512-instance batch at N = 128 -- and the FP64 dz), through
gpt_sqp_solve_batched_trace, which records every iterate of the host-driven loop.  For sampled
instances and every iteration the oracle is fed the GPU's own KKT blocks at the recorded iterate
(the CUDA KKT kernel through gpt_form_kkt) and solves the same linear system in FP64 (Schur
complement, banded Cholesky, dz: the reference's sqpSolve linear algebra, toplevel.cuh:254-335 with
the qdldl solve of qdldl_helper.cuh:62-180 replaced by its exact FP64 counterpart).  Bars:
  * lambda and dz within 1e-4 relative (max |err| / max |oracle|) of the FP64 solution;
  * the line-search merits within 5e-5 relative plus the FP32 rounding of their defect sums of the
    oracle's FP64 merits of the same candidates (the merit is FP32 arithmetic, as the reference's: each
    defect component x_{k+1} - f(x_k, u_k) cancels, leaving ~eps32 |x| per component, weighted by mu);
  * the accept decision the argmin of the GPU's own merits exactly, and the oracle's argmin up to a
    tie within the merits' FP32 error; rho after the schedule identical bit for bit
    (toplevel.cuh:384-412, float arithmetic); the next iterate equal to fl32(xu + alpha dz) bit for bit.
"""
import numpy as np
import pytest

from conftest import ref_problem

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SPEC_CFG = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)
REF_CFG = dict(timestep=1.0 / 64, integrator=0, qd_cost=1e-4, r_cost=1e-4)
LAM_DZ_RTOL = 1e-4
MERIT_RTOL = 5e-5


def _rel(got, want):
    den = np.abs(want).max()
    return np.abs(got - want).max() / den if den > 0 else np.abs(got).max()


def rho_law(rho, drho, accepted, f=1.2, rho_min=1e-3, rho_max=10.0, rho_reset=1e-3):
    """toplevel.cuh:396-412 in float32: the schedule the accept kernel applies (a failed line search
    that pushes rho above rho_max resets it and ends the solve)."""
    f32 = np.float32
    rho, drho, f, rho_min = f32(rho), f32(drho), f32(f), f32(rho_min)
    if accepted:
        drho = min(f32(drho / f), f32(f32(1.0) / f))
    else:
        drho = max(f32(drho * f), f)
    rho = max(f32(rho * drho), rho_min)
    if not accepted and rho > f32(rho_max):
        rho = f32(rho_reset)
    return rho, drho


def check_trace(gpt, oracle, sv, par, Ns, batch, sample, iters):
    B = len(Ns)
    offs = np.concatenate([[0], np.cumsum(Ns)])
    xu = torch.as_tensor(batch["xu"], device="cuda")
    goal = torch.as_tensor(batch["goal"], device="cuda")
    lam = torch.as_tensor(batch["lam"], device="cuda")
    _, stats, tr = sv.sqp_solve_batched_trace(Ns, goal, lam, xu, [1e-3] * B, iters)
    torch.cuda.synchronize()
    rec = gpt.trace_record_fields(tr["rec"])
    worst = {"lam": 0.0, "dz": 0.0, "merit": 0.0}
    checked = 0
    for b in sample:
        N, o = Ns[b], int(offs[b])
        gb = batch["goal"][6 * o:6 * o + 6 * N]
        xs = batch["xu"][21 * o:21 * o + 14]
        xu_b = tr["xu"][:, 21 * o:21 * o + 21 * N - 7].cpu().numpy()
        lam_b = tr["lam"][:, 14 * o:14 * o + 14 * N].cpu().numpy()
        dz_b = tr["dz"][:, 21 * o:21 * o + 21 * N - 7].cpu().numpy()
        drho = np.float32(1.0)
        n_active = int(stats[b]["sqp_iters"])
        for i in range(min(iters, n_active)):
            assert rec["active"][i, b] == 1, (b, i)
            rho = float(rec["rho"][i, b])
            G, Cm, g, c = (torch.zeros(n, device="cuda") for n in (245 * N - 49, 294 * (N - 1), 21 * N - 7, 14 * N))
            sv.form_kkt(N, torch.as_tensor(xu_b[i], device="cuda"), torch.as_tensor(gb, device="cuda"),
                        torch.as_tensor(xs, device="cuda"), G, Cm, g, c)
            G, Cm, g, c = (t.cpu().numpy().astype(np.float64) for t in (G, Cm, g, c))
            S, _, gam, Gi = oracle.form_schur(N, rho, G, Cm, g, c, "f64")
            lam_o = oracle.banded_cholesky(N, S, gam, "f64")
            dz_o = oracle.compute_dz(N, Gi, Cm, g, lam_o, "f64")
            e_l, e_d = _rel(lam_b[i], lam_o), _rel(dz_b[i], dz_o)
            assert e_l <= LAM_DZ_RTOL, f"instance {b} iteration {i}: lambda rel err {e_l:.3e}"
            assert e_d <= LAM_DZ_RTOL, f"instance {b} iteration {i}: dz rel err {e_d:.3e}"
            worst["lam"], worst["dz"] = max(worst["lam"], e_l), max(worst["dz"], e_d)
            # line-search merits of the GPU's candidates xu + alpha_p dz, in FP64 by the oracle
            mo = np.array([oracle.merit(par, N, xu_b[i], dz_b[i], -2.0 ** -a, gb, xs, 1)[0] for a in range(8)])
            mg = rec["merits"][i, b].astype(np.float64)
            # FP32 rounding of the defect sums: mu x 4 eps32 per unit of |x| at the candidates
            xs_abs = np.array([np.abs(xu_b[i].astype(np.float64) - 2.0 ** -a * dz_b[i]).sum() for a in range(8)])
            tolm = MERIT_RTOL * np.abs(mo) + par.mu * 4 * 2.0 ** -23 * xs_abs
            em = (np.abs(mg - mo) / tolm).max()
            assert em <= 1.0, f"instance {b} iteration {i}: merit error {em:.3f} x its bound"
            worst_m = (np.abs(mg - mo) / np.abs(mo)).max()
            worst["merit"] = max(worst["merit"], worst_m)
            # the accept decision: exactly the argmin of the GPU's merits against the iterate's merit
            # (strict <, first minimum, toplevel.cuh:384-392) ...
            m_prev = np.float32(rec["merit_prev"][i, b])
            mg32 = rec["merits"][i, b]
            best_g, a_g = m_prev, -1
            for a in range(8):
                if mg32[a] < best_g:
                    best_g, a_g = mg32[a], a
            alpha = float(rec["alpha"][i, b])
            acc_g = alpha != 0.0
            assert alpha == (0.0 if a_g < 0 else -2.0 ** -a_g), (b, i, alpha, mg32, m_prev)
            # ... and the oracle's own choice, unless its FP64 merits are within the FP32 error of a tie
            a_o = int(np.argmin(mo))
            acc_o = mo[a_o] < m_prev
            if acc_g != acc_o or (acc_g and a_g != a_o):
                alt = mo[a_g] if acc_g else float(m_prev)
                assert abs(alt - mo[a_o]) <= 2 * tolm.max(), (b, i, alpha, mo, m_prev)
            rho_n, drho = rho_law(rho, drho, acc_g)
            assert np.float32(rec["rho_next"][i, b]) == rho_n, (b, i, rec["rho_next"][i, b], rho_n)
            if i + 1 < min(iters, n_active):
                want = (xu_b[i] + np.float32(alpha) * dz_b[i]).astype(np.float32) if acc_g else xu_b[i]
                assert np.array_equal(xu_b[i + 1], want), (b, i)
                assert np.float32(rec["rho"][i + 1, b]) == rho_n
            checked += 1
    assert checked > 0
    return worst, checked


def test_default_batched_path_matches_oracle_per_iterate(gpt, oracle, problem_mod):
    """Bench configuration: 512 seeded instances x N = 128, dt 0.01 semi-implicit Euler, QD 0.01,
    R 1e-4, PCG relative residual 1e-5, 40 SQP iterations; instance 0 and 8 seeded samples."""
    B, N = 512, 128
    Ns = [N] * B
    batch = problem_mod.make_batch(Ns, seed0=0, dt=0.01)
    sv = gpt.Solver(max_knot_points=N, max_batch=B, **SPEC_CFG)
    try:
        sv.set_solver(sqp_max_iter=40, pcg_max_iter=10000, pcg_exit_tol=1e-5, pcg_exit_mode=0)
        assert sv.solver.schur_fp64 == 1 and sv.solver.pcg_precond == 1
        cs = sv.autotune(Ns, *(torch.as_tensor(batch[k], device="cuda") for k in ("goal", "lam", "xu")), [1e-3] * B)
        assert cs in (gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD), f"the autotuner chose {cs} for the bench shape"
        sample = [0] + sorted(np.random.default_rng(11).choice(np.arange(1, B), 8, replace=False).tolist())
        par = oracle.make_params(dt=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)
        worst, n = check_trace(gpt, oracle, sv, par, Ns, batch, sample, 40)
        print("bench config:", n, "iterates checked, worst", worst)
    finally:
        sv.close()


@pytest.mark.parametrize("cluster", [32, 64])
@pytest.mark.parametrize("N", [32, 128])
def test_reference_trajectory_batch_matches_oracle_per_iterate(gpt, oracle, golden, N, cluster):
    """The reference's own trajectory testfiles/0_0_traj.csv (dt 1/64, explicit Euler, QD = R = 1e-4,
    the settings of its logged runs): 16 windows of N rows as a batch, every iterate of 4 of them."""
    B = 16
    starts = [1 + 30 * i for i in range(B)]
    probs = [ref_problem(golden, N, s) for s in starts]
    Ns = [N] * B
    batch = {"xu": np.zeros(21 * N * B, np.float32), "goal": np.concatenate([p["goal"] for p in probs]),
             "lam": np.zeros(14 * N * B, np.float32)}
    for b, p in enumerate(probs):
        batch["xu"][21 * N * b:21 * N * b + 21 * N - 7] = p["xu"]
    sv = gpt.Solver(max_knot_points=N, max_batch=B, **REF_CFG)
    try:
        sv.set_solver(sqp_max_iter=40, pcg_max_iter=10000, pcg_exit_tol=1e-5, pcg_exit_mode=0,
                      pcg_cluster_size=cluster)
        par = oracle.make_params()
        worst, n = check_trace(gpt, oracle, sv, par, Ns, batch, [0, 5, 10, 15], 40)
        print(f"reference trajectory N={N}:", n, "iterates checked, worst", worst)
    finally:
        sv.close()


def test_trace_equals_untraced_solve(gpt, problem_mod):
    """Recording the iterates changes nothing: the traced host loop and the graph solve agree bit for bit."""
    Ns = [64, 33, 128, 17]
    batch = problem_mod.make_batch(Ns, seed0=40, dt=0.01)
    sv = gpt.Solver(max_knot_points=128, max_batch=len(Ns), **SPEC_CFG)
    try:
        sv.set_solver(sqp_max_iter=12, pcg_max_iter=10000, pcg_exit_tol=1e-5)
        outs = []
        for traced in (False, True):
            xu = torch.as_tensor(batch["xu"], device="cuda")
            lam = torch.as_tensor(batch["lam"], device="cuda")
            goal = torch.as_tensor(batch["goal"], device="cuda")
            if traced:
                rho, st, tr = sv.sqp_solve_batched_trace(Ns, goal, lam, xu, [1e-3] * len(Ns), 5)
                rec = gpt.trace_record_fields(tr["rec"])
                assert (rec["active"][0] == 1).all()
                # iterate 0 is the input
                assert torch.equal(tr["xu"][0, :21 * sum(Ns) - 7], torch.as_tensor(batch["xu"][:21 * sum(Ns) - 7],
                                                                                     device="cuda"))
            else:
                rho, st = sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * len(Ns))
            outs.append((xu.cpu().numpy(), lam.cpu().numpy(), rho, [s["sqp_iters"] for s in st]))
        assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
        assert outs[0][2] == outs[1][2] and outs[0][3] == outs[1][3]
    finally:
        sv.close()
