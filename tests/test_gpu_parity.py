"""Parity of the CUDA kernels (through the C ABI) against the CPU oracle.

Every kernel is fed the same inputs as the oracle; the oracle runs in FP64
unless noted.  Tolerances are written next to each check: FP32 kernels vs an
FP64 restatement, scaled by the magnitude of the compared block.
"""
import numpy as np
import pytest

from conftest import ref_problem

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def close(got, want, rtol, what, scale=None):
    """|got - want| <= rtol * scale elementwise, scale = max|want| by default."""
    s = np.abs(want).max() if scale is None else scale
    err = np.abs(got - want).max()
    assert err <= rtol * max(s, 1e-30), f"{what}: max err {err:.3e} vs scale {s:.3e} (rtol {rtol})"


REF_CFG = dict(timestep=1.0 / 64, integrator=0, qd_cost=1e-4, r_cost=1e-4)
SPEC_CFG = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)


def problems(golden, problem_mod):
    out = []
    for N in (2, 3, 32, 128):
        out.append(("ref", N, REF_CFG, ref_problem(golden, N)))
    for N in (4, 64):
        out.append(("spec", N, SPEC_CFG, problem_mod.make_problem(N, 7, dt=0.01)))
    return out


def oracle_params(oracle, cfg, ref_terminal=1):
    return oracle.make_params(dt=cfg["timestep"], integrator=cfg["integrator"], qd_cost=cfg["qd_cost"],
                              r_cost=cfg["r_cost"], ref_terminal=ref_terminal)


@pytest.fixture(scope="module")
def solvers(gpt):
    cache = {}

    def get(cfg, **extra):
        key = tuple(sorted(cfg.items())) + tuple(sorted(extra.items()))
        if key not in cache:
            cache[key] = gpt.Solver(max_knot_points=512, **cfg, **extra)
        cache[key].reset_solver()  # no solver setting carries over from another test
        return cache[key]
    yield get
    for s in cache.values():
        s.close()


def kkt_gpu(sv, N, p):
    G, Cm, g, c = (torch.zeros(n, device="cuda") for n in (245 * N - 49, 294 * (N - 1), 21 * N - 7, 14 * N))
    sv.form_kkt(N, dev(p["xu"]), dev(p["goal"]), dev(p["xs"]), G, Cm, g, c)
    return host(G), host(Cm), host(g), host(c)


@pytest.mark.parametrize("ref_terminal", [1, 0])
def test_form_kkt(gpt, oracle, golden, problem_mod, solvers, ref_terminal):
    for kind, N, cfg, p in problems(golden, problem_mod):
        sv = solvers(cfg, ref_terminal=ref_terminal)
        G, Cm, g, c = kkt_gpu(sv, N, p)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, cfg, ref_terminal), N, p["xu"], p["goal"], p["xs"])
        for k in range(N):
            # Q_k holds q q^T (the reference's Hessian, iiwa_eepos_plant.cuh:362-373): relative 2e-5 of its block
            close(G[245 * k:245 * k + 196], oG[245 * k:245 * k + 196], 2e-5, f"{kind} N={N} Q_{k}")
        close(G, oG, 2e-5, f"{kind} N={N} G")
        for k in range(N - 1):
            close(Cm[294 * k:294 * k + 294], oC[294 * k:294 * k + 294], 2e-5, f"{kind} N={N} C_{k}")
        close(g, og, 2e-5, f"{kind} N={N} g")
        # defects are differences of nearby states: absolute 1e-5 of the state scale
        close(c, oc, 1e-5, f"{kind} N={N} c", scale=max(1.0, np.abs(p["xu"]).max()))


def test_form_schur(gpt, oracle, golden, problem_mod, solvers):
    for kind, N, cfg, p in problems(golden, problem_mod):
        sv = solvers(cfg)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, cfg), N, p["xu"], p["goal"], p["xs"])
        for rho in (1e-3, 0.5):
            # inputs rounded to float32 once; the oracle works on the same rounded values
            f = [x.astype(np.float32).astype(np.float64) for x in (oG, oC, og, oc)]
            S, Pv, gam, Gi = (torch.zeros(n, device="cuda") for n in (588 * N, 588 * N, 14 * N, 245 * N - 49))
            sv.form_schur(N, rho, *(dev(x) for x in f), S, Pv, gam, Gi)
            S, Pv, gam, Gi = map(host, (S, Pv, gam, Gi))
            wS, wP, wg, wGi = oracle.form_schur(N, rho, *f)
            for k in range(N):
                for b in range(3):
                    if (k == 0 and b == 0) or (k == N - 1 and b == 2):
                        assert np.abs(S[588 * k + 196 * b:588 * k + 196 * (b + 1)]).max() == 0.0
                        continue
                    blk = slice(588 * k + 196 * b, 588 * k + 196 * (b + 1))
                    close(S[blk], wS[blk], 1e-4, f"{kind} N={N} rho={rho} S[{k}][{b}]")
                Sd = S[588 * k + 196:588 * k + 392].reshape(14, 14, order="F")
                Pd = Pv[588 * k + 196:588 * k + 392].reshape(14, 14, order="F")
                # Pinv diag = (S diag)^{-1} (theta inverted in FP64): residual test
                assert np.abs(Sd @ Pd - np.eye(14)).max() < 1e-3, (kind, N, rho, k)
                assert np.abs(Pv[588 * k:588 * k + 196]).max() == 0 and np.abs(Pv[588 * k + 392:588 * k + 588]).max() == 0
            close(gam, wg, 1e-4, f"{kind} N={N} gamma")
            close(Gi, wGi, 1e-4, f"{kind} N={N} Ginv")


def test_form_schur_csc_matches_block_layout(gpt, oracle, golden, solvers):
    N = 16
    p = ref_problem(golden, N)
    sv = solvers(REF_CFG)
    f = [x.astype(np.float32) for x in oracle.form_kkt(oracle_params(oracle, REF_CFG), N, p["xu"], p["goal"], p["xs"])]
    S, Pv, gam, Gi = (torch.zeros(n, device="cuda") for n in (588 * N, 588 * N, 14 * N, 245 * N - 49))
    sv.form_schur(N, 1e-3, *(dev(x) for x in f), S, Pv, gam, Gi)
    val = torch.zeros(196 * (N - 1) + 105 * N, device="cuda")
    gam2, Gi2 = torch.zeros_like(gam), torch.zeros_like(Gi)
    sv.form_schur_csc(N, 1e-3, *(dev(x) for x in f), val, gam2, Gi2)
    # the CSC values are exactly the block matrix's upper triangle (same arithmetic)
    np.testing.assert_array_equal(host(val), oracle.csc_values(N, host(S)))
    np.testing.assert_array_equal(host(gam2), host(gam))


def schur_residual(S, lam, gam, N):
    M = S.astype(np.float64)
    Sl = np.concatenate([
        sum(M[588 * k + 196 * b:588 * k + 196 * (b + 1)].reshape(14, 14, order="F") @ lam[14 * kk:14 * kk + 14]
            for b, kk in ((0, k - 1), (1, k), (2, k + 1)) if 0 <= kk < N) for k in range(N)])
    return np.linalg.norm(gam - Sl) / np.linalg.norm(gam)


@pytest.mark.parametrize("precond", [0, 1])
@pytest.mark.parametrize("cluster", [0, 1, 2, 4, 8, 16, 32, 64])
def test_pcg_reaches_tolerance(gpt, oracle, golden, problem_mod, solvers, cluster, precond):
    """Exit mode 0 stops on the TRUE relative residual (FP64-evaluated); the
    returned lambda satisfies ||gamma - S lambda|| <= tol ||gamma|| for every
    cluster size (CTAs per instance; 32 = the warp-pair kernel, one CTA per
    instance with a twisted factorisation; 64 = the partitioned kernel, one CTA
    per instance, four factoring warps) and both preconditioners (0: the
    reference's block-Jacobi, 1: exact block-tridiagonal LDL^T per chunk); a
    warm start at the solution needs at most a few iterations."""
    pair = cluster in (gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD)
    if pair and precond == 0:
        pytest.skip("the one-CTA kernels have the exact preconditioner only")
    for kind, N, cfg, p in problems(golden, problem_mod):
        if cluster > N and not pair:
            continue
        sv = solvers(cfg)
        sv.set_solver(pcg_cluster_size=cluster, pcg_precond=precond)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, cfg), N, p["xu"], p["goal"], p["xs"])
        S, Pv, gam, _ = oracle.form_schur(N, 1e-1, *(x.astype(np.float32) for x in (oG, oC, og, oc)))
        S, Pv, gam = (x.astype(np.float32) for x in (S, Pv, gam))
        tol = 1e-5
        lam = torch.zeros(14 * N, device="cuda")
        lam64 = torch.zeros(14 * N, device="cuda", dtype=torch.float64)
        it, maxed = sv.pcg(N, dev(S), dev(Pv), dev(gam), lam, 20000, tol, 0, lam64=lam64)
        torch.cuda.synchronize()
        l64 = lam64.cpu().numpy()
        relres = schur_residual(S, l64, gam.astype(np.float64), N)
        assert not maxed, (kind, N, cluster, it, relres)
        # the kernel's FP64 true residual and this host evaluation agree to rounding
        assert relres <= 1.02 * tol, (kind, N, cluster, relres, it)
        # the FP32 copy is the FP64 iterate rounded
        np.testing.assert_array_equal(host(lam).astype(np.float32), l64.astype(np.float32))
        # warm start from the FP32 copy: the FP32 rounding floor may need a few iterations, no more
        lam2 = lam.clone()
        it2, maxed2 = sv.pcg(N, dev(S), dev(Pv), dev(gam), lam2, 20000, tol, 0)
        if precond == 1:
            assert not maxed2 and it2 <= max(5, it // 10), (kind, N, cluster, it2, it)
        else:
            # block-Jacobi with an FP32 search direction: at cond(S) ~ 1e7 the FP32 rounding of
            # the start perturbs the residual by ~eps32 cond(S), so a warm start is no better than
            # a cold one
            assert not maxed2 and it2 <= it, (kind, N, cluster, it2, it)
        if precond == 1 and (cluster in (0, 1) or pair):
            # one chunk = the whole horizon: the preconditioner is the inverse up to rounding
            assert it <= 4, (kind, N, it)
        # eta-based exit (|r^T Pinv r| < tol) runs and stops
        lam3 = torch.zeros(14 * N, device="cuda")
        it3, maxed3 = sv.pcg(N, dev(S), dev(Pv), dev(gam), lam3, 20000, 1e-12 * float(np.abs(gam).max()) ** 2, 1)
        assert it3 > 0
        sv.set_solver(pcg_cluster_size=0, pcg_precond=0)


def test_pcg_cluster_sizes_agree(gpt, oracle, problem_mod, solvers):
    """Different CTA splits of one instance reach the same solution (to the tolerance)."""
    N = 64
    cfg = SPEC_CFG
    p = problem_mod.make_problem(N, 3, dt=0.01)
    sv = solvers(cfg)
    oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, cfg), N, p["xu"], p["goal"], p["xs"])
    S, Pv, gam, _ = oracle.form_schur(N, 1e-2, *(x.astype(np.float32) for x in (oG, oC, og, oc)))
    S, Pv, gam = (x.astype(np.float32) for x in (S, Pv, gam))
    lam_star = oracle.banded_cholesky(N, S, gam)
    sols = {}
    for cs in (1, 2, 4, 8, 16, gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD):
        sv.set_solver(pcg_cluster_size=cs)
        lam = torch.zeros(14 * N, device="cuda")
        lam64 = torch.zeros(14 * N, device="cuda", dtype=torch.float64)
        sv.pcg(N, dev(S), dev(Pv), dev(gam), lam, 50000, 1e-5, 0, lam64=lam64)
        torch.cuda.synchronize()
        sols[cs] = lam64.cpu().numpy()
    sv.set_solver(pcg_cluster_size=0)
    ref = np.linalg.norm(lam_star)
    # one CTA per instance (cyclic reduction) and the warp pair (twisted factorisation) both apply
    # the exact inverse: their solutions differ by rounding only
    assert np.linalg.norm(sols[1] - sols[gpt.PCG_WARP_PAIR]) <= 1e-7 * ref
    assert np.linalg.norm(sols[1] - sols[gpt.PCG_WARP_QUAD]) <= 1e-7 * ref
    errs = {cs: np.linalg.norm(v - lam_star) / ref for cs, v in sols.items()}
    # every split lands within the accuracy the 1e-5 residual allows of the FP64 Cholesky
    # solution (one CTA per instance solves exactly; the chunked splits stop at the tolerance)
    assert max(errs.values()) <= 2e-5, errs


def test_compute_dz(gpt, oracle, golden, problem_mod, solvers):
    """dz from lambda (FP32 inputs).  The right-hand sides cancel heavily, so the
    bound is componentwise: |dz - dz64| <= 4e-6 * |Ginv| (|g| + |lambda_k| + |C|^T |lambda_{k+1}|)
    (FP32 storage of the inputs, FP64 accumulation inside the kernel)."""
    for kind, N, cfg, p in problems(golden, problem_mod):
        sv = solvers(cfg)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, cfg), N, p["xu"], p["goal"], p["xs"])
        f = [x.astype(np.float32).astype(np.float64) for x in (oG, oC, og, oc)]
        S, Pv, gam, Gi = oracle.form_schur(N, 1e-2, *f)
        lam = oracle.banded_cholesky(N, S, gam).astype(np.float32).astype(np.float64)
        Gi = Gi.astype(np.float32).astype(np.float64)
        dz = torch.zeros(21 * N - 7, device="cuda")
        sv.compute_dz(N, dev(Gi), dev(f[1]), dev(f[2]), dev(lam), dz)  # FP32 inputs as the reference
        got = host(dz)
        want = oracle.compute_dz(N, Gi, f[1], f[2], lam)
        bound = np.zeros(21 * N - 7)
        for k in range(N):
            Gq = np.abs(Gi[245 * k:245 * k + 196]).reshape(14, 14, order="F")
            sx = np.abs(f[2][21 * k:21 * k + 14]) + np.abs(lam[14 * k:14 * k + 14])
            if k < N - 1:
                mA = np.abs(f[1][294 * k:294 * k + 196]).reshape(14, 14, order="F")
                mB = np.abs(f[1][294 * k + 196:294 * k + 294]).reshape(14, 7, order="F")
                ln = np.abs(lam[14 * (k + 1):14 * (k + 2)])
                sx = sx + mA.T @ ln
                Gr = np.abs(Gi[245 * k + 196:245 * k + 245]).reshape(7, 7, order="F")
                bound[21 * k + 14:21 * k + 21] = Gr @ (np.abs(f[2][21 * k + 14:21 * k + 21]) + mB.T @ ln)
            bound[21 * k:21 * k + 14] = Gq @ sx
        err = np.abs(got - want)
        assert (err <= 4e-6 * bound + 1e-12).all(), (kind, N, float((err / (bound + 1e-30)).max()))


def test_merits(gpt, oracle, golden, problem_mod, solvers):
    for kind, N, cfg, p in problems(golden, problem_mod):
        sv = solvers(cfg)
        par = oracle_params(oracle, cfg)
        m = torch.zeros(1, device="cuda")
        sv.compute_merit(N, dev(p["xu"]), dev(p["goal"]), m)
        want, _ = oracle.merit(par, N, p["xu"].astype(np.float64), None, 0.0, p["goal"], p["xs"], 0)
        # cost terms: relative 2e-5; defect terms are differences of states: mu * 14 (N-1) * 2 eps32 |x|
        xmax = max(1.0, float(np.abs(p["xu"]).max()))
        dtol = 10.0 * 14 * (N - 1) * 2.4e-7 * xmax
        assert abs(host(m)[0] - want) <= 2e-5 * abs(want) + dtol, (kind, N, host(m)[0], want)
        rng = np.random.default_rng(N)
        dz = (rng.normal(0, 0.05, 21 * N - 7)).astype(np.float32)
        xs = (p["xs"] + rng.normal(0, 0.01, 14)).astype(np.float32)
        ms = torch.zeros(8, device="cuda")
        sv.ls_compute_merit(N, dev(xs), dev(p["xu"]), dev(p["goal"]), dev(dz), ms)
        got = host(ms)
        for a in range(8):
            w, _ = oracle.merit(par, N, p["xu"], dz, -1.0 / (1 << a), p["goal"], xs, 1)
            assert abs(got[a] - w) <= 5e-5 * abs(w) + dtol + 1e-5, (kind, N, a, got[a], w)


def kkt_residual(N, G, Cm, g, c, rho, dz, lam):
    """Relative FP64 residual of [Gt C^T; C 0][dz; lambda] = [g; c] (oldschur.cuh:966-1092)."""
    from test_oracle_golden import kkt_dense
    Gt, Cc = kkt_dense(N, G, Cm, g, c, rho)
    r1 = Gt @ dz + Cc.T @ lam - g
    r2 = Cc @ dz - c
    return np.sqrt(np.sum(r1 ** 2) + np.sum(r2 ** 2)) / np.sqrt(np.sum(g ** 2) + np.sum(c ** 2))


def test_linear_system_solution_satisfies_kkt(gpt, oracle, golden, problem_mod, solvers):
    """The whole linear-algebra chain on the GPU -- Schur complement, PCG (FP64
    iterate) to relative residual 1e-6, dz recovery -- returns (dz, lambda) that
    satisfy the reference's KKT system (formed by the GPU in FP32) with an FP64
    relative residual at the floor that FP32 formation of S leaves (measured on
    the oracle's FP32 Schur data), and dz agrees with the FP64 oracle solution of
    the same FP32 KKT data.  cond(S) reaches 1e7 at these sizes, so agreement is
    stated against the FP64 solve of identical inputs."""
    for kind, N, cfg, p in problems(golden, problem_mod):
        if N > 64:
            continue
        sv = solvers(cfg)
        G, Cm, g, c = kkt_gpu(sv, N, p)
        rho = 1e-3
        S, Pv, gam, Gi = (torch.zeros(n, device="cuda") for n in (588 * N, 588 * N, 14 * N, 245 * N - 49))
        Gi64 = torch.zeros(245 * N - 49, device="cuda", dtype=torch.float64)
        sv.form_schur(N, rho, dev(G), dev(Cm), dev(g), dev(c), S, Pv, gam, Gi, Ginv64=Gi64)
        lam = torch.zeros(14 * N, device="cuda")
        lam64 = torch.zeros(14 * N, device="cuda", dtype=torch.float64)
        it, maxed = sv.pcg(N, S, Pv, gam, lam, 100000, 1e-6, 0, lam64=lam64)
        assert not maxed, (kind, N, it)
        dz = torch.zeros(21 * N - 7, device="cuda")
        sv.compute_dz(N, None, dev(Cm), dev(g), None, dz, lam64=lam64, Ginv64=Gi64)
        torch.cuda.synchronize()
        l64 = lam64.cpu().numpy()
        res = kkt_residual(N, G, Cm, g, c, rho, host(dz), l64)
        # FP64 oracle on the same FP32 KKT data
        oS, oP, og, oGi = oracle.form_schur(N, rho, G, Cm, g, c)
        olam = oracle.banded_cholesky(N, oS, og)
        odz = oracle.compute_dz(N, oGi, Cm, g, olam)
        assert kkt_residual(N, G, Cm, g, c, rho, odz, olam) < 1e-9
        # floor: the reference forms S and gamma in FP32 (schur.cuh:391-524); the exact solution
        # of the oracle's FP32-formed system, with dz rounded to FP32, leaves this residual
        fS, _, fg, _ = oracle.form_schur(N, rho, G, Cm, g, c, precision="f32")
        flam = oracle.banded_cholesky(N, np.asarray(fS, np.float64), np.asarray(fg, np.float64))
        fdz = oracle.compute_dz(N, oGi, Cm, g, flam).astype(np.float32).astype(np.float64)
        floor = kkt_residual(N, G, Cm, g, c, rho, fdz, flam)
        # the FP64 path (FP64 lambda and inverses, as the SQP loop uses): the floor plus the PCG
        # tolerance (1e-6 on S)
        assert res < 2 * floor + 2e-5, (kind, N, res, floor)
        # the reference-layout FP32 inverses (schur.cuh:236-256) add their own rounding,
        # conditioned up to ~1e3 at rho = 1e-3
        dz32 = torch.zeros(21 * N - 7, device="cuda")
        sv.compute_dz(N, Gi, dev(Cm), dev(g), None, dz32, lam64=lam64)
        assert kkt_residual(N, G, Cm, g, c, rho, host(dz32), l64) < 4 * floor + 2e-4
        # dz vs the FP64 solution, against the spread that FP32 formation of S alone causes
        # (~1e-2 on the spec problem at N = 64, where cond(S) ~ 1e7)
        rel = np.linalg.norm(host(dz) - odz) / np.linalg.norm(odz)
        frel = np.linalg.norm(fdz - odz) / np.linalg.norm(odz)
        assert rel < max(1e-3, 4 * frel), (kind, N, rel, frel)


def test_sqp_first_iterate_matches_oracle(gpt, oracle, golden, problem_mod, solvers):
    """One SQP iteration (KKT, Schur, PCG, dz, 8-step line search, step) on the
    GPU vs the oracle's iteration (FP64, exact Cholesky solve) from the same
    iterate: the same step length is accepted, the merit decreases by the same
    amount to 1e-3 relative and the new iterates agree to 1e-2 relative, or to
    three times the spread FP32 formation of S causes in dz where that is
    larger (the KKT data differ by FP32 rounding, amplified by cond(S) ~ 1e7)."""
    for kind, N, cfg, p in problems(golden, problem_mod):
        # the reference trajectories are already near a stationary point: their 8 line-search
        # merits tie to FP32 rounding, so the accepted step length is not a stable comparison there
        if N > 64 or kind == "ref":
            continue
        sv = solvers(cfg)
        sv.set_solver(sqp_max_iter=1, pcg_max_iter=100000, pcg_exit_tol=1e-7, pcg_exit_mode=0)
        xu = dev(p["xu"])
        lam = dev(p["lam"])
        res = sv.sqp_solve(N, dev(p["goal"]), lam, xu, 1e-3)
        sv.set_solver(sqp_max_iter=40, pcg_max_iter=167, pcg_exit_tol=1e-5)
        sol = oracle.make_solver(linsys=2, sqp_max_iter=1)
        oxu, olam, orho, ost, _ = oracle.sqp_solve(oracle_params(oracle, cfg), sol, N, p["goal"], p["lam"], p["xu"], 1e-3)
        assert res.sqp_iters == 1 and ost.sqp_iters == 1
        assert abs(res.rho - orho) <= 1e-6 * orho  # same accept / reject decision
        step_g = host(xu) - p["xu"]
        step_o = oxu - p["xu"]
        # the spread that FP32 formation of S alone causes in dz at this iterate (the oracle's
        # FP32 Schur data solved exactly vs its FP64 Schur data), ~1e-2 where cond(S) ~ 1e7
        rho = 1e-3
        kG, kC, kg, kc = (np.asarray(a, np.float32).astype(np.float64)
                          for a in oracle.form_kkt(oracle_params(oracle, cfg), N, p["xu"], p["goal"], p["xs"]))
        oS, _, ogam, oGi = oracle.form_schur(N, rho, kG, kC, kg, kc)
        odz = oracle.compute_dz(N, oGi, kC, kg, oracle.banded_cholesky(N, oS, ogam))
        fS, _, fgam, _ = oracle.form_schur(N, rho, kG, kC, kg, kc, precision="f32")
        fdz = oracle.compute_dz(N, oGi, kC, kg, oracle.banded_cholesky(N, np.asarray(fS, np.float64),
                                                                       np.asarray(fgam, np.float64)))
        frel = np.linalg.norm(fdz - odz) / np.linalg.norm(odz)
        assert np.linalg.norm(step_g - step_o) <= max(1e-2, 3 * frel) * max(np.linalg.norm(step_o), 1e-6) + 1e-5, (
            kind, N, np.linalg.norm(step_g - step_o), np.linalg.norm(step_o), frel)
        dm_g = res.stats["merit_initial"] - res.stats["merit_final"]
        dm_o = ost.merit_final
        m0, _ = oracle.merit(oracle_params(oracle, cfg), N, p["xu"], None, 0.0, p["goal"], p["xs"], 0)
        assert abs(dm_g - (m0 - dm_o)) <= 1e-3 * abs(m0 - dm_o) + 1e-5, (kind, N, dm_g, m0 - dm_o)


def test_sqp_solve_full_reduces_merit_like_oracle(gpt, oracle, golden, problem_mod, solvers):
    for kind, N, cfg, p in problems(golden, problem_mod):
        if N not in (32, 64):
            continue
        sv = solvers(cfg)
        sv.set_solver(sqp_max_iter=10, pcg_max_iter=4000, pcg_exit_tol=1e-6)
        res = sv.sqp_solve(N, dev(p["goal"]), dev(p["lam"]), dev(p["xu"]), 1e-3)
        sv.set_solver(sqp_max_iter=40, pcg_max_iter=167, pcg_exit_tol=1e-5)
        sol = oracle.make_solver(linsys=2, sqp_max_iter=10)
        oxu, olam, orho, ost, _ = oracle.sqp_solve(oracle_params(oracle, cfg), sol, N, p["goal"], p["lam"], p["xu"], 1e-3)
        m0 = res.stats["merit_initial"]
        assert res.stats["merit_final"] < m0
        # both descend to within 5% of each other's merit after 10 iterations
        assert abs(res.stats["merit_final"] - ost.merit_final) <= 0.05 * abs(m0 - ost.merit_final) + 1e-4, (
            kind, N, res.stats, ost.merit_final)


def test_batched_equals_plain(gpt, problem_mod, solvers):
    Ns = [8, 16, 5, 32]
    batch = problem_mod.make_batch(Ns, seed0=11)
    sv = gpt.Solver(max_knot_points=64, max_batch=8, **SPEC_CFG)
    # same CTA split for both calls, so the reductions run in the same order
    sv.set_solver(sqp_max_iter=6, pcg_max_iter=500, pcg_exit_tol=1e-5, pcg_cluster_size=1)
    xu = dev(batch["xu"])
    lam = dev(batch["lam"])
    rho, stats = sv.sqp_solve_batched(Ns, dev(batch["goal"]), lam, xu, [1e-3] * len(Ns))
    gxu = host(xu)
    off = 0
    for b, N in enumerate(Ns):
        p = problem_mod.make_problem(N, 11 + b)
        xu1 = dev(p["xu"])
        r1 = sv.sqp_solve(N, dev(p["goal"]), dev(p["lam"]), xu1, 1e-3)
        np.testing.assert_array_equal(gxu[21 * off:21 * off + 21 * N - 7], host(xu1))
        assert r1.sqp_iters == stats[b]["sqp_iters"]
        assert abs(r1.rho - rho[b]) == 0.0
        off += N
    sv.close()


def test_bad_arguments_are_rejected_without_launch(gpt, solvers):
    sv = solvers(REF_CFG)
    t = torch.zeros(1000, device="cuda")
    with pytest.raises(gpt.GptError) as e:
        sv.form_kkt(1, t, t, t, t, t, t, t)  # N < 2
    assert e.value.status == 1
    with pytest.raises(gpt.GptError):
        sv.pcg(600, t, t, t, t, 10, 1e-5)  # N above the handle's capacity
    with pytest.raises(ValueError):
        sv.form_kkt(4, t.cpu(), t, t, t, t, t, t)


def test_sqp_solve_chain_preconditioner_matches_block_jacobi(gpt, problem_mod):
    """Same SQP solve with both preconditioners (relative residual 1e-8): the
    iterates agree to the PCG tolerance and the chain LDL^T needs far fewer
    PCG iterations."""
    N = 64
    p = problem_mod.make_problem(N, 5, dt=0.01)
    out = {}
    for pre in (0, 1):
        sv = gpt.Solver(max_knot_points=N, **SPEC_CFG)
        sv.set_solver(sqp_max_iter=3, pcg_max_iter=50000, pcg_exit_tol=1e-8, pcg_precond=pre, pcg_cluster_size=1)
        xu = dev(p["xu"])
        r = sv.sqp_solve(N, dev(p["goal"]), dev(p["lam"]), xu, 1e-3)
        out[pre] = (host(xu), r)
        sv.close()
    (x0, r0), (x1, r1) = out[0], out[1]
    assert r0.sqp_iters == r1.sqp_iters and abs(r0.rho - r1.rho) <= 1e-6 * r0.rho
    step = np.linalg.norm(x0 - p["xu"])
    # cond(S) ~ 1e7: two solutions at relative residual 1e-8 differ by up to ~1e-1 in lambda,
    # a few 1e-3 in the iterate after three steps
    assert np.linalg.norm(x0 - x1) <= 1e-2 * step, (np.linalg.norm(x0 - x1), step)
    # the merit's mu-weighted L1 defect term is the most sensitive to those differences
    assert abs(r0.stats["merit_final"] - r1.stats["merit_final"]) <= 3e-2 * abs(r0.stats["merit_final"])
    assert sum(r1.pcg_iters) * 20 < sum(r0.pcg_iters), (r1.pcg_iters, r0.pcg_iters)


@pytest.mark.parametrize("schur_fp64", [1, 0])
@pytest.mark.parametrize("exit_mode", [0, 1])
def test_sqp_warp_pair_pcg_matches_chain(gpt, problem_mod, schur_fp64, exit_mode):
    """The warp-pair PCG (one CTA per instance, twisted factorisation) and the
    one-CTA chain PCG (cyclic reduction) apply the same exact preconditioner to
    the same S.  On a batch of uneven horizons (2 and 3 knots included: no top
    sweep, one knot each side): one SQP iteration from the same iterate gives
    the same step to 1e-6 (the two factorisation orders differ by FP64
    rounding only); four iterations take the same SQP decisions with 1-2 PCG
    iterations per linear system and end within 1e-3 of the step (an FP32
    rounding difference of an iterate is amplified by cond(S) ~ 1e7 in the
    next linear system)."""
    Ns = [2, 3, 17, 64, 128, 5]
    ps = [problem_mod.make_problem(n, 60 + i, dt=0.01) for i, n in enumerate(Ns)]
    cat = lambda key, pad: np.concatenate([np.concatenate([p[key], np.zeros(pad, np.float32)]) for p in ps])
    goal, xu0, lam0 = dev(cat("goal", 0)), dev(cat("xu", 7)), dev(cat("lam", 0))
    x0 = host(xu0)
    for iters, tol in ((1, 1e-6), (4, 1e-3)):
        out = {}
        for cs in (1, gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD):
            sv = gpt.Solver(max_knot_points=128, max_batch=len(Ns), **SPEC_CFG)
            sv.set_solver(sqp_max_iter=iters, pcg_max_iter=1000, pcg_exit_tol=1e-9 if exit_mode == 0 else 1e-14,
                          pcg_exit_mode=exit_mode, pcg_cluster_size=cs, schur_fp64=schur_fp64)
            xu, lam = xu0.clone(), lam0.clone()
            rho, stats = sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * len(Ns))
            out[cs] = (host(xu), rho, stats)
            sv.close()
        x1, r1, s1 = out[1]
        for other in (gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD):
            x2, r2, s2 = out[other]
            assert [s["sqp_iters"] for s in s1] == [s["sqp_iters"] for s in s2]
            assert r1 == r2
            off = 0
            for b, n in enumerate(Ns):
                sl = slice(21 * off, 21 * off + 21 * n - 7)
                step = np.linalg.norm(x1[sl] - x0[sl])
                diff = np.linalg.norm(x2[sl] - x1[sl])
                assert diff <= tol * step + 1e-6, (other, iters, n, diff, step)
                assert s2[b]["pcg_maxiter_count"] == 0
                assert s2[b]["pcg_iters_total"] <= 2 * s2[b]["sqp_iters"], (other, n, s2[b])
                off += n


@pytest.mark.parametrize("cluster", [1, 32, 64])
def test_sqp_graph_equals_host_loop(gpt, problem_mod, cluster):
    """The solve as one CUDA graph (device-side while loop, the default), the graph with
    the batch split in parts on concurrent branches (sqp_graph 2: 2 + 3 instances of
    uneven horizon; 4: 1 + 1 + 1 + 2) and the host-driven loop give bit-identical results,
    on the first call of a batch shape (capture) and on later calls (the cached graph),
    for a batch whose instances stop at different SQP iterations; with the chain and
    the warp-pair PCG kernels."""
    Ns = [16, 24, 32, 8, 20]
    ps = [problem_mod.make_problem(n, 40 + i, dt=0.01) for i, n in enumerate(Ns)]
    cat = lambda key, pad: np.concatenate([np.concatenate([p[key], np.zeros(pad, np.float32)]) for p in ps])
    goal, xu0, lam0 = dev(cat("goal", 0)), dev(cat("xu", 7)), dev(cat("lam", 0))
    out = {}
    B = len(Ns)
    for graph in (0, 1, 2, 4):
        sv = gpt.Solver(max_knot_points=32, max_batch=B, **SPEC_CFG)
        sv.set_solver(sqp_graph=graph, sqp_max_iter=12, pcg_cluster_size=cluster)
        res = []
        for rep in range(2):
            xu, lam = xu0.clone(), lam0.clone()
            rho, stats = sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * B)
            res.append((host(xu), host(lam), rho, [s["sqp_iters"] for s in stats]))
        sv.close()
        out[graph] = res
    for graph in (1, 2, 4):
        for rep in range(2):
            (x0, l0, r0, i0), (x1, l1, r1, i1) = out[0][rep], out[graph][rep]
            assert i0 == i1 and r0 == r1, (graph, i0, i1, r0, r1)
            np.testing.assert_array_equal(x0, x1)
            np.testing.assert_array_equal(l0, l1)


def test_autotune_choice_is_used(gpt, problem_mod):
    """gpt_autotune leaves its inputs unchanged, returns one of its candidate cluster
    sizes, and a later solve of that batch shape with pcg_cluster_size 0 equals a
    solve with that size given explicitly, bit for bit."""
    N = 64
    p = problem_mod.make_problem(N, 9, dt=0.01)
    goal, xu0, lam0 = dev(p["goal"]), dev(p["xu"]), dev(p["lam"])
    sv = gpt.Solver(max_knot_points=N, **SPEC_CFG)
    sv.set_solver(sqp_max_iter=4)
    x_in, l_in = xu0.clone(), lam0.clone()
    sched = {}
    cs = sv.autotune([N], goal, l_in, x_in, [1e-3], schedule=sched)
    assert torch.equal(x_in, xu0) and torch.equal(l_in, lam0)
    assert cs in (1, 2, 4, gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD)
    assert sorted(sched) == ["branches", "dz", "kkt", "merit", "schur"], sched
    assert sched["branches"] == 1, sched  # one instance: no part-batch branches to try
    assert {sched[k] for k in ("kkt", "schur", "merit", "dz")} <= {4, 5, 6, 8, 16}, sched
    out = []
    for given in (0, cs):
        sv.set_solver(pcg_cluster_size=given)
        xu, lam = xu0.clone(), lam0.clone()
        sv.sqp_solve(N, goal, lam, xu, 1e-3)
        out.append(host(xu))
    sv.close()
    np.testing.assert_array_equal(out[0], out[1])



@pytest.mark.gpu
def test_autotune_picks_graph_branches(gpt, problem_mod):
    """With sqp_graph 1 the autotuner also times 2 and 4 part-batch branches per graph iteration for a
    batch (8 instances of N = 32); the solve that uses its choice gives the bits of the host-driven loop
    with the same tuned PCG kernel and grids."""
    Ns = [32] * 8
    batch = problem_mod.make_batch(Ns, seed0=21, dt=0.01)
    goal, xu0, lam0 = (dev(batch[k]) for k in ("goal", "xu", "lam"))
    sv = gpt.Solver(max_knot_points=32, max_batch=8, sqp_graph=1, **SPEC_CFG)
    try:
        sv.set_solver(sqp_max_iter=4)
        sched = {}
        sv.autotune(Ns, goal, lam0, xu0, [1e-3] * 8, schedule=sched)
        assert sched["branches"] in (1, 2, 4), sched
        out = []
        for graph in (1, 0):
            sv.set_solver(sqp_graph=graph)
            xu, lam = xu0.clone(), lam0.clone()
            sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * 8)
            out.append((host(xu), host(lam)))
    finally:
        sv.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])

def test_form_ss_matches_oracle(gpt, oracle, golden, problem_mod, solvers):
    """gpt_form_ss (gato_form_ss_inner) on the GPU's own S and block-Jacobi Pinv against the
    oracle's stair formation of the same FP32 inputs: off-diagonal blocks within 1e-5 of the
    largest block entry (FP32 products of 14x14 blocks, FMA vs separate rounding), diagonal
    blocks untouched, row 0's left and row N-1's right blocks left zero."""
    for kind, N, cfg, p in problems(golden, problem_mod):
        if N < 3:
            continue
        sv = solvers(cfg)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, cfg), N, p["xu"], p["goal"], p["xs"])
        f = [x.astype(np.float32) for x in (oG, oC, og, oc)]
        S, Pv, gam, Gi = (torch.zeros(n, device="cuda") for n in (588 * N, 588 * N, 14 * N, 245 * N - 49))
        sv.form_schur(N, 1e-3, *(dev(x) for x in f), S, Pv, gam, Gi)
        P0 = host(Pv)
        sv.form_ss(N, S, Pv)
        got = host(Pv)
        want = oracle.form_ss(N, host(S), P0)
        for k in range(N):
            np.testing.assert_array_equal(got[588 * k + 196:588 * k + 392], P0[588 * k + 196:588 * k + 392])
            for b in (0, 2):
                blk = slice(588 * k + 196 * b, 588 * k + 196 * (b + 1))
                if (k == 0 and b == 0) or (k == N - 1 and b == 2):
                    assert np.abs(got[blk]).max() == 0.0
                    continue
                close(got[blk], want[blk], 1e-5, f"{kind} N={N} SS[{k}][{b}]", scale=np.abs(want).max())


@pytest.mark.parametrize("N", [64, 128, 256, 512])
def test_plain_sweep_linear_solve_accuracy(gpt, oracle, problem_mod, solvers, N):
    """The plain method's linear solve over the horizon / tolerance sweep (N in {64, 128, 256,
    512} x PCG tolerance in {1e-4, 1e-5, 1e-6}) on the first SQP iterate's Schur system of a
    seeded problem: for the plain path's default PCG (cluster 0, exact preconditioner) and the
    warp-pair kernel, the FP64 true relative residual meets the tolerance, and the multipliers lie
    at least as close to the FP64 banded-Cholesky solution as the FP32 LDL^T of the reference's
    qdldl path does."""
    p = problem_mod.make_problem(N, 11, dt=0.01)
    sv = solvers(SPEC_CFG)
    oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, SPEC_CFG), N, p["xu"], p["goal"], p["xs"])
    S, Pv, gam, _ = oracle.form_schur(N, 1e-3, *(x.astype(np.float32) for x in (oG, oC, og, oc)))
    S, Pv, gam = (x.astype(np.float32) for x in (S, Pv, gam))
    ref = oracle.banded_cholesky(N, S.astype(np.float64), gam.astype(np.float64))
    ldl = oracle.ldl_solve(N, S.astype(np.float64), gam.astype(np.float64)).astype(np.float64)
    err_ldl = np.abs(ldl - ref).max() / np.abs(ref).max()
    for cluster in (0, gpt.PCG_WARP_PAIR, gpt.PCG_WARP_QUAD):
        sv.set_solver(pcg_cluster_size=cluster, pcg_precond=1)
        for tol in (1e-4, 1e-5, 1e-6):
            lam = torch.zeros(14 * N, device="cuda")
            lam64 = torch.zeros(14 * N, device="cuda", dtype=torch.float64)
            it, maxed = sv.pcg(N, dev(S), dev(Pv), dev(gam), lam, 2000, tol, 0, lam64=lam64)
            torch.cuda.synchronize()
            l64 = lam64.cpu().numpy()
            relres = schur_residual(S, l64, gam.astype(np.float64), N)
            assert not maxed and relres <= 1.02 * tol, (N, cluster, tol, it, relres)
            err = np.abs(l64 - ref).max() / np.abs(ref).max()
            assert err <= max(err_ldl, 1e-6), (N, cluster, tol, err, err_ldl)
    sv.set_solver(pcg_cluster_size=0, pcg_precond=0)


def test_partitioned_pcg_every_part_layout(gpt, oracle, problem_mod, solvers):
    """The partitioned kernel (GPT_PCG_WARP_QUAD) over horizons whose part layouts differ: one part
    (N = 2), two and three parts with empty parts (N = 3 .. 7), four parts with empty middle parts
    (N = 7 .. 10) and the long horizons.  It applies the exact inverse of S: the true relative residual
    meets a 1e-9 tolerance within two iterations and the solution is the FP64 Cholesky solution to
    the rounding cond(S) allows."""
    sv = solvers(SPEC_CFG)
    sv.set_solver(pcg_cluster_size=gpt.PCG_WARP_QUAD, pcg_precond=1)
    for N in list(range(2, 21)) + [31, 33, 64, 100, 128, 129, 255, 256, 511, 512]:
        p = problem_mod.make_problem(N, 70 + N, dt=0.01)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, SPEC_CFG), N, p["xu"], p["goal"], p["xs"])
        S, Pv, gam, _ = oracle.form_schur(N, 1e-2, *(x.astype(np.float32) for x in (oG, oC, og, oc)))
        S, Pv, gam = (x.astype(np.float32) for x in (S, Pv, gam))
        ref = oracle.banded_cholesky(N, S.astype(np.float64), gam.astype(np.float64))
        lam = torch.zeros(14 * N, device="cuda")
        lam64 = torch.zeros(14 * N, device="cuda", dtype=torch.float64)
        it, maxed = sv.pcg(N, dev(S), dev(Pv), dev(gam), lam, 50, 1e-9, 0, lam64=lam64)
        torch.cuda.synchronize()
        l64 = lam64.cpu().numpy()
        relres = schur_residual(S, l64, gam.astype(np.float64), N)
        assert not maxed and it <= 2 and relres <= 1.02e-9, (N, it, relres)
        err = np.abs(l64 - ref).max() / np.abs(ref).max()
        assert err <= 1e-6, (N, err)
    sv.set_solver(pcg_cluster_size=0, pcg_precond=0)


@pytest.mark.parametrize("cluster", [0, 1, 2, 4])
def test_stair_preconditioner_on_the_gpu(gpt, oracle, problem_mod, solvers, cluster):
    """pcg_precond 2: the block-Jacobi PCG kernel applying the stair preconditioner (the blocks of
    gpt_form_ss, gato_form_ss_inner, oldschur.cuh:334-494) as a block-tridiagonal Pinv, with the
    residual's neighbouring knots exchanged between the chunks of a cluster.  Against the same S:
    the true relative residual meets the tolerance, the iterations are well below block-Jacobi's
    (the oracle's FP64 PCG halves them on these problems), and the count is within 25 % of the
    oracle's PCG applying the same Pinv blocks (FP32 search directions on both sides)."""
    sv = solvers(SPEC_CFG)
    for N in (32, 64, 128):
        if cluster and cluster * 64 < N:
            continue
        p = problem_mod.make_problem(N, 21, dt=0.01)
        oG, oC, og, oc = oracle.form_kkt(oracle_params(oracle, SPEC_CFG), N, p["xu"], p["goal"], p["xs"])
        f = [x.astype(np.float32) for x in (oG, oC, og, oc)]
        S, Pv, gam, Gi = (torch.zeros(n, device="cuda") for n in (588 * N, 588 * N, 14 * N, 245 * N - 49))
        sv.form_schur(N, 1e-2, *(dev(x) for x in f), S, Pv, gam, Gi)
        Pbj = Pv.clone()
        sv.form_ss(N, S, Pv)
        tol = 1e-5
        its = {}
        # the PCG kernels read each diagonal block's lower triangle (S is symmetric; the FP32 products
        # that form it are not exactly): the residual is checked on that symmetric S
        Ssym = host(S)
        for k in range(N):
            D = Ssym[588 * k + 196:588 * k + 392].reshape(14, 14, order="F")
            L = np.tril(D)
            Ssym[588 * k + 196:588 * k + 392] = (L + np.tril(D, -1).T).reshape(-1, order="F")
        for pre, Pm in ((0, Pbj), (2, Pv)):
            sv.set_solver(pcg_cluster_size=cluster, pcg_precond=pre)
            lam = torch.zeros(14 * N, device="cuda")
            lam64 = torch.zeros(14 * N, device="cuda", dtype=torch.float64)
            it, maxed = sv.pcg(N, S, Pm, gam, lam, 50000, tol, 0, lam64=lam64)
            torch.cuda.synchronize()
            relres = schur_residual(Ssym, lam64.cpu().numpy(), host(gam), N)
            assert not maxed and relres <= 1.02 * tol, (N, cluster, pre, it, relres)
            its[pre] = it
        assert its[2] <= 0.75 * its[0], (N, cluster, its)
        _, o_it, o_max = oracle.pcg(N, host(S), host(Pv), host(gam), np.zeros(14 * N), 50000, tol, 0, "f32")
        print(f"stair N={N} cluster={cluster}: block-Jacobi {its[0]}, stair {its[2]}, oracle stair {o_it}")
        assert not o_max and abs(its[2] - o_it) <= 0.25 * o_it + 5, (N, cluster, its[2], o_it)
    sv.set_solver(pcg_cluster_size=0, pcg_precond=0)


def test_sqp_solve_stair_preconditioner_matches_exact(gpt, problem_mod):
    """The SQP loop with pcg_precond 2 (reference-layout Schur rows, the stair blocks formed on the
    batch, the block-Jacobi kernel applying them) on a batch of uneven horizons takes the same SQP
    decisions as the exact preconditioner at relative residual 1e-8, lands within 1e-2 of its step
    (cond(S) ~ 1e7 amplifies the FP32 Schur formation of this path), and needs fewer PCG iterations
    than block-Jacobi."""
    Ns = [16, 40, 24]
    batch = problem_mod.make_batch(Ns, seed0=30, dt=0.01)
    out = {}
    for pre in (0, 1, 2):
        sv = gpt.Solver(max_knot_points=64, max_batch=len(Ns), **SPEC_CFG)
        sv.set_solver(sqp_max_iter=3, pcg_max_iter=50000, pcg_exit_tol=1e-8, pcg_precond=pre, pcg_cluster_size=1)
        xu = dev(batch["xu"])
        rho, st = sv.sqp_solve_batched(Ns, dev(batch["goal"]), dev(batch["lam"]), xu, [1e-3] * len(Ns))
        out[pre] = (host(xu), rho, [s["sqp_iters"] for s in st], sum(s["pcg_iters_total"] for s in st))
        sv.close()
    x0 = batch["xu"].astype(np.float64)
    x1, x2 = out[1][0], out[2][0]
    assert out[2][2] == out[1][2] and out[2][1] == pytest.approx(out[1][1], rel=1e-6)
    step = np.linalg.norm(x1 - x0)
    assert np.linalg.norm(x2 - x1) <= 1e-2 * step, (np.linalg.norm(x2 - x1), step)
    assert out[2][3] < out[0][3], (out[2][3], out[0][3])
