"""Parity against the reference's own kernels.

oracle/ref_harness builds the reference's gato_form_kkt, form_schur,
form_schur_qdl, prep_csr, compute_dz and its qdldl helper from the
reference's sources (stand-ins only for the three empty submodules).  On the
same inputs, these tests check
  * the CUDA product against the reference kernels, and
  * the C restatement (oracle.c, FP64) against the reference kernels, which
    pins the oracle the other parity tests use.
Tolerances are relative to the largest magnitude of each quantity over the
instance: both sides compute in FP32, so they agree to FP32 rounding
(1e-7 .. 1e-5 relative after the reductions), except where the reference's
FP32 Gauss-Jordan sets the floor (Ginv), stated per check.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ref_problem

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ref_py  # noqa: E402

REF_CFG = dict(timestep=1.0 / 64, integrator=0, qd_cost=1e-4, r_cost=1e-4)
SPEC_CFG = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)


def dev(a, dtype=np.float32):
    return torch.as_tensor(np.ascontiguousarray(a, dtype), device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def zeros(n):
    return torch.zeros(n, device="cuda")


def cases(golden, problem_mod):
    out = []
    for N in (2, 3, 32, 128):
        out.append(("ref", N, REF_CFG, ref_problem(golden, N)))
    for N in (4, 64, 128):
        out.append(("spec", N, SPEC_CFG, problem_mod.make_problem(N, 7, dt=0.01)))
    return out


@pytest.fixture(scope="module")
def reference():
    if not (ref_py.available(1e-4) and ref_py.available(1e-2)):
        pytest.skip("reference harness not built (make -C oracle ref needs the reference tree)")
    return {1e-4: ref_py.Reference(1e-4), 1e-2: ref_py.Reference(1e-2)}


@pytest.fixture(scope="module")
def solvers(gpt):
    cache = {}

    def get(cfg):
        key = tuple(sorted(cfg.items()))
        if key not in cache:
            cache[key] = gpt.Solver(max_knot_points=512, **cfg)
        cache[key].reset_solver()
        return cache[key]
    yield get
    for s in cache.values():
        s.close()


def agree(got, want, rtol, what, scale=None):
    s = np.abs(want).max() if scale is None else scale
    err = np.abs(got - want).max() if got.size else 0.0
    assert err <= rtol * max(s, 1e-30), f"{what}: max err {err:.3e} vs scale {s:.3e} (rtol {rtol})"


def kkt_blocks(N, G, g):
    Q = np.concatenate([G[245 * k:245 * k + 196] for k in range(N)])
    R = np.concatenate([G[245 * k + 196:245 * k + 245] for k in range(N - 1)])
    qq = np.concatenate([g[21 * k:21 * k + 7] for k in range(N)])
    qd = np.concatenate([g[21 * k + 7:21 * k + 14] for k in range(N)])
    r = np.concatenate([g[21 * k + 14:21 * k + 21] for k in range(N - 1)])
    return {"Q": Q, "R": R, "q_q": qq, "q_qd": qd, "r": r}


def ref_kkt(reference, cfg, N, p):
    R = reference[cfg["qd_cost"]]
    G, Cm, g, c = zeros(245 * N - 49), zeros(294 * (N - 1)), zeros(21 * N - 7), zeros(14 * N)
    R.form_kkt(N, cfg["timestep"], cfg["integrator"], G, Cm, g, c, dev(p["goal"]), dev(p["xs"]), dev(p["xu"]))
    return host(G), host(Cm), host(g), host(c)


def test_kkt_matches_reference_kernel(gpt, oracle, golden, problem_mod, reference, solvers):
    """gato_form_kkt (schur.cuh:391-524) vs gpt_form_kkt and vs the oracle's
    form_kkt, including the reference's terminal target (its kernel overwrites
    goal_{N-1} in shared memory before reading it)."""
    for kind, N, cfg, p in cases(golden, problem_mod):
        rG, rC, rg, rc = ref_kkt(reference, cfg, N, p)
        sv = solvers(cfg)
        G, Cm, g, c = (zeros(n) for n in (245 * N - 49, 294 * (N - 1), 21 * N - 7, 14 * N))
        sv.form_kkt(N, dev(p["xu"]), dev(p["goal"]), dev(p["xs"]), G, Cm, g, c)
        par = oracle.make_params(dt=cfg["timestep"], integrator=cfg["integrator"], qd_cost=cfg["qd_cost"],
                                 r_cost=cfg["r_cost"], ref_terminal=1)
        oG, oC, og, oc = (np.asarray(a) for a in oracle.form_kkt(par, N, p["xu"], p["goal"], p["xs"]))
        refb = kkt_blocks(N, rG, rg)
        for who, (GG, CC, gg, cc) in (("gpu", (host(G), host(Cm), host(g), host(c))), ("oracle", (oG, oC, og, oc))):
            b = kkt_blocks(N, GG, gg)
            # position-cost gradient and q q^T: FK in FP32 on both sides
            agree(b["Q"], refb["Q"], 1e-5, f"{who} {kind} N={N} Q")
            agree(b["q_q"], refb["q_q"], 1e-5, f"{who} {kind} N={N} q_q")
            # QD, R terms are single products of the same FP32 inputs
            agree(b["R"], refb["R"], 1e-7, f"{who} {kind} N={N} R")
            agree(b["q_qd"], refb["q_qd"], 1e-6, f"{who} {kind} N={N} q_qd")
            agree(b["r"], refb["r"], 1e-6, f"{who} {kind} N={N} r", scale=max(np.abs(refb["r"]).max(), 1e-12))
            # -A, -B from the dynamics gradient (FP32 Minv and RNEA derivatives)
            agree(CC, rC, 1e-5, f"{who} {kind} N={N} C")
            # defects: differences of FP32 states, |x| <= ~5
            agree(cc, rc, 1e-5, f"{who} {kind} N={N} c", scale=np.abs(p["xu"]).max())


def test_schur_matches_reference_kernel(gpt, oracle, golden, problem_mod, reference, solvers):
    """form_schur (oldschur.cuh:518-963) vs gpt_form_schur and the oracle on the
    reference's own KKT output: S (3-block layout), gamma, the block-Jacobi
    Pinv diagonal, and the inverses the reference writes over G."""
    rho = 1e-3
    for kind, N, cfg, p in cases(golden, problem_mod):
        rG, rC, rg, rc = ref_kkt(reference, cfg, N, p)
        R = reference[cfg["qd_cost"]]
        rS, rP, rgam, rGi = zeros(588 * N), zeros(588 * N), zeros(14 * N), dev(rG)
        R.form_schur(N, rho, rGi, dev(rC), dev(rg), dev(rc), rS, rP, rgam)
        rS, rP, rgam, rGi = host(rS), host(rP), host(rgam), host(rGi)
        sv = solvers(cfg)
        S, Pv, gam, Gi = zeros(588 * N), zeros(588 * N), zeros(14 * N), zeros(245 * N - 49)
        sv.form_schur(N, rho, dev(rG), dev(rC), dev(rg), dev(rc), S, Pv, gam, Gi)
        oS, oP, ogam, oGi = (np.asarray(a) for a in oracle.form_schur(N, rho, rG, rC, rg, rc))
        diag = np.concatenate([np.arange(588 * k + 196, 588 * k + 392) for k in range(N)])
        for who, (SS_, PP, GA, GI) in (("gpu", (host(S), host(Pv), host(gam), host(Gi))),
                                       ("oracle", (oS, oP, ogam, oGi))):
            agree(SS_, rS, 1e-6, f"{who} {kind} N={N} S")
            agree(GA, rgam, 1e-4, f"{who} {kind} N={N} gamma")
            agree(PP[diag], rP[diag], 1e-5, f"{who} {kind} N={N} Pinv diagonal")
            # the reference inverts Q + rho I, R + rho I by FP32 Gauss-Jordan without pivoting
            # (oldschur.cuh:214-332); cond ~1e3 at rho = 1e-3 sets its error (~2e-6 of the scale)
            agree(GI, rGi, 1e-5, f"{who} {kind} N={N} Ginv")


def test_csc_pattern_and_values_match_reference(gpt, golden, problem_mod, reference, solvers):
    """prep_csr (utils.cuh:84-118) and form_schur_qdl (schur.cuh:57-383): the CSC
    pattern is identical, the values and gamma agree to FP32 rounding."""
    rho = 1e-3
    for kind, N, cfg, p in cases(golden, problem_mod):
        rG, rC, rg, rc = ref_kkt(reference, cfg, N, p)
        R = reference[cfg["qd_cost"]]
        nnz = 196 * (N - 1) + 105 * N
        rcp = torch.zeros(14 * N + 1, dtype=torch.int32, device="cuda")
        rri = torch.zeros(nnz, dtype=torch.int32, device="cuda")
        R.prep_csr(N, rcp, rri)
        cp, ri = gpt.prep_csr(N)
        assert np.array_equal(rcp.cpu().numpy(), cp) and np.array_equal(rri.cpu().numpy(), ri), (kind, N)
        rval, rgam = zeros(nnz), zeros(14 * N)
        R.form_schur_qdl(N, rho, dev(rG), dev(rC), dev(rg), dev(rc), rval, rgam)
        sv = solvers(cfg)
        val, gam, Gi = zeros(nnz), zeros(14 * N), zeros(245 * N - 49)
        sv.form_schur_csc(N, rho, dev(rG), dev(rC), dev(rg), dev(rc), val, gam, Gi)
        agree(host(val), host(rval), 1e-6, f"{kind} N={N} csc values")
        agree(host(gam), host(rgam), 1e-4, f"{kind} N={N} csc gamma")


def test_dz_matches_reference_kernel(gpt, oracle, golden, problem_mod, reference, solvers):
    """compute_dz (oldschur.cuh:966-1105) on the reference's Ginv, C, g and a
    seeded lambda: GPU and oracle vs the reference kernel."""
    rho = 1e-3
    for kind, N, cfg, p in cases(golden, problem_mod):
        rG, rC, rg, rc = ref_kkt(reference, cfg, N, p)
        R = reference[cfg["qd_cost"]]
        rS, rP, rgam, rGi = zeros(588 * N), zeros(588 * N), zeros(14 * N), dev(rG)
        R.form_schur(N, rho, rGi, dev(rC), dev(rg), dev(rc), rS, rP, rgam)
        lam = np.random.default_rng(N).normal(0, 1, 14 * N).astype(np.float32)
        rdz, dz = zeros(21 * N - 7), zeros(21 * N - 7)
        R.compute_dz(N, rGi, dev(rC), dev(rg), dev(lam), rdz)
        sv = solvers(cfg)
        sv.compute_dz(N, rGi, dev(rC), dev(rg), dev(lam), dz)
        odz = np.asarray(oracle.compute_dz(N, host(rGi), rC, rg, lam.astype(np.float64)))
        agree(host(dz), host(rdz), 1e-6, f"gpu {kind} N={N} dz")
        agree(odz, host(rdz), 1e-6, f"oracle {kind} N={N} dz")


def test_reference_qdldl_path_accuracy(gpt, oracle, golden, problem_mod, reference, solvers):
    """The reference's qdldl linear solve (qdldl_helper.cuh:62-180, FP32, with
    the oracle's QDLDL-API LDL^T) against the FP64 banded Cholesky of the same
    Schur system, next to the B200 PCG (block-tridiagonal preconditioner,
    relative residual 1e-8): the B200 solve is as close to FP64 as the
    reference's qdldl path, or as the floor that FP32 formation of S sets for
    both (the qdldl path's FP32 factorisation loses up to ~1e-2 at
    cond(S) ~ 1e7)."""
    rho = 1e-3
    for kind, N, cfg, p in cases(golden, problem_mod):
        if N < 32:
            continue
        rG, rC, rg, rc = ref_kkt(reference, cfg, N, p)
        R = reference[cfg["qd_cost"]]
        nnz = 196 * (N - 1) + 105 * N
        rval, rgam = zeros(nnz), zeros(14 * N)
        R.form_schur_qdl(N, rho, dev(rG), dev(rC), dev(rg), dev(rc), rval, rgam)
        cp, ri = gpt.prep_csr(N)
        lam_q = np.zeros(14 * N, np.float32)
        R.qdldl_solve(N, cp, ri, host(rval).astype(np.float32), host(rgam).astype(np.float32), lam_q)
        oS, oP, ogam, oGi = (np.asarray(a) for a in oracle.form_schur(N, rho, rG, rC, rg, rc))
        lam64 = np.asarray(oracle.banded_cholesky(N, oS, ogam))
        sv = solvers(cfg)
        S, Pv, gam, Gi = zeros(588 * N), zeros(588 * N), zeros(14 * N), zeros(245 * N - 49)
        sv.form_schur(N, rho, dev(rG), dev(rC), dev(rg), dev(rc), S, Pv, gam, Gi)
        lam, l64 = zeros(14 * N), torch.zeros(14 * N, device="cuda", dtype=torch.float64)
        it, maxed = sv.pcg(N, S, Pv, gam, lam, 100000, 1e-8, 0, lam64=l64)
        assert not maxed
        # floor shared by both: S formed in FP32 (exact FP64 solve of the oracle's FP32 Schur data)
        fS, _, fgam, _ = oracle.form_schur(N, rho, rG, rC, rg, rc, precision="f32")
        lam_f = np.asarray(oracle.banded_cholesky(N, np.asarray(fS, np.float64), np.asarray(fgam, np.float64)))
        nrm = np.linalg.norm(lam64)
        e_q = np.linalg.norm(lam_q - lam64) / nrm
        e_g = np.linalg.norm(host(l64) - lam64) / nrm
        e_f = np.linalg.norm(lam_f - lam64) / nrm
        assert e_q < 5e-2, (kind, N, e_q)
        assert e_g <= 2 * max(e_q, e_f), (kind, N, e_g, e_q, e_f)
