"""gpt_ls_compute_merit_noalloc (the handle-free, allocation-free line-search
merit) against gpt_ls_compute_merit on the same inputs, through the C ABI.

The file name sorts last so that a run stopping at its first failure has run
every other test before this one."""
import ctypes as C

import numpy as np
import pytest

from conftest import ref_problem

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

REF_CFG = dict(timestep=1.0 / 64, integrator=0, qd_cost=1e-4, r_cost=1e-4)
SPEC_CFG = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def case(N, p, seed):
    rng = np.random.default_rng(seed)
    dz = rng.normal(0, 0.05, 21 * N - 7).astype(np.float32)
    xs = (p["xs"] + rng.normal(0, 0.01, 14)).astype(np.float32)
    return dev(xs), dev(p["xu"]), dev(p["goal"]), dev(dz)


def test_noalloc_merit_matches_handle_entry_point(gpt, golden, problem_mod):
    """Calls in a row (N = 64 spec problem, then N = 32 reference problem, so the second
    call leaves the first call's tail of the shared scratch untouched, then the largest
    accepted size, GPT_NOALLOC_MAX_KNOTS = 512, which fills the whole array): each call's
    8 merits equal the handle-based entry point's within the line-search merit tolerance
    of the parity tests (relative 5e-5 + 1e-5)."""
    L = gpt.lib()
    cases = [(64, SPEC_CFG, problem_mod.make_problem(64, 3, dt=0.01), 11),
             (32, REF_CFG, ref_problem(golden, 32), 12),
             (gpt.NOALLOC_MAX_KNOTS, SPEC_CFG, problem_mod.make_problem(gpt.NOALLOC_MAX_KNOTS, 4, dt=0.01), 13)]
    for N, cfg, p, seed in cases:
        xs, xu, goal, dz = case(N, p, seed)
        pc = gpt.default_problem_config(**cfg)
        got = torch.full((8,), float("nan"), device="cuda")
        st = L.gpt_ls_compute_merit_noalloc(C.byref(pc), N, gpt._ptr(xs), gpt._ptr(xu), gpt._ptr(goal),
                                            gpt._ptr(dz), gpt._ptr(got), gpt._stream(None))
        assert st == gpt.GPT_OK, L.gpt_last_error().decode()
        sv = gpt.Solver(max_knot_points=N, **cfg)
        want = torch.zeros(8, device="cuda")
        sv.ls_compute_merit(N, xs, xu, goal, dz, want)
        torch.cuda.synchronize()
        sv.close()
        g, w = got.cpu().numpy().astype(np.float64), want.cpu().numpy().astype(np.float64)
        assert np.all(np.isfinite(g)), (N, g)
        assert np.all(np.abs(g - w) <= 5e-5 * np.abs(w) + 1e-5), (N, g, w)


def test_noalloc_merit_rejects_sizes_beyond_its_scratch(gpt):
    pc = gpt.default_problem_config(**SPEC_CFG)
    N = gpt.NOALLOC_MAX_KNOTS + 1
    x = torch.zeros(21 * N, device="cuda")
    with pytest.raises(gpt.GptError, match="knot_points out of range"):
        gpt.ls_compute_merit_noalloc(pc, N, x, x, x, x, x)
