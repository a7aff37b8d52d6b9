"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE, not the product.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may import
this module, and only as the checker.  It wraps oracle/liboracle.so (built by
oracle/Makefile from oracle.c + ldl.c), the C restatement of the reference's
SQP inner loop (gpu-pcg-tracking toplevel.cuh:24-503 and the kernels it calls).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class Params(C.Structure):
    """orc_params (oracle.h)."""
    _fields_ = [("dt", C.c_double), ("integrator", C.c_int), ("q_ee", C.c_double),
                ("qd_cost", C.c_double), ("r_cost", C.c_double), ("mu", C.c_double),
                ("ref_terminal", C.c_int)]


class Solver(C.Structure):
    """orc_solver (oracle.h)."""
    _fields_ = [("linsys", C.c_int), ("sqp_max_iter", C.c_int), ("pcg_max_iter", C.c_int),
                ("pcg_tol", C.c_double), ("pcg_exit_mode", C.c_int), ("rho_factor", C.c_double),
                ("rho_max", C.c_double), ("rho_min", C.c_double)]


class TrackCfg(C.Structure):
    """orc_track_cfg (oracle.h)."""
    _fields_ = [("sim_period_us", C.c_double), ("sim_step", C.c_double), ("shift_threshold", C.c_double),
                ("max_control_updates", C.c_int), ("jitter_solves", C.c_int), ("rho_reset", C.c_double)]


class TrackStats(C.Structure):
    """orc_track_stats (oracle.h)."""
    _fields_ = [("control_updates", C.c_int), ("shifts", C.c_int), ("sqp_iters_total", C.c_int),
                ("pcg_iters_total", C.c_int), ("ls_fail_total", C.c_int), ("rho_exits", C.c_int),
                ("final_error", C.c_double), ("rho_final", C.c_double)]


class Stats(C.Structure):
    """orc_stats (oracle.h)."""
    _fields_ = [("sqp_iters", C.c_int), ("rho_exit", C.c_int), ("ls_fail_count", C.c_int),
                ("pcg_iters_total", C.c_int), ("pcg_maxiter_count", C.c_int),
                ("linsys_count", C.c_int), ("merit_final", C.c_double), ("rho_final", C.c_double)]


def build() -> str:
    """Compile the oracle with its Makefile (gcc); returns the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        _LIB = C.CDLL(LIB_PATH)
        _declare(_LIB)
    return _LIB


def _declare(L):
    for sfx, rp, rt in (("f32", _f32p, C.c_float), ("f64", _f64p, C.c_double)):
        def fn(name, argtypes, restype=None):
            f = getattr(L, f"orc_{sfx}_{name}")
            f.argtypes = argtypes
            f.restype = restype
        fn("fk", [rp, rp])
        fn("fk_grad", [rp, rp])
        fn("rnea", [rp, rp, rp, rp])
        fn("minv", [rp, rp])
        fn("fd", [rp, rp, rp, rp])
        fn("fd_grad", [rp, rp, rp, rp, rp])
        fn("form_kkt", [C.POINTER(Params), C.c_int, rp, rp, rp, rp, rp, rp, rp])
        fn("form_schur", [C.c_int, rt, rp, rp, rp, rp, rp, rp, rp, rp])
        fn("csc_pattern", [C.c_int, _i32p, _i32p])
        fn("csc_values", [C.c_int, rp, _f32p])
        fn("pcg", [C.c_int, rp, rp, rp, rp, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int)], C.c_int)
        fn("banded_cholesky", [C.c_int, rp, rp, _f64p], C.c_int)
        fn("compute_dz", [C.c_int, rp, rp, rp, rp, rp])
        fn("merit", [C.POINTER(Params), C.c_int, rp, C.c_void_p, rt, rp, rp, C.c_int, C.c_void_p], rt)
        fn("sqp_solve", [C.POINTER(Params), C.POINTER(Solver), C.c_int, rp, rp, rp, C.POINTER(rt), rt,
                         C.POINTER(Stats), C.c_void_p], C.c_int)
        fn("simulate", [C.c_int, rp, rp, C.c_double, C.c_double, C.c_double, C.c_double])
        fn("form_ss", [C.c_int, rp, rp])
        fn("track", [C.POINTER(Params), C.POINTER(Solver), C.POINTER(TrackCfg), C.c_int, C.c_int, rp, rp, rp, rp,
                     C.POINTER(TrackStats)], C.c_int)
    L.orc_ldl_solve.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p]
    L.orc_ldl_solve.restype = C.c_int


def _dt(precision):
    return np.float32 if precision == "f32" else np.float64


def _a(x, precision):
    return np.ascontiguousarray(x, dtype=_dt(precision))


def make_params(dt=1.0 / 64, integrator=0, q_ee=1.0, qd_cost=1e-4, r_cost=1e-4, mu=10.0, ref_terminal=1):
    return Params(dt, integrator, q_ee, qd_cost, r_cost, mu, ref_terminal)


def make_solver(linsys=0, sqp_max_iter=40, pcg_max_iter=167, pcg_tol=1e-5, pcg_exit_mode=0,
                rho_factor=1.2, rho_max=10.0, rho_min=1e-3):
    return Solver(linsys, sqp_max_iter, pcg_max_iter, pcg_tol, pcg_exit_mode, rho_factor, rho_max, rho_min)


def fk(q, precision="f64"):
    out = np.zeros(6, _dt(precision))
    getattr(lib(), f"orc_{precision}_fk")(_a(q, precision), out)
    return out


def fk_grad(q, precision="f64"):
    out = np.zeros(42, _dt(precision))
    getattr(lib(), f"orc_{precision}_fk_grad")(_a(q, precision), out)
    return out


def rnea(q, qd, qdd, precision="f64"):
    out = np.zeros(7, _dt(precision))
    getattr(lib(), f"orc_{precision}_rnea")(_a(q, precision), _a(qd, precision), _a(qdd, precision), out)
    return out


def minv(q, precision="f64"):
    out = np.zeros(49, _dt(precision))
    getattr(lib(), f"orc_{precision}_minv")(_a(q, precision), out)
    return out.reshape(7, 7, order="F")


def fd(q, qd, u, precision="f64"):
    out = np.zeros(7, _dt(precision))
    getattr(lib(), f"orc_{precision}_fd")(_a(q, precision), _a(qd, precision), _a(u, precision), out)
    return out


def fd_grad(q, qd, u, precision="f64"):
    qdd = np.zeros(7, _dt(precision))
    dfdu = np.zeros(147, _dt(precision))
    getattr(lib(), f"orc_{precision}_fd_grad")(_a(q, precision), _a(qd, precision), _a(u, precision), qdd, dfdu)
    return qdd, dfdu


def form_kkt(params, N, xu, goal, xs, precision="f64"):
    d = _dt(precision)
    G = np.zeros(245 * N - 49, d)
    Cm = np.zeros(294 * (N - 1), d)
    g = np.zeros(21 * N - 7, d)
    c = np.zeros(14 * N, d)
    # the oracle writes full strides; give it padded buffers and trim
    Gp, Cp, gp = np.zeros(245 * N, d), np.zeros(294 * N, d), np.zeros(21 * N, d)
    getattr(lib(), f"orc_{precision}_form_kkt")(C.byref(params), N, _a(xu, precision), _a(goal, precision),
                                               _a(xs, precision), Gp, Cp, gp, c)
    G[:] = Gp[:245 * N - 49]
    Cm[:] = Cp[:294 * (N - 1)]
    g[:] = gp[:21 * N - 7]
    return G, Cm, g, c


def form_schur(N, rho, G, Cm, g, c, precision="f64"):
    d = _dt(precision)
    Gp = np.zeros(245 * N, d); Gp[:len(G)] = G
    Cp = np.zeros(294 * N, d); Cp[:len(Cm)] = Cm
    gp = np.zeros(21 * N, d); gp[:len(g)] = g
    S = np.zeros(588 * N, d)
    P = np.zeros(588 * N, d)
    gam = np.zeros(14 * N, d)
    Gi = np.zeros(245 * N, d)
    getattr(lib(), f"orc_{precision}_form_schur")(N, rho, Gp, Cp, gp, _a(c, precision), S, P, gam, Gi)
    return S, P, gam, Gi[:245 * N - 49]


def csc_pattern(N):
    n = 14 * N
    nnz = 196 * (N - 1) + 105 * N
    cp = np.zeros(n + 1, np.int32)
    ri = np.zeros(nnz, np.int32)
    lib().orc_f64_csc_pattern(N, cp, ri)
    return cp, ri


def csc_values(N, S, precision="f64"):
    nnz = 196 * (N - 1) + 105 * N
    val = np.zeros(nnz, np.float32)
    getattr(lib(), f"orc_{precision}_csc_values")(N, _a(S, precision), val)
    return val


def ldl_solve(N, S, gamma, precision="f64"):
    cp, ri = csc_pattern(N)
    val = csc_values(N, S, precision)
    x = np.zeros(14 * N, np.float32)
    rc = lib().orc_ldl_solve(14 * N, cp, ri, val, np.ascontiguousarray(gamma, np.float32), x)
    if rc < 0:
        raise RuntimeError("LDL factorisation failed")
    return x


def pcg(N, S, P, gamma, lam0, max_iter, tol, exit_mode=0, precision="f64"):
    lam = _a(lam0, precision).copy()
    mx = C.c_int(0)
    it = getattr(lib(), f"orc_{precision}_pcg")(N, _a(S, precision), _a(P, precision), _a(gamma, precision),
                                               lam, max_iter, tol, exit_mode, C.byref(mx))
    return lam, it, bool(mx.value)


def banded_cholesky(N, S, gamma, precision="f64"):
    lam = np.zeros(14 * N, np.float64)
    rc = getattr(lib(), f"orc_{precision}_banded_cholesky")(N, _a(S, precision), _a(gamma, precision), lam)
    if rc < 0:
        raise RuntimeError("banded Cholesky failed (matrix not definite)")
    return lam


def compute_dz(N, Gi, Cm, g, lam, precision="f64"):
    d = _dt(precision)
    Gp = np.zeros(245 * N, d); Gp[:len(Gi)] = Gi
    Cp = np.zeros(294 * N, d); Cp[:len(Cm)] = Cm
    gp = np.zeros(21 * N, d); gp[:len(g)] = g
    dz = np.zeros(21 * N, d)
    getattr(lib(), f"orc_{precision}_compute_dz")(N, Gp, Cp, gp, _a(lam, precision), dz)
    return dz[:21 * N - 7]


def merit(params, N, xu, dz, alpha, goal, xs, line_search, precision="f64"):
    d = _dt(precision)
    xu_a = _a(xu, precision)
    knots = np.zeros(N, d)
    dz_a = None if dz is None else _a(dz, precision)
    f = getattr(lib(), f"orc_{precision}_merit")
    m = f(C.byref(params), N, xu_a, None if dz_a is None else dz_a.ctypes.data, alpha, _a(goal, precision),
          _a(xs, precision), int(line_search), knots.ctypes.data)
    return float(m), knots


def sqp_solve(params, solver, N, goal, lam, xu, rho, rho_reset=1e-3, precision="f64"):
    """Returns (xu, lambda, rho, stats, pcg_iters) after one reference-semantics sqpSolve."""
    d = _dt(precision)
    xu_a = _a(xu, precision).copy()
    lam_a = _a(lam, precision).copy()
    rho_c = (C.c_float if precision == "f32" else C.c_double)(rho)
    st = Stats()
    pit = np.zeros(max(1, solver.sqp_max_iter), np.int32)
    rc = getattr(lib(), f"orc_{precision}_sqp_solve")(C.byref(params), C.byref(solver), N, _a(goal, precision),
                                                     lam_a, xu_a, C.byref(rho_c), d(rho_reset).item(),
                                                     C.byref(st), pit.ctypes.data)
    if rc < 0:
        raise RuntimeError("oracle linear solve failed")
    return xu_a, lam_a, float(rho_c.value), st, pit[:st.linsys_count]


def make_track_cfg(sim_period_us=2000.0, sim_step=2e-4, shift_threshold=1.0 / 64, max_control_updates=100000,
                   jitter_solves=0, rho_reset=1e-3):
    return TrackCfg(sim_period_us, sim_step, shift_threshold, max_control_updates, jitter_solves, rho_reset)


def simulate(N, xs, xu, timestep, time_offset_us, sim_time_us, sim_step=2e-4, precision="f64"):
    """simple_simulate (integrator.cuh:365-398) on a copy of xs; returns the new state."""
    x = _a(xs, precision).copy()
    getattr(lib(), f"orc_{precision}_simulate")(N, x, _a(xu, precision), float(timestep), float(time_offset_us),
                                               float(sim_time_us), float(sim_step))
    return x


def track(params, solver, cfg, N, eePos_traj, xu_traj, xs, precision="f64"):
    """track (toplevel.cuh:507-796): returns (final xs, per-shift tracking errors, TrackStats)."""
    ee = _a(eePos_traj, precision).reshape(-1)
    tr = _a(xu_traj, precision).reshape(-1)
    S = ee.size // 6
    x = _a(xs, precision).copy()
    err = np.zeros(max(S, 1), _dt(precision))
    ts = TrackStats()
    rc = getattr(lib(), f"orc_{precision}_track")(C.byref(params), C.byref(solver), C.byref(cfg), N, S, ee, tr, x,
                                                 err, C.byref(ts))
    if rc < 0:
        raise RuntimeError("oracle linear solve failed")
    return x, err[:ts.shifts], ts


def form_ss(N, S, Pinv, precision="f64"):
    """gato_form_ss_inner (oldschur.cuh:334-494): Pinv with the stair preconditioner's
    off-diagonal blocks filled in (a copy)."""
    P = _a(Pinv, precision).copy()
    getattr(lib(), f"orc_{precision}_form_ss")(N, _a(S, precision), P)
    return P
