"""B200-native SQP inner loop for 7-DOF iiwa end-effector tracking.

Python front end of libgpt.so (the C ABI in include/gpt.h).  It mirrors the
reference's host interface for this path (gpu-pcg-tracking toplevel.cuh
sqpSolve and the kernels it launches) on torch CUDA tensors; torch only
supplies device memory and streams.  There is no CPU implementation: if the
CUDA library is missing or no GPU is visible, every call raises.

The directory name contains hyphens, so import it with
``importlib.import_module("gpu-pcg-tracking_b200")``.
"""
from __future__ import annotations

import collections.abc
import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpt.so")

GPT_OK = 0
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "CUDA", 3: "NO_DEVICE", 4: "CAPACITY", 5: "NONFINITE", 6: "FACTOR"}
EXIT_RHO_MAX, EXIT_PCG_MAXITER, EXIT_NONFINITE, EXIT_ITER_LIMIT, EXIT_FACTOR = 1, 2, 4, 8, 16

STATE_SIZE, CONTROL_SIZE = 14, 7
PCG_WARP_PAIR = 32  # GPT_PCG_WARP_PAIR: pcg_cluster_size of the one-CTA-per-instance warp-pair PCG
PCG_WARP_QUAD = 64  # GPT_PCG_WARP_QUAD: pcg_cluster_size of the one-CTA-per-instance partitioned PCG (4 warps)

# The C-ABI entry points include/gpt.h declares (checked by the CPU tests).
EXPORTED = [
    "gpt_default_problem_config", "gpt_default_solver_config", "gpt_create", "gpt_destroy",
    "gpt_set_solver_config", "gpt_last_error", "gpt_version", "gpt_sqp_solve", "gpt_sqp_solve_batched",
    "gpt_form_kkt", "gpt_form_schur", "gpt_form_schur_csc", "gpt_prep_csr", "gpt_pcg", "gpt_compute_dz",
    "gpt_compute_merit", "gpt_ls_compute_merit", "gpt_set_profiling", "gpt_get_phase_stats",
    "gpt_ls_compute_merit_noalloc", "gpt_sqp_adjoint", "gpt_set_cost_weights", "gpt_autotune",
    "gpt_default_track_config", "gpt_track", "gpt_track_batched", "gpt_track_batched_adjoint", "gpt_simulate",
    "gpt_end_effector_positions", "gpt_forward_dynamics", "gpt_read_csv", "gpt_form_ss",
    "gpt_forward_dynamics_gradient", "gpt_sqp_solve_batched_trace",
]
PHASES = ["init", "kkt", "schur", "pcg", "dz", "merit", "accept"]
# gpt_iterate_record as 14 floats: rho, rho_next, merit_prev, merits[8], alpha, active (uint32), pcg_iters (uint32)
TRACE_REC_FLOATS = 14
TRACE_REC = {"rho": 0, "rho_next": 1, "merit_prev": 2, "merits": slice(3, 11), "alpha": 11, "active": 12,
             "pcg_iters": 13}


def trace_record_fields(rec):
    """Decode rows of gpt_iterate_record (a float32 tensor/array [..., 14]) into a dict of numpy arrays."""
    import numpy as np
    a = rec.cpu().numpy() if hasattr(rec, "cpu") else np.asarray(rec, dtype=np.float32)
    u = a.view(np.uint32)
    return {"rho": a[..., 0], "rho_next": a[..., 1], "merit_prev": a[..., 2], "merits": a[..., 3:11],
            "alpha": a[..., 11], "active": u[..., 12], "pcg_iters": u[..., 13]}


class ProblemConfig(C.Structure):
    """gpt_problem_config (include/gpt.h)."""
    _fields_ = [("state_size", C.c_uint32), ("control_size", C.c_uint32), ("max_knot_points", C.c_uint32),
                ("max_batch", C.c_uint32), ("timestep", C.c_float), ("integrator", C.c_uint32),
                ("q_ee", C.c_float), ("qd_cost", C.c_float), ("r_cost", C.c_float), ("mu", C.c_float),
                ("ref_terminal", C.c_uint32)]


class SolverConfig(C.Structure):
    """gpt_solver_config (include/gpt.h)."""
    _fields_ = [("sqp_max_iter", C.c_uint32), ("pcg_max_iter", C.c_uint32), ("pcg_exit_tol", C.c_float),
                ("pcg_exit_mode", C.c_uint32), ("rho_factor", C.c_float), ("rho_max", C.c_float),
                ("rho_min", C.c_float), ("pcg_cluster_size", C.c_uint32), ("pcg_precond", C.c_uint32),
                ("schur_fp64", C.c_uint32), ("sqp_graph", C.c_uint32)]


class SqpStats(C.Structure):
    """gpt_sqp_stats (include/gpt.h)."""
    _fields_ = [("sqp_iters", C.c_uint32), ("exit_flags", C.c_uint32), ("pcg_iters_total", C.c_uint32),
                ("pcg_maxiter_count", C.c_uint32), ("ls_fail_count", C.c_uint32), ("merit_initial", C.c_float),
                ("merit_final", C.c_float), ("rho_final", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TrackConfig(C.Structure):
    """gpt_track_config (include/gpt.h)."""
    _fields_ = [("sim_period_us", C.c_float), ("sim_step", C.c_float), ("shift_threshold", C.c_float),
                ("max_control_updates", C.c_uint32), ("jitter_solves", C.c_uint32), ("rho_reset", C.c_float)]


class TrackStats(C.Structure):
    """gpt_track_stats (include/gpt.h)."""
    _fields_ = [("control_updates", C.c_uint32), ("shifts", C.c_uint32), ("sqp_iters_total", C.c_uint32),
                ("pcg_iters_total", C.c_uint32), ("ls_fail_total", C.c_uint32), ("pcg_maxiter_total", C.c_uint32),
                ("rho_exits", C.c_uint32), ("nonfinite", C.c_uint32), ("tracking_error_mean", C.c_float),
                ("final_tracking_error", C.c_float), ("rho_final", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StatsList(collections.abc.Sequence):
    """Per-instance stats of a batched call, converted to dicts on access (a batch of
    hundreds of instances costs milliseconds of host time to convert eagerly)."""

    def __init__(self, arr):
        self._arr = arr

    def __len__(self):
        return len(self._arr)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self._arr[j].as_dict() for j in range(*i.indices(len(self._arr)))]
        return self._arr[i].as_dict()


class GptError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gpt {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def build(force: bool = False) -> str:
    """Compile libgpt.so for sm_100a with nvcc (csrc/Makefile)."""
    args = ["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


_LIB = None


def lib():
    """The loaded CUDA library; raises if it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with csrc/Makefile (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _LIB = L
    return _LIB


def _declare(L):
    vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    P = C.POINTER
    sig = {
        "gpt_default_problem_config": ([P(ProblemConfig)], None),
        "gpt_default_solver_config": ([P(SolverConfig)], None),
        "gpt_create": ([P(ProblemConfig), P(SolverConfig), P(vp)], C.c_int),
        "gpt_destroy": ([vp], C.c_int),
        "gpt_set_solver_config": ([vp, P(SolverConfig)], C.c_int),
        "gpt_last_error": ([], C.c_char_p),
        "gpt_version": ([], C.c_char_p),
        "gpt_sqp_solve": ([vp, u32, vp, vp, vp, P(f32), f32, P(SqpStats), vp, vp, vp], C.c_int),
        "gpt_sqp_solve_batched": ([vp, u32, vp, vp, vp, vp, vp, f32, vp, vp], C.c_int),
        "gpt_form_kkt": ([vp, u32, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_form_schur": ([vp, u32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_form_schur_csc": ([vp, u32, f32, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_prep_csr": ([u32, vp, vp], C.c_int),
        "gpt_pcg": ([vp, u32, vp, vp, vp, vp, vp, u32, f32, u32, P(u32), P(C.c_uint8), vp], C.c_int),
        "gpt_compute_dz": ([vp, u32, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_compute_merit": ([vp, u32, vp, vp, vp, vp], C.c_int),
        "gpt_ls_compute_merit": ([vp, u32, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_set_profiling": ([vp, C.c_int], C.c_int),
        "gpt_get_phase_stats": ([vp, vp, vp, C.c_int], C.c_int),
        "gpt_ls_compute_merit_noalloc": ([P(ProblemConfig), u32, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_sqp_adjoint": ([vp, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "gpt_set_cost_weights": ([vp, f32, f32, f32], C.c_int),
        "gpt_autotune": ([vp, u32, vp, vp, vp, vp, vp, P(u32), vp, vp], C.c_int),
        "gpt_default_track_config": ([P(TrackConfig)], None),
        "gpt_track": ([vp, u32, u32, vp, vp, vp, P(TrackConfig), vp, vp, u32, P(TrackStats), vp], C.c_int),
        "gpt_track_batched": ([vp, u32, vp, vp, vp, vp, vp, P(TrackConfig), vp, vp, u32, vp, vp], C.c_int),
        "gpt_track_batched_adjoint": ([vp, u32, vp, vp, vp, vp, vp, P(TrackConfig), vp, vp, u32, vp, vp, vp, vp, vp],
                                      C.c_int),
        "gpt_simulate": ([vp, u32, vp, vp, C.c_double, C.c_double, f32, vp], C.c_int),
        "gpt_end_effector_positions": ([u32, vp, u32, vp, vp], C.c_int),
        "gpt_forward_dynamics": ([u32, vp, u32, vp, vp], C.c_int),
        "gpt_read_csv": ([C.c_char_p, vp, C.c_size_t, P(u32), P(u32)], C.c_int),
        "gpt_form_ss": ([vp, u32, vp, vp, vp], C.c_int),
        "gpt_forward_dynamics_gradient": ([u32, vp, u32, vp, vp, vp], C.c_int),
        "gpt_sqp_solve_batched_trace": ([vp, u32, vp, vp, vp, vp, vp, f32, vp, u32, vp, vp, vp, vp, vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res


def _check(st: int):
    if st != GPT_OK:
        raise GptError(st, lib().gpt_last_error().decode())


def default_problem_config(**kw) -> ProblemConfig:
    pc = ProblemConfig()
    lib().gpt_default_problem_config(C.byref(pc))
    for k, v in kw.items():
        setattr(pc, k, v)
    return pc


def default_solver_config(**kw) -> SolverConfig:
    sc = SolverConfig()
    lib().gpt_default_solver_config(C.byref(sc))
    for k, v in kw.items():
        setattr(sc, k, v)
    return sc


def default_track_config(**kw) -> TrackConfig:
    tc = TrackConfig()
    lib().gpt_default_track_config(C.byref(tc))
    for k, v in kw.items():
        setattr(tc, k, v)
    return tc


def end_effector_positions(x, row_stride: int, out=None, stream=None):
    """gpt_end_effector_positions: xyz + roll/pitch/yaw of every row of x (CUDA tensor, rows of
    row_stride floats starting with q) -> tensor [rows, 6]."""
    import torch
    n = x.numel() // row_stride
    if out is None:
        out = torch.empty(n, 6, device=x.device)
    _check(lib().gpt_end_effector_positions(n, _ptr(x), row_stride, _ptr(out), _stream(stream)))
    return out


def forward_dynamics(xu, row_stride: int = 21, out=None, stream=None):
    """gpt_forward_dynamics: qdd of every row [q, qd, u] of xu (CUDA tensor) -> tensor [rows, 7]."""
    import torch
    n = xu.numel() // row_stride
    if out is None:
        out = torch.empty(n, 7, device=xu.device)
    _check(lib().gpt_forward_dynamics(n, _ptr(xu), row_stride, _ptr(out), _stream(stream)))
    return out


def forward_dynamics_gradient(xu, row_stride: int = 21, stream=None):
    """gpt_forward_dynamics_gradient: (qdd [rows, 7], df/du [rows, 147] = 7 x 21 column-major)."""
    import torch
    n = xu.numel() // row_stride
    qdd = torch.empty(n, 7, device=xu.device)
    df = torch.empty(n, 147, device=xu.device)
    _check(lib().gpt_forward_dynamics_gradient(n, _ptr(xu), row_stride, _ptr(qdd), _ptr(df), _stream(stream)))
    return qdd, df


def read_csv(path: str):
    """gpt_read_csv (readCSVToVecVec, runme.cu:18-44): a float32 numpy array [rows, cols]."""
    import numpy as np
    r, c = C.c_uint32(0), C.c_uint32(0)
    _check(lib().gpt_read_csv(path.encode(), None, 0, C.byref(r), C.byref(c)))
    out = np.zeros((r.value, c.value), np.float32)
    _check(lib().gpt_read_csv(path.encode(), out.ctypes.data_as(C.c_void_p), out.size, C.byref(r), C.byref(c)))
    return out


NOALLOC_MAX_KNOTS = 512  # GPT_NOALLOC_MAX_KNOTS


def ls_compute_merit_noalloc(problem: ProblemConfig, N, xs, xu, eePos, dz, out, stream=None):
    """gpt_ls_compute_merit_noalloc: the 8 line-search merits with no handle and no
    device allocation (scratch is a fixed 16 KiB array inside the library, shared
    by every call on a device)."""
    _check(lib().gpt_ls_compute_merit_noalloc(C.byref(problem), N, _ptr(xs), _ptr(xu), _ptr(eePos), _ptr(dz),
                                              _ptr(out), _stream(stream)))


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


@dataclass
class SqpResult:
    """What sqpSolve returns (toplevel.cuh:502) plus the device-side stats."""
    pcg_iters: List[int]
    pcg_exit: List[bool]
    sqp_iters: int
    rho: float
    stats: dict = field(default_factory=dict)


class Solver:
    """A gpt_handle: workspace for max_batch x max_knot_points, preallocated."""

    def __init__(self, problem: Optional[ProblemConfig] = None, solver: Optional[SolverConfig] = None, **kw):
        pkw = {k: v for k, v in kw.items() if k in dict(ProblemConfig._fields_)}
        skw = {k: v for k, v in kw.items() if k in dict(SolverConfig._fields_)}
        unknown = set(kw) - set(pkw) - set(skw)
        if unknown:
            raise TypeError(f"unknown config keys {sorted(unknown)}")
        self.problem = problem or default_problem_config(**pkw)
        self.solver = solver or default_solver_config(**skw)
        h = C.c_void_p()
        _check(lib().gpt_create(C.byref(self.problem), C.byref(self.solver), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().gpt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_solver(self, **kw):
        for k, v in kw.items():
            setattr(self.solver, k, v)
        _check(lib().gpt_set_solver_config(self._h, C.byref(self.solver)))

    def set_cost_weights(self, q_ee: float, qd_cost: float, r_cost: float):
        """gpt_set_cost_weights: the end-effector, joint-velocity and control weights of later calls."""
        _check(lib().gpt_set_cost_weights(self._h, q_ee, qd_cost, r_cost))
        self.problem.q_ee, self.problem.qd_cost, self.problem.r_cost = q_ee, qd_cost, r_cost

    def reset_solver(self, **kw):
        """gpt_default_solver_config, then the given fields."""
        self.solver = default_solver_config(**kw)
        _check(lib().gpt_set_solver_config(self._h, C.byref(self.solver)))

    def set_profiling(self, enable: bool):
        _check(lib().gpt_set_profiling(self._h, int(bool(enable))))

    def phase_stats(self, reset: bool = False):
        """{phase: (device ms, launches)} accumulated while profiling was on."""
        ms = (C.c_double * len(PHASES))()
        n = (C.c_uint64 * len(PHASES))()
        _check(lib().gpt_get_phase_stats(self._h, C.cast(ms, C.c_void_p), C.cast(n, C.c_void_p), int(reset)))
        return {p: (ms[i], n[i]) for i, p in enumerate(PHASES)}

    # ---- the SQP solve (toplevel.cuh:24-503) ----
    def sqp_solve(self, knot_points: int, eePos_traj, lam, xu, rho: float, rho_reset: float = 1e-3,
                  stream=None) -> SqpResult:
        r = C.c_float(rho)
        st = SqpStats()
        n = self.solver.sqp_max_iter
        iters = (C.c_uint32 * n)()
        ex = (C.c_uint8 * n)()
        _check(lib().gpt_sqp_solve(self._h, knot_points, _ptr(eePos_traj), _ptr(lam), _ptr(xu), C.byref(r),
                                   rho_reset, C.byref(st), C.cast(iters, C.c_void_p), C.cast(ex, C.c_void_p),
                                   _stream(stream)))
        k = st.sqp_iters
        return SqpResult(list(iters)[:k], [bool(x) for x in list(ex)[:k]], k, r.value, st.as_dict())

    def sqp_solve_batched(self, knot_points: Sequence[int], eePos_traj, lam, xu, rho: Sequence[float],
                          rho_reset: float = 1e-3, stream=None):
        B = len(knot_points)
        Ns = (C.c_uint32 * B)(*knot_points)
        rr = (C.c_float * B)(*rho)
        sts = (SqpStats * B)()
        _check(lib().gpt_sqp_solve_batched(self._h, B, C.cast(Ns, C.c_void_p), _ptr(eePos_traj), _ptr(lam),
                                           _ptr(xu), C.cast(rr, C.c_void_p), rho_reset, C.cast(sts, C.c_void_p),
                                           _stream(stream)))
        return list(rr), StatsList(sts)

    def sqp_solve_batched_trace(self, knot_points: Sequence[int], eePos_traj, lam, xu, rho: Sequence[float],
                                trace_iters: int, rho_reset: float = 1e-3, stream=None):
        """gpt_sqp_solve_batched_trace: the batched solve with its first trace_iters iterates recorded.
        Returns (rho list, stats, trace) with trace = {"xu": [I, 21T], "lam": [I, 14T] (FP64),
        "dz": [I, 21T], "rec": [I, B, 14] float32 rows of gpt_iterate_record (TRACE_REC fields)}."""
        import torch
        B = len(knot_points)
        T = int(sum(knot_points))
        dev = xu.device
        tr = {"xu": torch.zeros(trace_iters, 21 * T, device=dev),
              "lam": torch.zeros(trace_iters, 14 * T, dtype=torch.float64, device=dev),
              "dz": torch.zeros(trace_iters, 21 * T, device=dev),
              "rec": torch.zeros(trace_iters, B, TRACE_REC_FLOATS, device=dev)}
        Ns = (C.c_uint32 * B)(*knot_points)
        rr = (C.c_float * B)(*rho)
        sts = (SqpStats * B)()
        _check(lib().gpt_sqp_solve_batched_trace(self._h, B, C.cast(Ns, C.c_void_p), _ptr(eePos_traj), _ptr(lam),
                                                 _ptr(xu), C.cast(rr, C.c_void_p), rho_reset,
                                                 C.cast(sts, C.c_void_p), trace_iters, _ptr(tr["xu"]),
                                                 _ptr(tr["lam"]), _ptr(tr["dz"]), _ptr(tr["rec"]), _stream(stream)))
        return list(rr), StatsList(sts), tr

    def autotune(self, knot_points: Sequence[int], eePos_traj, lam, xu, rho: Sequence[float], stream=None,
                 schedule: Optional[dict] = None) -> int:
        """gpt_autotune: pick and remember the fastest PCG kernel and per-knot launch schedule for this batch
        shape.  Returns the PCG cluster size; `schedule` (a dict, optional) receives the CTAs per SM chosen
        for the KKT, Schur, merit and dz launches and the part-batch branches per graph iteration
        ("branches": tuned when sqp_graph is 1, else the configured value)."""
        B = len(knot_points)
        Ns = (C.c_uint32 * B)(*knot_points)
        rr = (C.c_float * B)(*rho)
        cs = C.c_uint32(0)
        sched = (C.c_uint32 * 5)()
        _check(lib().gpt_autotune(self._h, B, C.cast(Ns, C.c_void_p), _ptr(eePos_traj), _ptr(lam), _ptr(xu),
                                  C.cast(rr, C.c_void_p), C.byref(cs), C.cast(sched, C.c_void_p), _stream(stream)))
        if schedule is not None:
            schedule.update(dict(zip(("kkt", "schur", "merit", "dz", "branches"), list(sched))))
        return cs.value

    def sqp_adjoint(self, knot_points: Sequence[int], eePos_traj, xs, xu, rho: Sequence[float], grad_xu_next,
                    xu_next=None, stream=None):
        """gpt_sqp_adjoint: gradients of l(xu - dz) at the iterate xu given dl/dxu+.
        Returns {"goal": [6 per knot], "qd": [B, 7], "r": [B, 7], "q_ee": [B]} (CUDA tensors)."""
        import torch
        B = len(knot_points)
        T = sum(knot_points)
        Ns = (C.c_uint32 * B)(*knot_points)
        rr = (C.c_float * B)(*rho)
        out = {"goal": torch.zeros(6 * T, device=xu.device), "qd": torch.zeros(B, 7, device=xu.device),
               "r": torch.zeros(B, 7, device=xu.device), "q_ee": torch.zeros(B, device=xu.device)}
        _check(lib().gpt_sqp_adjoint(self._h, B, C.cast(Ns, C.c_void_p), _ptr(eePos_traj), _ptr(xs), _ptr(xu),
                                     C.cast(rr, C.c_void_p), _ptr(grad_xu_next), _ptr(xu_next), _ptr(out["goal"]),
                                     _ptr(out["qd"]), _ptr(out["r"]), _ptr(out["q_ee"]), _stream(stream)))
        return out

    # ---- the MPC tracking loop (toplevel.cuh:507-796) ----
    def track(self, knot_points: int, eePos_traj, xu_traj, xs, config: Optional[TrackConfig] = None,
              errors=None, sqp_iters_log=None, stream=None):
        """gpt_track: receding-horizon tracking of one trajectory (rows of 6 / 21 floats); xs is the
        plant state, updated in place.  Returns (per-shift tracking errors, stats dict)."""
        import torch
        S = eePos_traj.numel() // 6
        if errors is None:
            errors = torch.zeros(S, device=xs.device)
        st = TrackStats()
        cap = 0 if sqp_iters_log is None else sqp_iters_log.numel()
        _check(lib().gpt_track(self._h, knot_points, S, _ptr(eePos_traj), _ptr(xu_traj), _ptr(xs),
                               None if config is None else C.byref(config), _ptr(errors), _ptr(sqp_iters_log), cap,
                               C.byref(st), _stream(stream)))
        d = st.as_dict()
        return errors[:st.shifts], d

    def track_batched(self, knot_points: Sequence[int], traj_steps: Sequence[int], eePos_traj, xu_traj, xs,
                      config: Optional[TrackConfig] = None, errors=None, sqp_iters_log=None, log_capacity=0,
                      stream=None):
        """gpt_track_batched: many tracking runs; instance b owns trajectory rows
        sum(traj_steps[:b]) .. + traj_steps[b]-1.  Returns (errors tensor, list of stats dicts)."""
        import torch
        B = len(knot_points)
        Ns = (C.c_uint32 * B)(*knot_points)
        Ss = (C.c_uint32 * B)(*traj_steps)
        if errors is None:
            errors = torch.zeros(int(sum(traj_steps)), device=xs.device)
        sts = (TrackStats * B)()
        _check(lib().gpt_track_batched(self._h, B, C.cast(Ns, C.c_void_p), C.cast(Ss, C.c_void_p), _ptr(eePos_traj),
                                       _ptr(xu_traj), _ptr(xs), None if config is None else C.byref(config),
                                       _ptr(errors), _ptr(sqp_iters_log), log_capacity, C.cast(sts, C.c_void_p),
                                       _stream(stream)))
        return errors, StatsList(sts)

    def track_batched_adjoint(self, knot_points: Sequence[int], traj_steps: Sequence[int], eePos_traj, xu_traj, xs,
                              config: Optional[TrackConfig] = None, errors=None, sqp_iters_log=None, log_capacity=0,
                              stream=None):
        """gpt_track_batched_adjoint: gpt_track_batched plus, after every control update's solve, the
        one-step adjoint of that update's horizon tracking loss; returns (errors, stats, weight_grad
        [B, 15] = (dl/dqd, dl/dr, dl/dq_ee) summed over each instance's updates, loss [B], adjoint
        failures per instance)."""
        import torch
        B = len(knot_points)
        Ns = (C.c_uint32 * B)(*knot_points)
        Ss = (C.c_uint32 * B)(*traj_steps)
        if errors is None:
            errors = torch.zeros(int(sum(traj_steps)), device=xs.device)
        wgrad = torch.zeros(B, 15, device=xs.device)
        loss = torch.zeros(B, device=xs.device)
        fails = (C.c_uint32 * B)()
        sts = (TrackStats * B)()
        _check(lib().gpt_track_batched_adjoint(
            self._h, B, C.cast(Ns, C.c_void_p), C.cast(Ss, C.c_void_p), _ptr(eePos_traj), _ptr(xu_traj), _ptr(xs),
            None if config is None else C.byref(config), _ptr(errors), _ptr(sqp_iters_log), log_capacity,
            _ptr(wgrad), _ptr(loss), C.cast(fails, C.c_void_p), C.cast(sts, C.c_void_p), _stream(stream)))
        return errors, StatsList(sts), wgrad, loss, list(fails)

    def simulate(self, knot_points: int, xs, xu, time_offset_us: float, sim_time_us: float, sim_step: float = 2e-4,
                 stream=None):
        """gpt_simulate (simple_simulate, integrator.cuh:365-398): advances xs in place."""
        _check(lib().gpt_simulate(self._h, knot_points, _ptr(xs), _ptr(xu), time_offset_us, sim_time_us, sim_step,
                                  _stream(stream)))

    # ---- the reference's kernels, one instance ----
    def form_kkt(self, N, xu, eePos, xs, G, Cm, g, c, stream=None):
        _check(lib().gpt_form_kkt(self._h, N, _ptr(xu), _ptr(eePos), _ptr(xs), _ptr(G), _ptr(Cm), _ptr(g), _ptr(c),
                                  _stream(stream)))

    def form_schur(self, N, rho, G, Cm, g, c, S, Pinv, gamma, Ginv, Ginv64=None, stream=None):
        _check(lib().gpt_form_schur(self._h, N, rho, _ptr(G), _ptr(Cm), _ptr(g), _ptr(c), _ptr(S), _ptr(Pinv),
                                    _ptr(gamma), _ptr(Ginv), _ptr(Ginv64), _stream(stream)))

    def form_schur_csc(self, N, rho, G, Cm, g, c, val, gamma, Ginv, stream=None):
        _check(lib().gpt_form_schur_csc(self._h, N, rho, _ptr(G), _ptr(Cm), _ptr(g), _ptr(c), _ptr(val),
                                        _ptr(gamma), _ptr(Ginv), _stream(stream)))

    def form_ss(self, N, S, Pinv, stream=None):
        """gpt_form_ss: the stair preconditioner's off-diagonal blocks written into Pinv."""
        _check(lib().gpt_form_ss(self._h, N, _ptr(S), _ptr(Pinv), _stream(stream)))

    def pcg(self, N, S, Pinv, gamma, lam, max_iter, exit_tol, exit_mode=0, lam64=None, stream=None):
        it = C.c_uint32(0)
        mx = C.c_uint8(0)
        _check(lib().gpt_pcg(self._h, N, _ptr(S), _ptr(Pinv), _ptr(gamma), _ptr(lam), _ptr(lam64), max_iter,
                             exit_tol, exit_mode, C.byref(it), C.byref(mx), _stream(stream)))
        return it.value, bool(mx.value)

    def compute_dz(self, N, Ginv, Cm, g, lam, dz, lam64=None, Ginv64=None, stream=None):
        _check(lib().gpt_compute_dz(self._h, N, _ptr(Ginv), _ptr(Ginv64), _ptr(Cm), _ptr(g), _ptr(lam), _ptr(lam64),
                                    _ptr(dz), _stream(stream)))

    def compute_merit(self, N, xu, eePos, out, stream=None):
        _check(lib().gpt_compute_merit(self._h, N, _ptr(xu), _ptr(eePos), _ptr(out), _stream(stream)))

    def ls_compute_merit(self, N, xs, xu, eePos, dz, out, stream=None):
        _check(lib().gpt_ls_compute_merit(self._h, N, _ptr(xs), _ptr(xu), _ptr(eePos), _ptr(dz), _ptr(out),
                                          _stream(stream)))


def prep_csr(N: int):
    """CSC pattern of the Schur matrix's upper triangle (prep_csr, utils.cuh:84-118)."""
    import numpy as np
    nnz = 196 * (N - 1) + 105 * N
    cp = np.zeros(14 * N + 1, np.int32)
    ri = np.zeros(nnz, np.int32)
    _check(lib().gpt_prep_csr(N, cp.ctypes.data_as(C.c_void_p), ri.ctypes.data_as(C.c_void_p)))
    return cp, ri
