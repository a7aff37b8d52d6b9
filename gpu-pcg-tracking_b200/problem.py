"""Seeded synthetic tracking problems for the iiwa14 SQP inner loop.

Input synthesis only (host numpy); the solver itself runs in libgpt.so.

One problem (instance seed s, horizon N, timestep dt):
  * 5 joint-space waypoints drawn uniform in +-0.5 * joint limits.  The
    limits are the KUKA LBR iiwa 14 R820 axis ranges from its public data
    sheet / URDF: A1..A7 = 170, 120, 170, 120, 170, 120, 175 degrees (the
    reference does not ship them).
  * a natural cubic spline through the waypoints, evenly spaced over a
    path duration T_path (default 2 s, i.e. the 200 control steps of the
    closed-loop rollout at dt = 0.01); knot k samples the path at
    t = min(k dt, T_path), so horizons longer than the path hold the last
    waypoint.  The reference end-effector path is the forward kinematics
    (xyz + roll/pitch/yaw, the layout of the reference's
    testfiles/*_eepos.traj) of the spline at every knot.
  * initial guess xu: spline q and qd at each knot, controls 0.
  * initial state x_s = waypoint 0 + N(0, sigma) per joint, zero velocity;
    it is written into x_0 (sqpSolve takes x_s from x_0, toplevel.cuh:110).
No public dataset or benchmark suite is involved.
"""
from __future__ import annotations

import numpy as np

JOINT_LIMITS_DEG = np.array([170.0, 120.0, 170.0, 120.0, 170.0, 120.0, 175.0])
JOINT_LIMITS = np.deg2rad(JOINT_LIMITS_DEG)

# joint origin offsets and fixed rotations of the iiwa14 kinematic chain
_JOINT_P = np.array([[0, 0, 0.1575], [0, 0, 0.2025], [0, 0.2045, 0], [0, 0, 0.2155],
                     [0, 0.1845, 0], [0, 0, 0.2155], [0, 0.081, 0]], dtype=np.float64)
_RF = {0: np.eye(3), 1: np.array([[-1.0, 0, 0], [0, 0, 1], [0, 1, 0]]), 2: np.array([[1.0, 0, 0], [0, 0, -1], [0, 1, 0]])}
_KIND = [0, 1, 1, 2, 1, 2, 1]


def fk_xyzrpy(q: np.ndarray) -> np.ndarray:
    """End-effector xyz + roll/pitch/yaw for joint vectors q [..., 7] (float64)."""
    q = np.asarray(q, np.float64)
    shp = q.shape[:-1]
    qf = q.reshape(-1, 7)
    out = np.zeros((qf.shape[0], 6))
    for n, qq in enumerate(qf):
        R = np.eye(3)
        o = np.zeros(3)
        for j in range(7):
            o = o + R @ _JOINT_P[j]
            c, s = np.cos(qq[j]), np.sin(qq[j])
            Rz = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
            R = R @ _RF[_KIND[j]] @ Rz
        out[n, :3] = o
        out[n, 3] = np.arctan2(R[2, 1], R[2, 2])
        out[n, 4] = -np.arctan2(R[2, 0], np.sqrt(R[2, 1] ** 2 + R[2, 2] ** 2))
        out[n, 5] = np.arctan2(R[1, 0], R[0, 0])
    return out.reshape(shp + (6,))


def _natural_spline(tw, W, t, deriv=0):
    from scipy.interpolate import CubicSpline
    return CubicSpline(tw, W, axis=0, bc_type="natural")(t, deriv)


def make_problem(N: int, seed: int, dt: float = 0.01, n_waypoints: int = 5, sigma: float = 0.01,
                 t_path: float = 2.0):
    """Returns dict(xu [21N-7], goal [6N], lam [14N], xs [14]) as float32 arrays."""
    rng = np.random.default_rng(1234 + seed)
    W = rng.uniform(-0.5, 0.5, size=(n_waypoints, 7)) * JOINT_LIMITS
    tw = np.linspace(0.0, t_path, n_waypoints)
    t_raw = np.arange(N) * dt
    t = np.minimum(t_raw, t_path)
    q = _natural_spline(tw, W, t, 0)
    qd = _natural_spline(tw, W, t, 1) * (t_raw <= t_path)[:, None]
    goal = fk_xyzrpy(q).astype(np.float32).reshape(-1)
    xs = np.concatenate([W[0] + rng.normal(0.0, sigma, 7), np.zeros(7)])
    xu = np.zeros(21 * N, np.float64)
    for k in range(N):
        xu[21 * k:21 * k + 7] = q[k]
        xu[21 * k + 7:21 * k + 14] = qd[k]
    xu[:14] = xs
    return {"xu": xu[:21 * N - 7].astype(np.float32), "goal": goal, "lam": np.zeros(14 * N, np.float32),
            "xs": xs.astype(np.float32)}


def make_batch(Ns, seed0: int = 0, dt: float = 0.01, sigma: float = 0.01, t_path: float = 2.0):
    """Concatenated batch (knot-slot layout of include/gpt.h): instance b uses seed seed0 + b."""
    Ns = [int(n) for n in Ns]
    K = int(np.sum(Ns))
    xu = np.zeros(21 * K, np.float32)
    goal = np.zeros(6 * K, np.float32)
    lam = np.zeros(14 * K, np.float32)
    off = 0
    for b, N in enumerate(Ns):
        p = make_problem(N, seed0 + b, dt=dt, sigma=sigma, t_path=t_path)
        xu[21 * off:21 * off + 21 * N - 7] = p["xu"]
        goal[6 * off:6 * off + 6 * N] = p["goal"]
        off += N
    return {"xu": xu, "goal": goal, "lam": lam, "Ns": Ns}


def make_trajectory_rows(S: int, seed: int, dt: float = 0.01, n_waypoints: int = 5, sigma: float = 0.01,
                         t_path: float = 2.0):
    """One seeded tracking trajectory as S rows of 21 floats (q, qd, u = 0) -- the row layout of the
    reference's testfiles/*_traj.csv -- and the initial plant state x_s (waypoint 0 + N(0, sigma),
    zero velocity), written into row 0.  The goal rows are the end-effector poses of the rows' q
    (make_problem computes them on the host; a batch can use gpt_end_effector_positions)."""
    rng = np.random.default_rng(1234 + seed)
    W = rng.uniform(-0.5, 0.5, size=(n_waypoints, 7)) * JOINT_LIMITS
    tw = np.linspace(0.0, t_path, n_waypoints)
    t_raw = np.arange(S) * dt
    t = np.minimum(t_raw, t_path)
    rows = np.zeros((S, 21), np.float64)
    rows[:, :7] = _natural_spline(tw, W, t, 0)
    rows[:, 7:14] = _natural_spline(tw, W, t, 1) * (t_raw <= t_path)[:, None]
    xs = np.concatenate([W[0] + rng.normal(0.0, sigma, 7), np.zeros(7)])
    rows[0, :14] = xs
    return rows.astype(np.float32), xs.astype(np.float32)
