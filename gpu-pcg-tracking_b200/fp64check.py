"""FP64 host re-solve of one SQP iteration's KKT system, for accuracy reports.

Given the KKT blocks that the CUDA KKT kernel formed at an iterate (G, C, g, c in the
reference's layouts, include/gpt.h) and the iteration's rho, this forms the Schur
complement in FP64 with the reference's formulas (gato_form_schur_jacobi_inner,
oldschur.cuh:518-963: phi_k = (-A_{k-1}) Q~_{k-1}^{-1}, theta_k, gamma_k), solves
(-S) lambda = (-gamma) by an FP64 block-tridiagonal Cholesky, and recovers dz
(oldschur.cuh:966-1105).  The product computes none of its results here: this is the
FP64 yardstick that bench.py and the tests hold the GPU's lambda and dz against
("relative error of every result against an FP64 host banded Cholesky").
"""
from __future__ import annotations

import numpy as np

NS, NC, NX = 14, 7, 21
SS, CC = NS * NS, NC * NC
GSTRIDE, CSTRIDE = SS + CC, SS + NS * NC


def _blocks(N, G, Cm, g, c):
    G = np.asarray(G, np.float64)
    Cm = np.asarray(Cm, np.float64)
    g = np.asarray(g, np.float64)
    c = np.asarray(c, np.float64).reshape(N, NS)
    Q = np.stack([G[GSTRIDE * k:GSTRIDE * k + SS].reshape(NS, NS, order="F") for k in range(N)])
    R = np.stack([G[GSTRIDE * k + SS:GSTRIDE * (k + 1)].reshape(NC, NC, order="F") for k in range(N - 1)])
    mA = np.stack([Cm[CSTRIDE * k:CSTRIDE * k + SS].reshape(NS, NS, order="F") for k in range(N - 1)])
    mB = np.stack([Cm[CSTRIDE * k + SS:CSTRIDE * (k + 1)].reshape(NS, NC, order="F") for k in range(N - 1)])
    q = np.stack([g[NX * k:NX * k + NS] for k in range(N)])
    r = np.stack([g[NX * k + NS:NX * (k + 1)] for k in range(N - 1)])
    return Q, R, mA, mB, q, r, c


def schur(N, rho, G, Cm, g, c):
    """FP64 Schur system of the KKT blocks: returns (M_diag [N,14,14], M_sub [N,14,14] (block (k, k-1)
    of M = -S; entry 0 unused), rhs = -gamma [N,14], Qi [N,14,14], Ri [N-1,7,7], mA, mB, q, r)."""
    Q, R, mA, mB, q, r, c = _blocks(N, G, Cm, g, c)
    Qi = np.linalg.inv(Q + rho * np.eye(NS))
    Ri = np.linalg.inv(R + rho * np.eye(NC)) if N > 1 else np.zeros((0, NC, NC))
    D = np.zeros((N, NS, NS))
    E = np.zeros((N, NS, NS))
    rhs = np.zeros((N, NS))
    D[0] = Qi[0]
    rhs[0] = Qi[0] @ q[0]
    if N > 1:
        phi = mA @ Qi[:-1]                       # (-A_{k-1}) Q~_{k-1}^{-1}, k = 1 .. N-1
        BRi = mB @ Ri                            # (-B_{k-1}) R~_{k-1}^{-1}
        D[1:] = phi @ np.transpose(mA, (0, 2, 1)) + BRi @ np.transpose(mB, (0, 2, 1)) + Qi[1:]
        E[1:] = phi                              # M_{k,k-1} = -S[k].left = phi_k
        rhs[1:] = (np.einsum("kij,kj->ki", Qi[1:], q[1:]) - c[1:] + np.einsum("kij,kj->ki", phi, q[:-1])
                   + np.einsum("kij,kj->ki", BRi, r))
    return D, E, rhs, Qi, Ri, mA, mB, q, r


def block_cholesky_solve(D, E, rhs):
    """Solve M x = rhs for the SPD block-tridiagonal M (diagonal D_k, sub-diagonal E_k = M_{k,k-1})
    by a block Cholesky factorisation in FP64."""
    N = D.shape[0]
    L = np.zeros_like(D)
    W = np.zeros_like(D)  # W_k = E_k L_{k-1}^{-T}
    for k in range(N):
        Dk = D[k].copy()
        if k > 0:
            W[k] = np.linalg.solve(L[k - 1], E[k].T).T
            Dk -= W[k] @ W[k].T
        L[k] = np.linalg.cholesky(0.5 * (Dk + Dk.T))
    y = np.zeros((N, NS))
    for k in range(N):
        b = rhs[k] - (W[k] @ y[k - 1] if k > 0 else 0.0)
        y[k] = np.linalg.solve(L[k], b)
    x = np.zeros((N, NS))
    for k in range(N - 1, -1, -1):
        b = y[k] - (W[k + 1].T @ x[k + 1] if k < N - 1 else 0.0)
        x[k] = np.linalg.solve(L[k].T, b)
    return x


def solve_step(N, rho, G, Cm, g, c):
    """The FP64 lambda [14N] and dz [21N-7] of one SQP iteration from its KKT blocks."""
    D, E, rhs, Qi, Ri, mA, mB, q, r = schur(N, rho, G, Cm, g, c)
    lam = block_cholesky_solve(D, E, rhs)
    dz = np.zeros(NX * N - NC)
    for k in range(N):
        s = lam[k] + (mA[k].T @ lam[k + 1] if k < N - 1 else 0.0)
        dz[NX * k:NX * k + NS] = Qi[k] @ (q[k] - s)
        if k < N - 1:
            dz[NX * k + NS:NX * (k + 1)] = Ri[k] @ (r[k] - mB[k].T @ lam[k + 1])
    return lam.reshape(-1), dz


def rel_err(got, want):
    """max |got - want| / max |want| (0 when both vanish)."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    den = np.abs(want).max() if want.size else 0.0
    num = np.abs(got - want).max() if want.size else 0.0
    return float(num / den) if den > 0 else float(num)
