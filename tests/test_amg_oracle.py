"""The CompactAMGPreconditioner restatement (oracle/ams_oracle.cpp, AmgOracle)
on the CPU: the hierarchy coarsens an H1 Laplacian down to a direct coarsest
level, and CG with its V-cycle converges in a mesh-independent handful of
iterations, with and without FreeDofs."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from sparsesolv_ngsolve import problems as P


def _cg(A, b, apply, tol=1e-10, maxit=300):
    x = np.zeros_like(b)
    r = b - A @ x
    z = apply(r)
    p = z.copy()
    rz = r @ z
    nb = np.linalg.norm(b)
    for it in range(1, maxit + 1):
        Ap = A @ p
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        if np.linalg.norm(r) / nb < tol:
            return x, it
        z = apply(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return x, maxit


def test_amg_oracle_hierarchy_and_cg():
    its = []
    for n in (12, 20):
        A = P.laplacian_7pt(n).tocsr()
        fd = P.boundary_freedofs_7pt(n)
        free = fd.astype(bool)
        Am = A.multiply(np.outer(free, free)).tolil()
        for i in np.where(~free)[0]:
            Am[i, i] = 1.0
        Am = Am.tocsr()
        b = np.where(free, P.random_rhs(A.shape[0], 0), 0)
        g = O.AmgOracle(A, freedofs=fd)
        lv = g.levels()
        assert len(lv) >= 2 and lv[-1][0] <= 500 and all(lv[k + 1][0] < lv[k][0] for k in range(len(lv) - 1))
        x, it = _cg(Am, b, g.apply)
        assert np.linalg.norm(b - Am @ x) <= 1e-9 * np.linalg.norm(b)
        assert not np.any(g.apply(b)[~free])
        its.append(it)
    assert its[1] <= its[0] + 6
