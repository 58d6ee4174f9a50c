"""Oracle (test infrastructure only): numpy restatement of GMRESSolverNGS::Mult
(include/sparsesolv/ngsolve/sparsesolv_solvers.hpp:409-584), the reference's
right-preconditioned, restarted GMRES with modified Gram-Schmidt and Givens
rotations, which lives only in its NGSolve adapter. NGSolve is absent here,
so this restatement is not pinned by a run of the reference ("parity
unpinned"); it follows the source line by line and the GPU path is checked
against it.

    x, iterations = gmres(A, b, pre=None, freedofs=None, maxiter=500, tol=1e-8, restart=0)

A: scipy sparse (real or complex), pre: callable y = M^{-1} x or None.
"""
from __future__ import annotations

import numpy as np


def _givens(a, b):
    """compute_givens (:547-562): [c s; -conj(s) c] [a; b] = [r; 0]."""
    if abs(b) < 1e-30:
        return 1.0, 0.0 * a
    if abs(a) < 1e-30:
        return 0.0, 1.0 + 0.0 * a
    denom = np.sqrt(abs(a) ** 2 + abs(b) ** 2)
    return abs(a) / denom, a * np.conj(b) / (abs(a) * denom)


def gmres(A, b, pre=None, freedofs=None, maxiter=500, tol=1e-8, restart=0):
    cplx = np.iscomplexobj(A.data) or np.iscomplexobj(b)
    dt = np.complex128 if cplx else np.float64
    n = A.shape[0]
    fd = None if freedofs is None else np.asarray(freedofs).astype(bool)

    def project(v):
        if fd is not None:
            v[~fd] = 0
        return v

    def inner(u, v):  # InnerProduct(u, v, conjugate = complex)
        return np.vdot(u, v) if cplx else float(u @ v)

    def norm(v):
        return float(np.sqrt(abs(inner(v, v))))

    sol = np.zeros(n, dt)
    r = project(np.array(b, dtype=dt))
    rhs = r.copy()
    rhs_norm = norm(r)
    if rhs_norm < 1e-30:
        return sol, 0
    beta = rhs_norm
    restart = restart if restart > 0 else maxiter
    m = min(maxiter, restart)
    total = 0
    cycle = 0
    while total < maxiter:
        if cycle > 0:
            r = project(rhs - A @ sol)
            beta = norm(r)
            if beta / rhs_norm < tol:
                break
        V = [(1.0 / beta) * r]
        Z = []
        H = []
        cs = np.zeros(m)
        sn = np.zeros(m, dt)
        g = np.zeros(m + 1, dt)
        g[0] = beta
        j = 0
        while j < m and total < maxiter:
            z = V[j].copy() if pre is None else np.asarray(pre(V[j]), dtype=dt)
            Z.append(z)
            w = project(A @ z)
            h = np.zeros(j + 2, dt)
            for i in range(j + 1):  # modified Gram-Schmidt
                h[i] = inner(V[i], w)
                w = w - h[i] * V[i]
            h_next = norm(w)
            h[j + 1] = h_next
            V.append((1.0 / h_next) * w if h_next > 1e-30 else np.zeros(n, dt))
            for i in range(j):  # previous rotations
                hi, hi1 = h[i], h[i + 1]
                h[i] = cs[i] * hi + sn[i] * hi1
                h[i + 1] = -np.conj(sn[i]) * hi + cs[i] * hi1
            cs[j], sn[j] = _givens(h[j], h[j + 1])
            h[j] = cs[j] * h[j] + sn[j] * h[j + 1]
            h[j + 1] = 0
            H.append(h)
            gj = g[j]
            g[j] = cs[j] * gj
            g[j + 1] = -np.conj(sn[j]) * gj
            res = abs(g[j + 1]) / rhs_norm
            if res < tol or h_next < 1e-30:
                j += 1
                total += 1
                break
            j += 1
            total += 1
        dim = j
        y = np.zeros(dim, dt)
        for i in range(dim - 1, -1, -1):  # back substitution
            y[i] = g[i]
            for k in range(i + 1, dim):
                y[i] -= H[k][i] * y[k]
            if abs(H[i][i]) > 1e-30:
                y[i] /= H[i][i]
        for i in range(dim):
            sol = sol + y[i] * Z[i]
        if abs(g[dim]) / rhs_norm < tol:
            break
        cycle += 1
    return sol, total
