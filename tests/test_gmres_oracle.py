"""The GMRES restatement (oracle/gmres_oracle.py) on the CPU: it solves
non-symmetric real and complex systems to its tolerance, with and without
restarts and a preconditioner, and its edge cases follow the reference's
source (zero right-hand side, maxiter exhausted)."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import gmres_oracle as G
from oracle import oracle as O
from sparsesolv_ngsolve import problems as P


def _nonsym(n3, cplx=False):
    A = P.laplacian_7pt(n3).tocsr()
    n = A.shape[0]
    E = sp.random(n, n, 0.004, random_state=3).tocsr()
    A = (A + 0.5 * E).tocsr()
    if cplx:
        A = (A + 0.3j * sp.eye(n)).tocsr()
    A.sort_indices()
    return A


def test_gmres_oracle_solves_nonsymmetric_systems():
    for cplx in (False, True):
        A = _nonsym(7, cplx)
        b = P.random_rhs(A.shape[0], 1, np.complex128 if cplx else np.float64)
        for restart in (0, 15):
            x, it = G.gmres(A, b, tol=1e-10, maxiter=400, restart=restart)
            assert 0 < it < 400
            assert np.linalg.norm(b - A @ x) <= 2e-10 * np.linalg.norm(b)
            np.testing.assert_allclose(x, spla.spsolve(A.tocsc(), b), rtol=0, atol=1e-8 * np.abs(x).max())


def test_gmres_oracle_preconditioned_and_edges():
    A = _nonsym(6)
    n = A.shape[0]
    b = P.random_rhs(n, 2)
    fd = P.boundary_freedofs_7pt(6)
    x0, it0 = G.gmres(A, b, freedofs=fd, tol=1e-10, maxiter=300)
    x1, it1 = G.gmres(A, b, pre=lambda v: O.sgs_mult(A, v, freedofs=fd), freedofs=fd, tol=1e-10, maxiter=300)
    assert it1 < it0
    assert not np.any(x1[~fd.astype(bool)])
    np.testing.assert_allclose(x1, x0, rtol=0, atol=1e-7 * np.abs(x0).max())
    x, it = G.gmres(A, np.zeros(n), tol=1e-10)
    assert it == 0 and not np.any(x)
    x, it = G.gmres(A, b, tol=1e-14, maxiter=5)
    assert it == 5
