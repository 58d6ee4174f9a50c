"""GMRESSolver on the GPU against the restatement of the reference's
GMRESSolverNGS (oracle/gmres_oracle.py; the reference's GMRES exists only in
its NGSolve adapter, so no run of it pins this): iteration counts within one
step, solutions to 1e-8 relative, true residual at the tolerance."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _nonsym(n3, cplx=False):
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(n3).tocsr()
    n = A.shape[0]
    A = (A + 0.5 * sp.random(n, n, 0.004, random_state=3).tocsr()).tocsr()
    if cplx:
        A = (A + 0.3j * sp.eye(n)).tocsr()
    A.sort_indices()
    return A


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("restart", [0, 12])
@pytest.mark.parametrize("with_pre", [False, True])
def test_gmres_matches_oracle(cplx, restart, with_pre):
    import sparsesolv_ngsolve as ss
    from oracle import gmres_oracle as G
    from oracle import oracle as O
    from sparsesolv_ngsolve import problems as P
    A = _nonsym(8, cplx)
    n = A.shape[0]
    b = P.random_rhs(n, 4, np.complex128 if cplx else np.float64)
    fd = P.boundary_freedofs_7pt(8)
    pre = ss.SGSPreconditioner(A, freedofs=fd) if with_pre else None
    opre = (lambda v: O.sgs_mult(A, v, freedofs=fd)) if with_pre else None
    inv = ss.GMRESSolver(A, pre, freedofs=fd, maxiter=400, tol=1e-10, restart=restart)
    assert isinstance(inv, ss.GMRESSolverC if cplx else ss.GMRESSolverD)
    x = inv * b
    xo, ito = G.gmres(A, b, pre=opre, freedofs=fd, maxiter=400, tol=1e-10, restart=restart)
    assert abs(inv.iterations - ito) <= 1, (inv.iterations, ito)
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()
    free = fd.astype(bool)
    assert not np.any(x[~free])
    Am = A.multiply(np.outer(free, free)).tocsr()
    bb = np.where(free, b, 0)
    assert np.linalg.norm((bb - Am @ x)[free]) <= 1e-9 * np.linalg.norm(bb)


def test_gmres_edges():
    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import problems as P
    A = _nonsym(6)
    n = A.shape[0]
    inv = ss.GMRESSolver(A, None, maxiter=5, tol=1e-14)
    x = inv * P.random_rhs(n, 1)
    assert inv.iterations == 5
    x = inv * np.zeros(n)
    assert inv.iterations == 0 and not np.any(x)
    with pytest.raises(TypeError):
        ss.GMRESSolver(A, ss.SGSPreconditioner(P.complex_shifted(P.laplacian_7pt(6), 0.1j)), maxiter=5) * np.ones(n)
