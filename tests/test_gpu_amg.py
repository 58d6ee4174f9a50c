"""CompactAMGPreconditioner on the GPU against its CPU restatement
(oracle.AmgOracle): the same hierarchy (level sizes and nonzeros), the same
V-cycle (applies within 1e-10 relative; the device sums rows in its own
order) and CG with it taking the oracle's iteration count."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(n, with_fd=True):
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(n).tocsr()
    fd = P.boundary_freedofs_7pt(n) if with_fd else None
    b = P.random_rhs(A.shape[0], 3)
    return A, fd, b


@pytest.mark.parametrize("with_fd", [True, False])
@pytest.mark.parametrize("kw", [dict(), dict(num_smooth=2), dict(min_coarse=200, theta=0.3), dict(max_levels=2)])
def test_amg_hierarchy_and_apply_match_oracle(with_fd, kw):
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A, fd, b = _system(14, with_fd)
    p = ss.CompactAMGPreconditioner(A, freedofs=fd, **kw)
    assert isinstance(p, ss.CompactAMGPreconditionerImpl)
    o = O.AmgOracle(A, freedofs=fd, **kw)
    assert p.levels() == o.levels()
    y = p * b
    yo = o.apply(b)
    assert np.abs(y - yo).max() <= 1e-10 * np.abs(yo).max()
    if fd is not None:
        assert not np.any(y[~fd.astype(bool)])


def test_amg_preconditioned_cg_matches_oracle():
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A, fd, b = _system(18)
    free = fd.astype(bool)
    Am = A.multiply(np.outer(free, free)).tolil()
    for i in np.where(~free)[0]:
        Am[i, i] = 1.0
    Am = Am.tocsr()
    bb = np.where(free, b, 0)
    p = ss.CompactAMGPreconditioner(A, freedofs=fd)
    cg = ss.PCGSolver(A, p, freedofs=fd, maxiter=200, tol=1e-10)
    x = np.zeros_like(b)
    r = cg.Solve(b, x)
    assert r.converged
    assert np.linalg.norm(bb - Am @ x) <= 1e-9 * np.linalg.norm(bb)
    o = O.AmgOracle(A, freedofs=fd)
    xs = np.zeros_like(b)
    rr = bb.copy()
    z = o.apply(rr)
    pp = z.copy()
    rz = rr @ z
    its = 0
    while its < 200:
        Ap = Am @ pp
        a = rz / (pp @ Ap)
        xs += a * pp
        rr -= a * Ap
        its += 1
        if np.linalg.norm(rr) / np.linalg.norm(bb) < 1e-10:
            break
        z = o.apply(rr)
        rzn = rr @ z
        pp = z + (rzn / rz) * pp
        rz = rzn
    assert abs(r.iterations - its) <= 1
    assert np.abs(x - xs).max() <= 1e-8 * np.abs(xs).max()


def test_amg_rejects_complex_and_updates():
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    from sparsesolv_ngsolve import _capi
    from sparsesolv_ngsolve import problems as P
    with pytest.raises(TypeError):
        ss.CompactAMGPreconditioner(P.complex_shifted(P.laplacian_7pt(6), 0.1j))
    A, fd, b = _system(10)
    p = ss.CompactAMGPreconditioner(A, freedofs=fd)
    A.data *= 3.0  # in place; ssv_precond_update re-reads the values and rebuilds
    p._mat.refresh()
    _capi.check(p._lib.ssv_precond_update(p._h))
    yo = O.AmgOracle(A, freedofs=fd).apply(b)
    assert np.abs(p * b - yo).max() <= 1e-10 * np.abs(yo).max()
