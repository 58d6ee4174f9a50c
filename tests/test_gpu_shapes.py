"""Ragged and tiny shapes for every sub-warp width of the CSR kernels:
sizes that are not multiples of the rows handled by one warp, 1x1 systems,
empty rows, dense rows."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _spd_band(n, half_bw, seed=0, cplx=False):
    """Diagonally dominant symmetric band matrix with half bandwidth half_bw."""
    rng = np.random.default_rng(seed)
    A = sp.lil_matrix((n, n), dtype=np.complex128 if cplx else np.float64)
    for i in range(n):
        for d in range(1, half_bw + 1):
            if i + d < n:
                v = -rng.uniform(0.1, 1.0)
                if cplx:
                    v = v + 0.1j * rng.uniform(-1, 1)
                A[i, i + d] = v
                A[i + d, i] = v
    A = A.tocsr()
    rs = np.asarray(abs(A).sum(axis=1)).ravel()
    A = (A + sp.diags(rs + 1.0)).tocsr()
    A.sort_indices()
    return A


# half bandwidth -> nnz/row ~ 1 + 2*hb: 1 (2 lanes), 2 (4), 4 (8), 8 (16), 16 (32)
@pytest.mark.parametrize("hb", [0, 1, 2, 4, 8, 16])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 17, 33, 131, 257])
def test_spmv_ragged(n, hb):
    from sparsesolv_ngsolve import _Matrix, _capi
    A = _spd_band(n, hb, seed=n + hb)
    m = _Matrix(A)
    x = np.random.default_rng(1).uniform(-1, 1, n)
    y = np.empty(n)
    _capi.check(_capi.load().ssv_matrix_spmv(m.h, _capi.vptr(x), _capi.vptr(y)))
    np.testing.assert_allclose(y, A @ x, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("method", ["CG", "ICCG", "COCR", "SGSMRTR"])
@pytest.mark.parametrize("n,hb", [(1, 0), (3, 1), (7, 2), (131, 4), (257, 8), (97, 16)])
def test_solve_ragged_vs_oracle(method, n, hb):
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A = _spd_band(n, hb, seed=3 * n + hb)
    b = np.random.default_rng(n).uniform(-1, 1, n)
    for abmc in (False, True):
        s = ss.SparseSolvSolver(A, method=method, use_abmc=abmc, maxiter=500)
        x = np.zeros(n)
        r = s.Solve(b, x)
        xo, ro, _ = O.solve(A, b, method, O.default_config(use_abmc=int(abmc), max_iterations=500))
        assert r.iterations == ro.iterations and r.converged == bool(ro.converged)
        assert np.abs(x - xo).max() <= 1e-8 * max(np.abs(xo).max(), 1e-300)


@pytest.mark.parametrize("n", [5, 66])
def test_complex_ragged(n):
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A = _spd_band(n, 3, seed=n, cplx=True)
    b = np.random.default_rng(n).uniform(-1, 1, n) + 1j
    for method in ("ICCG", "COCR", "CG"):
        s = ss.SparseSolvSolver(A, method=method, use_abmc=True, maxiter=300)
        x = np.zeros(n, complex)
        r = s.Solve(b, x)
        xo, ro, _ = O.solve(A, b, method, O.default_config(use_abmc=1, max_iterations=300))
        assert r.iterations == ro.iterations
        assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()


def test_empty_rows_identity_freedofs():
    """Constrained rows become identity rows; a row with no entries at all is
    handled by the CG path (no IC)."""
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A = _spd_band(40, 2, seed=7)
    fd = np.ones(40, np.uint8)
    fd[[0, 13, 39]] = 0
    b = np.random.default_rng(2).uniform(-1, 1, 40)
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, use_abmc=True)
    x = np.full(40, 7.0)
    r = s.Solve(b, x)
    xo, ro, _ = O.solve(A, b, "ICCG", O.default_config(use_abmc=1), freedofs=fd, x0=np.full(40, 7.0))
    assert r.iterations == ro.iterations
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()
    assert np.all(x[[0, 13, 39]] == 7.0)  # constrained entries untouched


@pytest.mark.parametrize("cplx", [False, True])
def test_large_value_refresh_through_staging(cplx):
    """Values above 16 MB are re-uploaded through the threaded pinned staging
    (8 host threads, 4 MB chunks, ragged last chunks): after an in-place change
    of the host matrix, refresh() must give exactly the new operator."""
    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(73, 71, 70).tocsr()  # 2.5M nnz: 20 MB of FP64 values, not a multiple of the chunk
    if cplx:
        A = P.complex_shifted(A, 0.3 + 0.7j).tocsr()
    rng = np.random.default_rng(5)
    m = ss._Matrix(A)
    A.data *= rng.uniform(0.5, 2.0, A.nnz)  # in place: same arrays, new values
    m.refresh()
    n = A.shape[0]
    x = rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)
    y = np.zeros(n, dtype=x.dtype)
    _capi.check(_capi.load().ssv_matrix_spmv(m.h, _capi.vptr(x), _capi.vptr(y)))
    ref = A @ x
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
