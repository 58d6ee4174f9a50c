"""The oracle (C restatement) against golden outputs of the reference itself."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, golden_system
from oracle import oracle as O


def _cfg_from(items):
    c = O.default_config()
    for k, v in items:
        setattr(c, k, v)
    return c


def test_oracle_matches_reference_golden(golden):
    for case, sysname, method, items in golden_cases(golden):
        A, b, fd = golden_system(golden, sysname)
        cfg = _cfg_from(items)
        if cfg.use_abmc and cfg.abmc_use_rcm:
            # Path 2 is not restated in C (RCM's order among rows of equal degree is
            # the reference's std::sort); those fixtures pin the GPU path directly
            with pytest.raises(RuntimeError):
                O.solve(A, b, method, cfg, freedofs=fd, which="port")
            continue
        x, res, hist = O.solve(A, b, method, cfg, freedofs=fd, which="port")
        conv, iters, fres = golden[f"case/{case}/meta"]
        xr = golden[f"case/{case}/x"]
        assert res.iterations == int(iters), case
        assert res.converged == int(conv), case
        scale = max(np.abs(xr).max(), 1e-300)
        assert np.abs(x - xr).max() / scale < 1e-12, case
        hr = golden[f"case/{case}/hist"]
        assert len(hist) == len(hr), case
        np.testing.assert_allclose(hist, hr, rtol=1e-6, atol=1e-9, err_msg=case)
        np.testing.assert_allclose(res.final_residual, fres, rtol=1e-6, atol=1e-14, err_msg=case)


@pytest.mark.parametrize("sysname", ["lap3d_6", "lap3d_8_fd", "lap2d_12", "cplx3d_6", "cplx3d_8_fd"])
def test_oracle_abmc_matches_reference(golden, sysname):
    A, _, _ = golden_system(golden, sysname)
    a = O.abmc(A, 4, 4, which="port")
    for k in ("color_offsets", "block_offsets", "ordering", "reverse"):
        np.testing.assert_array_equal(a[k], golden[f"abmc/{sysname}/{k}"], err_msg=k)
    assert a["num_colors"] == int(golden[f"abmc/{sysname}/num_colors"])


@pytest.mark.parametrize("sysname", ["lap3d_6", "lap3d_8_fd", "cplx3d_8_fd"])
def test_oracle_ic_mult_matches_reference(golden, sysname):
    A, b, fd = golden_system(golden, sysname)
    for kind, cfg in (("abmc", O.default_config(use_abmc=1)), ("level", O.default_config())):
        y, _ = O.ic_mult(A, b, cfg, freedofs=fd, which="port")
        yr = golden[f"icmult/{sysname}/{kind}"]
        assert np.abs(y - yr).max() <= 1e-13 * np.abs(yr).max()


def test_oracle_unknown_method_raises():
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(3)
    with pytest.raises(RuntimeError, match="Unknown method"):
        O.solve(A, np.ones(27), "INVALID")


def test_oracle_missing_diagonal_raises():
    import scipy.sparse as sp
    A = sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 2.0]]))
    A.eliminate_zeros()
    with pytest.raises(RuntimeError, match="missing diagonal"):
        O.solve(A, np.ones(2), "ICCG")


def test_oracle_live_reference_small():
    """Where the reference library is built here, compare live on a fresh case."""
    ref = O.reference()
    if ref is None:
        pytest.skip("reference library not built on this machine")
    from sparsesolv_ngsolve import problems as P
    ref.ref_set_threads(1)
    A = P.laplacian_7pt(10)
    b = P.random_rhs(A.shape[0], 11)
    cfg = O.default_config(use_abmc=1, save_residual_history=1, abmc_block_size=3, abmc_num_colors=5)
    x1, r1, h1 = O.solve(A, b, "ICCG", cfg, which="port")
    x2, r2, h2 = O.solve(A, b, "ICCG", cfg, which="ref")
    assert r1.iterations == r2.iterations
    assert np.abs(x1 - x2).max() < 1e-12 * np.abs(x2).max()


@pytest.mark.parametrize("sysname", ["lap3d_6", "lap3d_8_fd", "lap2d_12", "cplx3d_6", "cplx3d_8_fd"])
def test_oracle_sgs_mult_matches_reference(golden, sysname):
    """SGSPreconditioner apply: bit-exact on real systems, complex to rounding
    (C99 complex against std::complex arithmetic)."""
    A, b, fd = golden_system(golden, sysname)
    y = O.sgs_mult(A, b, freedofs=fd, which="port")
    yr = golden[f"sgsmult/{sysname}"]
    assert np.abs(y - yr).max() <= 1e-14 * np.abs(yr).max()
    if not np.iscomplexobj(yr):
        assert np.array_equal(y, yr)
