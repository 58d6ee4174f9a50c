"""ssv_spmv_dot_noalloc: the allocation-free SpMV + dot entry point.

Callers that must not allocate device memory (their framework owns the
device's memory pool, or they run under a fixed memory budget) pass every
buffer themselves; the entry point keeps its reduction scratch in a fixed
array inside the library. This file is collected last so that, if it fails,
a run that stops at the first failure has already run every other test; it
must pass both alone in a fresh process and after the other tests."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def test_noalloc_matches_existing_spmv_two_calls_in_a_row():
    import torch

    from sparsesolv_ngsolve import _Matrix, _capi
    from sparsesolv_ngsolve import problems as P
    lib = _capi.load()
    A = P.laplacian_7pt(23)  # 12,167 rows: not a multiple of 32 rows per CTA
    n = A.shape[0]
    m = _Matrix(A)  # existing entry point's matrix handle
    rp, ci, val = _dev(A.indptr.astype(np.int32)), _dev(A.indices.astype(np.int32)), _dev(A.data)
    rng = np.random.default_rng(0)
    for call in range(2):  # the scratch keeps the previous call's contents
        x = rng.uniform(-1, 1, n)
        dx = _dev(x)
        dy = torch.empty(n, dtype=torch.float64, device="cuda:0")
        dref = torch.empty(n, dtype=torch.float64, device="cuda:0")
        ddot = torch.full((1,), np.nan, dtype=torch.float64, device="cuda:0")
        rc = lib.ssv_spmv_dot_noalloc(n, ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(ci.data_ptr()),
                                      ctypes.c_void_p(val.data_ptr()), ctypes.c_void_p(dx.data_ptr()),
                                      ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(ddot.data_ptr()))
        assert rc == 0, lib.ssv_last_error()
        _capi.check(lib.ssv_matrix_spmv_dev(m.h, ctypes.c_void_p(dx.data_ptr()), ctypes.c_void_p(dref.data_ptr())))
        torch.cuda.synchronize()
        y = dy.cpu().numpy()
        yref = dref.cpu().numpy()
        ys = A @ x  # scipy, FP64 on the host
        np.testing.assert_allclose(y, yref, rtol=1e-14, atol=1e-14)
        np.testing.assert_allclose(y, ys, rtol=1e-13, atol=1e-13 * np.abs(ys).max())
        np.testing.assert_allclose(ddot.item(), float(x @ ys), rtol=1e-12)


def test_noalloc_rejects_too_many_rows():
    from sparsesolv_ngsolve import _capi
    lib = _capi.load()
    one = _dev(np.zeros(4, np.int32))
    v = _dev(np.zeros(4))
    p = ctypes.c_void_p(one.data_ptr())
    q = ctypes.c_void_p(v.data_ptr())
    rc = lib.ssv_spmv_dot_noalloc(2097152 + 1, p, p, q, q, q, q)
    assert rc == _capi.SSV_ERR_INVALID_ARG
    assert b"exceed the maximum of 2097152" in lib.ssv_last_error()


def test_noalloc_refuses_host_pointers():
    """A host array where device memory is required is refused before any
    launch (it would otherwise reach the kernel as an invalid address)."""
    from sparsesolv_ngsolve import _capi
    from sparsesolv_ngsolve import problems as P
    lib = _capi.load()
    A = P.laplacian_7pt(6)
    n = A.shape[0]
    rp, ci, val = _dev(A.indptr.astype(np.int32)), _dev(A.indices.astype(np.int32)), _dev(A.data)
    hx = np.ones(n)
    dy = _dev(np.zeros(n))
    ddot = _dev(np.zeros(1))
    rc = lib.ssv_spmv_dot_noalloc(n, ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(ci.data_ptr()),
                                  ctypes.c_void_p(val.data_ptr()), ctypes.c_void_p(hx.ctypes.data),
                                  ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(ddot.data_ptr()))
    assert rc == _capi.SSV_ERR_INVALID_ARG
    assert b"d_x is not device memory" in lib.ssv_last_error()
