"""C ABI: the library loads, exports every declared symbol, and its host-side
set-up logic (ABMC ordering, level schedules) equals the reference's."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_system

HEADER = os.path.join(ROOT, "include", "sparsesolv_b200.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ssv_[a-z0-9_]+)\s*\(", txt)))


def _lib():
    from sparsesolv_ngsolve import _capi
    return _capi.load()


def test_library_exports_every_declared_symbol():
    lib = _lib()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/sparsesolv_b200.h but not exported"


def test_python_binding_covers_header():
    from sparsesolv_ngsolve import _capi
    bound = {n for n, _, _ in _capi.SIGNATURES}
    assert set(_declared()) <= bound


def _abmc(lib, A, bs, nc):
    n = A.shape[0]
    rp = np.ascontiguousarray(A.indptr, np.int32)
    ci = np.ascontiguousarray(A.indices, np.int32)
    out = [np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)]
    ncol, nblk = ctypes.c_int32(), ctypes.c_int32()
    P = ctypes.POINTER(ctypes.c_int32)
    rc = lib.ssv_abmc_build(n, rp.ctypes.data_as(P), ci.ctypes.data_as(P), bs, nc, ctypes.byref(ncol),
                            ctypes.byref(nblk), *[o.ctypes.data_as(P) for o in out])
    assert rc == 0
    return {"num_colors": ncol.value, "color_offsets": out[0][: ncol.value + 1],
            "block_offsets": out[1][: nblk.value + 1], "ordering": out[2], "reverse": out[3]}


@pytest.mark.parametrize("sysname", ["lap3d_6", "lap3d_8_fd", "lap2d_12", "cplx3d_6"])
def test_abmc_host_equals_reference(golden, sysname):
    A, _, _ = golden_system(golden, sysname)
    a = _abmc(_lib(), A, 4, 4)
    assert a["num_colors"] == int(golden[f"abmc/{sysname}/num_colors"])
    for k in ("color_offsets", "block_offsets", "ordering", "reverse"):
        np.testing.assert_array_equal(a[k], golden[f"abmc/{sysname}/{k}"], err_msg=k)


@pytest.mark.parametrize("nx,bs,nc", [(12, 4, 4), (10, 2, 3), (9, 8, 2), (7, 1, 2), (11, 16, 6)])
def test_abmc_host_equals_oracle_various(nx, bs, nc):
    from oracle import oracle as O
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(nx)
    a = _abmc(_lib(), A, bs, nc)
    o = O.abmc(A, bs, nc, which="port")
    assert a["num_colors"] == o["num_colors"]
    for k in ("color_offsets", "block_offsets", "ordering", "reverse"):
        np.testing.assert_array_equal(a[k], o[k], err_msg=k)


def test_abmc_config1_colours():
    """64^3 7-point Laplacian: 4 target colours become 9 (as the reference does)."""
    from oracle import oracle as O
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(64)
    a = _abmc(_lib(), A, 4, 4)
    o = O.abmc(A, 4, 4, which="port")
    assert a["num_colors"] == o["num_colors"] == 9
    np.testing.assert_array_equal(a["ordering"], o["ordering"])


@pytest.mark.parametrize("sysname", ["lap3d_6", "lap2d_12"])
def test_level_schedule_equals_reference(golden, sysname):
    import scipy.sparse as sp
    A, _, _ = golden_system(golden, sysname)
    L = sp.tril(A, format="csr")
    L.sort_indices()
    n = A.shape[0]
    lev = np.zeros(n, np.int32)
    nl = ctypes.c_int32()
    P = ctypes.POINTER(ctypes.c_int32)
    rp = np.ascontiguousarray(L.indptr, np.int32)
    ci = np.ascontiguousarray(L.indices, np.int32)
    assert _lib().ssv_level_schedule(n, rp.ctypes.data_as(P), ci.ctypes.data_as(P), 0, lev.ctypes.data_as(P),
                                     ctypes.byref(nl)) == 0
    np.testing.assert_array_equal(lev, golden[f"levels/{sysname}/lower"])


def test_no_device_fails_loudly():
    """Without a CUDA device the library refuses to work (no CPU fallback)."""
    from sparsesolv_ngsolve import _capi
    lib = _lib()
    cnt = ctypes.c_int32(-1)
    name = ctypes.create_string_buffer(128)
    assert lib.ssv_device_info(ctypes.byref(cnt), name, 128) == 0
    if cnt.value > 0:
        pytest.skip("a CUDA device is present")
    rp = np.array([0, 1], np.int32)
    ci = np.array([0], np.int32)
    v = np.array([2.0])
    h = ctypes.c_void_p()
    P = ctypes.POINTER(ctypes.c_int32)
    rc = lib.ssv_matrix_create(1, 1, rp.ctypes.data_as(P), ci.ctypes.data_as(P), ctypes.c_void_p(v.ctypes.data),
                               0, ctypes.byref(h))
    assert rc == _capi.SSV_ERR_NO_DEVICE
    assert b"no CUDA device" in lib.ssv_last_error()


def test_config_default_matches_reference_defaults():
    from sparsesolv_ngsolve import _capi
    c = _capi.ssv_config()
    _lib().ssv_config_default(ctypes.byref(c))
    d = _capi.default_config()
    for f, _ in _capi.ssv_config._fields_:
        assert getattr(c, f) == getattr(d, f), f
    assert c.tolerance == 1e-10 and c.max_iterations == 1000 and c.abs_tolerance == 1e-12
    assert c.divergence_threshold == 1000.0 and c.divergence_count == 100 and c.save_best_result == 1


def _rcm(lib, rp, ci, n):
    P = ctypes.POINTER(ctypes.c_int32)
    rp = np.ascontiguousarray(rp, np.int32)
    ci = np.ascontiguousarray(ci, np.int32)
    od = np.zeros(max(n, 1), np.int32)
    rv = np.zeros(max(n, 1), np.int32)
    assert lib.ssv_rcm_order(n, rp.ctypes.data_as(P), ci.ctypes.data_as(P), od.ctypes.data_as(P),
                             rv.ctypes.data_as(P)) == 0
    return od[:n], rv[:n]


@pytest.mark.parametrize("sysname", ["lap3d_6", "lap3d_8_fd", "lap2d_12", "cplx3d_6", "cplx3d_8_fd"])
def test_rcm_host_equals_reference(golden, sysname):
    """The abmc_use_rcm pre-ordering is bit-identical to compute_rcm_ordering."""
    A, _, _ = golden_system(golden, sysname)
    od, rv = _rcm(_lib(), A.indptr, A.indices, A.shape[0])
    np.testing.assert_array_equal(od, golden[f"rcm/{sysname}/ordering"])
    np.testing.assert_array_equal(rv, golden[f"rcm/{sysname}/reverse"])


def test_rcm_permutation_and_edge_shapes():
    import scipy.sparse as sp
    lib = _lib()
    # disconnected pattern (two blocks and an isolated row), ragged degrees
    A = sp.block_diag([sp.random(9, 9, 0.4, random_state=1) + sp.eye(9), sp.eye(1),
                       sp.random(6, 6, 0.5, random_state=2) + sp.eye(6)]).tocsr()
    A = (A + A.T).tocsr()
    A.sort_indices()
    od, rv = _rcm(lib, A.indptr, A.indices, A.shape[0])
    assert sorted(od.tolist()) == list(range(A.shape[0]))
    assert (rv[od] == np.arange(A.shape[0])).all()
    from oracle import oracle as O
    if O.reference() is not None:
        ro, rr = O.rcm(A)
        np.testing.assert_array_equal(od, ro)
        np.testing.assert_array_equal(rv, rr)
    # empty and single-row patterns
    assert _rcm(lib, np.zeros(1, np.int32), np.zeros(0, np.int32), 0)[0].size == 0
    od1, rv1 = _rcm(lib, np.array([0, 1], np.int32), np.array([0], np.int32), 1)
    assert od1.tolist() == [0] and rv1.tolist() == [0]


def test_hcurl_assemble_validates_inputs_before_the_device():
    """ssv_hcurl_assemble checks its mesh arrays on the host first: out-of-range
    ids, signs other than +-1 and edges not listed low -> high are refused with
    SSV_ERR_INVALID_ARG (on a machine without a device too); a valid mesh then
    reaches the device check."""
    from sparsesolv_ngsolve import _capi
    from sparsesolv_ngsolve import hcurl as H
    lib = _lib()
    m = H.kuhn_mesh(2)
    xyz = np.ascontiguousarray(m.coords, dtype=np.float64)
    tets = np.ascontiguousarray(m.tets, dtype=np.int32)
    te = np.ascontiguousarray(m.tet_edges, dtype=np.int32)
    sg = np.ascontiguousarray(m.tet_signs, dtype=np.int8)
    ev = np.ascontiguousarray(m.edges, dtype=np.int32)

    def call(tets=tets, te=te, sg=sg, ev=ev):
        hs = [ctypes.c_void_p() for _ in range(3)]
        rc = lib.ssv_hcurl_assemble(m.nv, _capi.vptr(xyz), tets.shape[0], _capi.vptr(tets), _capi.vptr(te),
                                    _capi.vptr(sg), m.ne, _capi.vptr(ev), None, None, ctypes.byref(hs[0]),
                                    ctypes.byref(hs[1]), ctypes.byref(hs[2]))
        for h in hs:
            if h.value:
                lib.ssv_matrix_destroy(h)
        return rc

    bad = tets.copy()
    bad[0, 0] = m.nv
    assert call(tets=bad) == _capi.SSV_ERR_INVALID_ARG
    bad = te.copy()
    bad[1, 2] = -1
    assert call(te=bad) == _capi.SSV_ERR_INVALID_ARG
    bad = sg.copy()
    bad[0, 0] = 0
    assert call(sg=bad) == _capi.SSV_ERR_INVALID_ARG
    bad = ev.copy()
    bad[3] = bad[3][::-1]
    assert call(ev=bad) == _capi.SSV_ERR_INVALID_ARG
    cnt = ctypes.c_int32(-1)
    name = ctypes.create_string_buffer(128)
    assert lib.ssv_device_info(ctypes.byref(cnt), name, 128) == 0
    if cnt.value == 0:
        assert call() == _capi.SSV_ERR_NO_DEVICE
