"""ctypes front end of the oracle -- TEST INFRASTRUCTURE.

Loads ``oracle/_build/libssv_oracle.so`` (the C restatement, rebuilt with gcc
when missing) and, where present, ``oracle/_ref/libssv_ref.so`` (the
reference's own headers). Only tests/, the smoke check and bench.py's CPU
baseline use this module, to check results (test infrastructure).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "ngsolve-sparsesolv_b200"))

from sparsesolv_ngsolve import _capi  # noqa: E402  (struct layouts only)
from oracle import build_oracle  # noqa: E402

ssv_config = _capi.ssv_config
ssv_result = _capi.ssv_result
default_config = _capi.default_config

P = ctypes.c_void_p
I32 = ctypes.c_int32
PI32 = ctypes.POINTER(ctypes.c_int32)
PU8 = ctypes.POINTER(ctypes.c_uint8)
PD = ctypes.POINTER(ctypes.c_double)
PRECOND_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)

_libs = {}


def _bind(lib, prefix):
    sig = {
        "solve": (I32, [I32, PI32, PI32, P, I32, PU8, ctypes.c_char_p, ctypes.POINTER(ssv_config),
                        P, P, ctypes.POINTER(ssv_result), PD, I32]),
        "ic_mult": (I32, [I32, PI32, PI32, P, I32, PU8, ctypes.POINTER(ssv_config), P, P, PD]),
        "abmc_build": (I32, [I32, PI32, PI32, I32, I32, PI32, PI32, PI32, PI32, PI32, PI32]),
        "level_schedule": (I32, [I32, PI32, PI32, I32, PI32, PI32]),
        "sgs_mult": (I32, [I32, PI32, PI32, P, I32, PU8, P, P]),
        "last_error": (ctypes.c_char_p, []),
    }
    if prefix == "orc_":
        sig["cocr_solve"] = (I32, [I32, PI32, PI32, P, I32, PU8, PRECOND_FN, P, I32,
                                   ctypes.c_double, P, P, PI32])
        sig["spmv"] = (I32, [I32, PI32, PI32, P, I32, P, P])
    else:
        sig["set_threads"] = (None, [I32])
        sig["get_threads"] = (I32, [])
        sig["rcm"] = (I32, [I32, PI32, PI32, PI32, PI32])
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
    return lib


def port():
    """The C restatement (always available: built with gcc on demand)."""
    if "port" not in _libs:
        path = build_oracle.build_oracle()
        _libs["port"] = _bind(ctypes.CDLL(path), "orc_")
    return _libs["port"]


def reference():
    """The reference's own headers compiled here, or None if not built."""
    if "ref" not in _libs:
        path = build_oracle.REF_SO
        if not os.path.exists(path):
            path = build_oracle.build_reference()
        _libs["ref"] = _bind(ctypes.CDLL(path), "ref_") if path and os.path.exists(path) else None
    return _libs["ref"]


def _csr_parts(A):
    rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    cplx = np.iscomplexobj(A.data)
    v = np.ascontiguousarray(A.data, dtype=np.complex128 if cplx else np.float64)
    return rp, ci, v, (1 if cplx else 0)


def _p(a, t=PI32):
    return None if a is None else a.ctypes.data_as(t)


def solve(A, b, method="ICCG", config=None, freedofs=None, x0=None, which="port",
          history_cap=100000):
    """SparseSolvSolver::Solve on the CPU. Returns (x, result, history)."""
    lib = port() if which == "port" else reference()
    if lib is None:
        raise RuntimeError("reference library oracle/_ref/libssv_ref.so is not built")
    rp, ci, v, dt = _csr_parts(A)
    n = A.shape[0]
    vdt = np.complex128 if dt else np.float64
    bb = np.ascontiguousarray(b, dtype=vdt)
    x = np.zeros(n, dtype=vdt) if x0 is None else np.array(x0, dtype=vdt, copy=True)
    cfg = config if config is not None else default_config()
    fd = None if freedofs is None else np.ascontiguousarray(freedofs, dtype=np.uint8)
    res = ssv_result()
    hist = np.zeros(max(history_cap, 1))
    rc = getattr(lib, ("orc_" if which == "port" else "ref_") + "solve")(
        n, _p(rp), _p(ci), P(v.ctypes.data), dt, _p(fd, PU8), method.encode(),
        ctypes.byref(cfg), P(bb.ctypes.data), P(x.ctypes.data), ctypes.byref(res),
        _p(hist, PD), history_cap)
    if rc != 0:
        msg = getattr(lib, ("orc_" if which == "port" else "ref_") + "last_error")().decode()
        raise RuntimeError(msg)
    return x, res, hist[: res.history_len].copy()


def ic_mult(A, x, config=None, freedofs=None, which="port"):
    """ICPreconditioner(A) followed by one Mult: returns (y, actual_shift)."""
    lib = port() if which == "port" else reference()
    rp, ci, v, dt = _csr_parts(A)
    n = A.shape[0]
    vdt = np.complex128 if dt else np.float64
    xx = np.ascontiguousarray(x, dtype=vdt)
    y = np.zeros(n, dtype=vdt)
    cfg = config if config is not None else default_config()
    fd = None if freedofs is None else np.ascontiguousarray(freedofs, dtype=np.uint8)
    sh = ctypes.c_double(0.0)
    rc = getattr(lib, ("orc_" if which == "port" else "ref_") + "ic_mult")(
        n, _p(rp), _p(ci), P(v.ctypes.data), dt, _p(fd, PU8), ctypes.byref(cfg),
        P(xx.ctypes.data), P(y.ctypes.data), ctypes.byref(sh))
    if rc != 0:
        raise RuntimeError(getattr(lib, ("orc_" if which == "port" else "ref_") + "last_error")().decode())
    return y, sh.value


def sgs_mult(A, x, freedofs=None, which="port"):
    """SGSPreconditioner(A, freedofs) * x (factory, Update and Mult)."""
    lib = port() if which == "port" else reference()
    rp, ci, v, cplx = _csr_parts(A)
    dt = np.complex128 if cplx else np.float64
    xx = np.ascontiguousarray(x, dtype=dt)
    y = np.zeros(A.shape[0], dtype=dt)
    fd = None if freedofs is None else np.ascontiguousarray(freedofs, np.uint8)
    rc = getattr(lib, ("orc_" if which == "port" else "ref_") + "sgs_mult")(
        A.shape[0], _p(rp), _p(ci), v.ctypes.data_as(P), cplx, _p(fd, PU8), xx.ctypes.data_as(P),
        y.ctypes.data_as(P))
    if rc != 0:
        raise RuntimeError("sgs_mult failed")
    return y


def abmc(A, block_size=4, num_colors=4, which="port"):
    """ABMCSchedule::build: returns dict of the schedule arrays."""
    lib = port() if which == "port" else reference()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    n = A.shape[0]
    nc = ctypes.c_int32(0)
    nb = ctypes.c_int32(0)
    co = np.zeros(n + 1, np.int32)
    bo = np.zeros(n + 1, np.int32)
    od = np.zeros(n, np.int32)
    rv = np.zeros(n, np.int32)
    rc = getattr(lib, ("orc_" if which == "port" else "ref_") + "abmc_build")(
        n, _p(rp), _p(ci), block_size, num_colors, ctypes.byref(nc), ctypes.byref(nb),
        _p(co), _p(bo), _p(od), _p(rv))
    if rc != 0:
        raise RuntimeError("abmc build failed")
    return {"num_colors": nc.value, "num_blocks": nb.value,
            "color_offsets": co[: nc.value + 1].copy(), "block_offsets": bo[: nb.value + 1].copy(),
            "ordering": od, "reverse": rv}


def rcm(A, which="ref"):
    """compute_rcm_ordering (rcm_ordering.hpp:38-140) of A's pattern, run by the
    reference library (the C restatement has no RCM: its tie order among rows
    of equal degree is the reference's std::sort, not restated in C).
    Returns (ordering[old] = new, reverse[new] = old)."""
    if which != "ref":
        raise ValueError("rcm: only the reference library computes it")
    lib = reference()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    n = A.shape[0]
    od = np.zeros(max(n, 1), np.int32)
    rv = np.zeros(max(n, 1), np.int32)
    if lib.ref_rcm(n, _p(rp), _p(ci), _p(od), _p(rv)) != 0:
        raise RuntimeError("rcm failed")
    return od[:n], rv[:n]


def level_schedule(rp, ci, n, upper=False, which="port"):
    lib = port() if which == "port" else reference()
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    lev = np.zeros(max(n, 1), np.int32)
    nl = ctypes.c_int32(0)
    getattr(lib, ("orc_" if which == "port" else "ref_") + "level_schedule")(
        n, _p(rp), _p(ci), 1 if upper else 0, _p(lev), ctypes.byref(nl))
    return lev[:n], nl.value


class AmgOracle:
    """CPU restatement of CompactAMGPreconditioner (compact_amg.hpp:49-183)."""

    def __init__(self, A, freedofs=None, theta=0.25, max_levels=25, min_coarse=50, num_smooth=1):
        lib = AmsOracle.lib()
        D = ctypes.POINTER(ctypes.c_double)
        rp = np.ascontiguousarray(A.indptr, np.int32)
        ci = np.ascontiguousarray(A.indices, np.int32)
        v = np.ascontiguousarray(A.data, np.float64)
        fd = None if freedofs is None else np.ascontiguousarray(freedofs, np.uint8)
        self.n = A.shape[0]
        self.h = lib.ams_oracle_amg_create(self.n, _p(rp), _p(ci), v.ctypes.data_as(D), _p(fd, PU8), float(theta),
                                           int(max_levels), int(min_coarse), int(num_smooth))

    def apply(self, b):
        D = ctypes.POINTER(ctypes.c_double)
        bb = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n)
        AmsOracle.lib().ams_oracle_amg_apply(self.h, bb.ctypes.data_as(D), x.ctypes.data_as(D))
        return x

    def levels(self):
        buf = np.zeros(256, np.int32)
        nl = AmsOracle.lib().ams_oracle_amg_levels(self.h, _p(buf), 256)
        return [(int(buf[2 * l]), int(buf[2 * l + 1])) for l in range(nl)]

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            AmsOracle.lib().ams_oracle_amg_destroy(h)
            self.h = None


class AmsOracle:
    """CPU restatement of CompactAMS / ComplexCompactAMS (oracle/ams_oracle.cpp)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(build_oracle.build_ams_oracle())
            D = ctypes.POINTER(ctypes.c_double)
            lib.ams_oracle_create.restype = ctypes.c_void_p
            lib.ams_oracle_create.argtypes = [I32, PI32, PI32, D, I32, PI32, PI32, D, PU8, D, D, D, I32, I32,
                                              ctypes.c_double, ctypes.c_double]
            lib.ams_oracle_update.argtypes = [P, D]
            lib.ams_oracle_destroy.argtypes = [P]
            lib.ams_oracle_apply.argtypes = [P, D, D]
            lib.ams_oracle_apply_complex.argtypes = [P, D, D]
            lib.ams_oracle_levels.restype = I32
            lib.ams_oracle_levels.argtypes = [P, I32, PI32, I32]
            lib.ams_oracle_level_matrix.restype = I32
            lib.ams_oracle_level_matrix.argtypes = [P, I32, I32, I32, PI32, PI32, D, I32]
            lib.ams_oracle_pcg.restype = I32
            lib.ams_oracle_pcg.argtypes = [P, D, D, ctypes.POINTER(ssv_config), ctypes.POINTER(ssv_result), D, I32]
            lib.ams_oracle_cocr.restype = I32
            lib.ams_oracle_cocr.argtypes = [P, I32, PI32, PI32, D, PU8, I32, ctypes.c_double, D, D, PI32, D, I32,
                                            PI32]
            lib.ams_oracle_amg_create.restype = ctypes.c_void_p
            lib.ams_oracle_amg_create.argtypes = [I32, PI32, PI32, D, PU8, ctypes.c_double, I32, I32, I32]
            lib.ams_oracle_amg_apply.argtypes = [P, D, D]
            lib.ams_oracle_amg_levels.restype = I32
            lib.ams_oracle_amg_levels.argtypes = [P, PI32, I32]
            lib.ams_oracle_amg_destroy.argtypes = [P]
            lib.ams_oracle_set_threads.restype = None
            lib.ams_oracle_set_threads.argtypes = [I32]
            lib.ams_oracle_set_threads(1)
            cls._lib = lib
        return cls._lib

    @classmethod
    def set_threads(cls, n):
        """Host threads of the restatement's row-parallel loops (results do not depend on it)."""
        cls.lib().ams_oracle_set_threads(int(n))

    def __init__(self, A, G, freedofs, cx, cy, cz, cycle_type=1, num_smooth=1, theta=0.25, weight=1.0):
        lib = self.lib()
        D = ctypes.POINTER(ctypes.c_double)
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        self.A = A
        arp, aci, av = arr(A.indptr, np.int32), arr(A.indices, np.int32), arr(A.data, np.float64)
        grp, gci, gv = arr(G.indptr, np.int32), arr(G.indices, np.int32), arr(G.data, np.float64)
        self.fd = None if freedofs is None else arr(freedofs, np.uint8)
        cxs = [arr(c, np.float64) for c in (cx, cy, cz)]
        self.n = A.shape[0]
        self.h = lib.ams_oracle_create(self.n, _p(arp), _p(aci), av.ctypes.data_as(D), G.shape[1], _p(grp), _p(gci),
                                       gv.ctypes.data_as(D), _p(self.fd, PU8), *[c.ctypes.data_as(D) for c in cxs],
                                       cycle_type, num_smooth, theta, weight)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().ams_oracle_destroy(self.h)
            self.h = None

    def update(self, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.lib().ams_oracle_update(self.h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def apply(self, b):
        D = ctypes.POINTER(ctypes.c_double)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        self.lib().ams_oracle_apply(self.h, bb.ctypes.data_as(D), x.ctypes.data_as(D))
        return x

    def apply_complex(self, f):
        D = ctypes.POINTER(ctypes.c_double)
        ff = np.ascontiguousarray(f, dtype=np.complex128)
        u = np.zeros(self.n, dtype=np.complex128)
        self.lib().ams_oracle_apply_complex(self.h, ff.ctypes.data_as(D), u.ctypes.data_as(D))
        return u

    def levels(self, s):
        buf = np.zeros(256, np.int32)
        nl = self.lib().ams_oracle_levels(self.h, s, _p(buf), 256)
        return [(int(buf[2 * l]), int(buf[2 * l + 1])) for l in range(nl)]

    def level_matrix(self, s, l, what=0):
        import scipy.sparse as sp
        D = ctypes.POINTER(ctypes.c_double)
        nnz = self.lib().ams_oracle_level_matrix(self.h, s, l, what, None, None, None, 0)
        sizes = self.levels(s)
        n = sizes[l][0]
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(nnz, np.int32)
        v = np.zeros(nnz)
        self.lib().ams_oracle_level_matrix(self.h, s, l, what, _p(rp), _p(ci), v.ctypes.data_as(D), nnz)
        m = n if what == 0 else sizes[l + 1][0]
        return sp.csr_matrix((v, ci, rp), shape=(n, m))

    def pcg(self, b, x0=None, config=None, history_cap=100000):
        D = ctypes.POINTER(ctypes.c_double)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        cfg = config if config is not None else default_config()
        res = ssv_result()
        hist = np.zeros(max(history_cap, 1))
        self.lib().ams_oracle_pcg(self.h, bb.ctypes.data_as(D), x.ctypes.data_as(D), ctypes.byref(cfg),
                                  ctypes.byref(res), hist.ctypes.data_as(D), history_cap)
        return x, res, hist[: res.history_len].copy()

    def cocr(self, Ac, f, freedofs=None, maxiter=500, tol=1e-8, history_cap=100000):
        D = ctypes.POINTER(ctypes.c_double)
        rp = np.ascontiguousarray(Ac.indptr, np.int32)
        ci = np.ascontiguousarray(Ac.indices, np.int32)
        v = np.ascontiguousarray(Ac.data, np.complex128)
        ff = np.ascontiguousarray(f, np.complex128)
        fd = None if freedofs is None else np.ascontiguousarray(freedofs, np.uint8)
        x = np.zeros(Ac.shape[0], np.complex128)
        it = ctypes.c_int32(0)
        hl = ctypes.c_int32(0)
        hist = np.zeros(max(history_cap, 1))
        self.lib().ams_oracle_cocr(self.h, Ac.shape[0], _p(rp), _p(ci), v.ctypes.data_as(D), _p(fd, PU8), maxiter,
                                   tol, ff.ctypes.data_as(D), x.ctypes.data_as(D), ctypes.byref(it),
                                   hist.ctypes.data_as(D), history_cap, ctypes.byref(hl))
        return x, it.value, hist[: hl.value].copy()


def cocr_solve(A, b, precond=None, freedofs=None, maxiter=500, tol=1e-8):
    """COCRSolverNGS::Mult on the CPU; precond is a python callable y=f(x)."""
    lib = port()
    rp, ci, v, dt = _csr_parts(A)
    n = A.shape[0]
    vdt = np.complex128 if dt else np.float64
    bb = np.ascontiguousarray(b, dtype=vdt)
    x = np.zeros(n, dtype=vdt)
    fd = None if freedofs is None else np.ascontiguousarray(freedofs, dtype=np.uint8)
    it = ctypes.c_int32(0)
    cb = None
    if precond is not None:
        def _cb(ctx, xp, yp):
            xs = np.ctypeslib.as_array(ctypes.cast(xp, ctypes.POINTER(ctypes.c_double)),
                                       shape=(n * (2 if dt else 1),)).view(vdt)
            ys = np.ctypeslib.as_array(ctypes.cast(yp, ctypes.POINTER(ctypes.c_double)),
                                       shape=(n * (2 if dt else 1),)).view(vdt)
            ys[:] = precond(xs.copy())
        cb = PRECOND_FN(_cb)
    rc = lib.orc_cocr_solve(n, _p(rp), _p(ci), P(v.ctypes.data), dt, _p(fd, PU8),
                            cb if cb is not None else PRECOND_FN(), None, maxiter, tol,
                            P(bb.ctypes.data), P(x.ctypes.data), ctypes.byref(it))
    if rc != 0:
        raise RuntimeError("oracle cocr failed")
    return x, it.value


def refined_cocr(A, f, precond, freedofs=None, maxiter=500, tol=1e-10, restart_drop=1e-5):
    """FP64 defect correction around COCRSolverNGS::Mult
    (ngsolve/sparsesolv_solvers.hpp:273-369), the mixed-precision form's
    driver (new: the reference has no counterpart). Cycles of the COCR
    recurrence, each started from the true residual r = P(b - A x) of the
    current x (rt = M^{-1} r, p = rt, q = P A p, rho = rt^T q) and ended when
    its residual ||r|| has dropped to restart_drop times the residual it
    started from, or is <= tol ||P b||, or on a breakdown (|mu|, |rho| below
    1e-30 (||r_start|| / ||P b||)^2), or out of iterations; the solve ends
    when the true relative residual is <= tol. precond: y = M^{-1} x.
    Returns (x, iterations over all cycles, cycles, true relative residual).
    Plain numpy loops over whole vectors: for the small systems of the tests."""
    fd = None if freedofs is None else np.asarray(freedofs).astype(bool)

    def proj(v):
        if fd is not None:
            v[~fd] = 0
        return v

    n = A.shape[0]
    x = np.zeros(n, dtype=np.result_type(A.dtype, f.dtype))
    r = proj(np.array(f, dtype=x.dtype))
    nb = float(np.linalg.norm(r))
    if nb < 1e-30:
        return x, 0, 0, 0.0
    used, cycles, rs = 0, 0, nb
    tr = 1.0
    while True:
        thr = 1e-30 * (rs / nb) ** 2
        stop = restart_drop * rs
        rt = precond(r.copy())
        p = rt.copy()
        q = proj(A @ p)
        rho = rt @ q
        steps = 0
        while used + steps < maxiter:
            qt = precond(q.copy())
            mu = qt @ q
            if abs(mu) < thr:
                break
            alpha = rho / mu
            x += alpha * p
            r -= alpha * q
            rt -= alpha * qt
            steps += 1
            res = float(np.linalg.norm(r))
            if res / nb <= tol or res <= stop:
                break
            t = proj(A @ rt)
            rho_new = rt @ t
            if abs(rho) < thr:
                break
            beta = rho_new / rho
            rho = rho_new
            p = rt + beta * p
            q = t + beta * q
        used += steps
        cycles += 1
        r = proj(np.array(f, dtype=x.dtype) - A @ x)
        rs = float(np.linalg.norm(r))
        tr = rs / nb
        if tr <= tol or used >= maxiter or steps == 0 or rs < 1e-300:
            return x, used, cycles, tr
