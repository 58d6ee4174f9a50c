"""sparsesolv_ngsolve -- the reference's Python API on the B200 solve path.

Same factories, keyword arguments, defaults, typed classes and error types as
ksugahar/ngsolve-sparsesolv's pybind11 module
(include/sparsesolv/ngsolve/sparsesolv_python_export.hpp), backed by the
sm_100a kernels of ``libsparsesolv_b200.so`` through its C ABI. There is no
CPU path: without a CUDA device every solve raises.

Matrices: a ``scipy.sparse`` matrix, or any object with NGSolve's
``SparseMatrix.CSR()`` (returning ``(values, col_indices, row_ptr)``).
Vectors: numpy arrays, or NGSolve vectors (``.FV().NumPy()``).
FreeDofs: a boolean/uint8 array, or an NGSolve ``BitArray``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import check

__all__ = [
    "SparseSolvResult", "SparseSolvSolver", "SparseSolvSolverD", "SparseSolvSolverC",
    "ICPreconditioner", "ICPreconditionerD", "ICPreconditionerC",
    "COCRSolver", "COCRSolverD", "COCRSolverC", "has_compact_ams",
    "MixedCOCRSolver", "MixedCOCRSolverD", "MixedCOCRSolverC",
    "CompactAMSPreconditioner", "CompactAMSPreconditionerImpl",
    "ComplexCompactAMSPreconditioner", "ComplexCompactAMSPreconditionerImpl", "PCGSolver",
    "BatchedCOCRSolver", "SGSPreconditioner", "SGSPreconditionerD", "SGSPreconditionerC",
    "GMRESSolver", "GMRESSolverD", "GMRESSolverC", "CompactAMGPreconditioner", "CompactAMGPreconditionerImpl",
]


# ---------------------------------------------------------------------------
# input adapters
# ---------------------------------------------------------------------------

def _csr_arrays(mat):
    """(indptr int32, indices int32, data, is_complex) of a sparse matrix."""
    if hasattr(mat, "tocsr") and hasattr(mat, "indptr") or hasattr(mat, "tocsr"):
        A = mat.tocsr()
        if not A.has_sorted_indices:
            A = A.sorted_indices()
        ip = np.ascontiguousarray(A.indptr, dtype=np.int32)
        ix = np.ascontiguousarray(A.indices, dtype=np.int32)
        data = A.data
        shape = A.shape
    elif hasattr(mat, "CSR"):  # NGSolve SparseMatrix
        vals, cols, rows = mat.CSR()
        data = np.asarray(vals)
        ix = np.ascontiguousarray(np.asarray(cols), dtype=np.int32)
        ip = np.ascontiguousarray(np.asarray(rows), dtype=np.int32)
        shape = (mat.height, mat.width)
    else:
        raise TypeError("expected SparseMatrix (scipy.sparse or NGSolve SparseMatrix)")
    cplx = np.iscomplexobj(data)
    data = np.ascontiguousarray(data, dtype=np.complex128 if cplx else np.float64)
    return ip, ix, data, cplx, shape


def _freedofs_array(freedofs, n):
    if freedofs is None:
        return None
    if hasattr(freedofs, "__len__") and not isinstance(freedofs, np.ndarray) and hasattr(freedofs, "__getitem__") \
            and not isinstance(freedofs, (list, tuple)):
        fd = np.fromiter((1 if freedofs[i] else 0 for i in range(len(freedofs))), dtype=np.uint8, count=len(freedofs))
    else:
        fd = np.asarray(freedofs).astype(bool).astype(np.uint8)
    if fd.shape[0] != n:
        raise ValueError(f"freedofs has {fd.shape[0]} entries, matrix has {n} rows")
    return np.ascontiguousarray(fd)


def _note_applies(pre, count):
    """Tells a preconditioner how many times a solve applied it (print_level diagnostics)."""
    f = getattr(pre, "_note_applies", None)
    if f is not None and count > 0:
        f(int(count))


def _vec_view(v):
    """Writable numpy view of a vector (numpy array or NGSolve BaseVector)."""
    if isinstance(v, np.ndarray):
        return v
    if hasattr(v, "FV"):
        return v.FV().NumPy()
    return np.asarray(v)


class _Matrix:
    """Device copy of a CSR matrix (ssv_matrix handle)."""

    def __init__(self, mat):
        self.src = mat
        ip, ix, data, cplx, shape = _csr_arrays(mat)
        self.n, self.m = int(shape[0]), int(shape[1])
        self.cplx = bool(cplx)
        self.dtype = np.complex128 if cplx else np.float64
        self.nnz = int(ip[-1])
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.ssv_matrix_create(self.n, self.m, _capi.i32ptr(ip), _capi.i32ptr(ix), _capi.vptr(data),
                                    _capi.SSV_C128 if cplx else _capi.SSV_F64, ctypes.byref(h)))
        self.h = h
        self._lib = lib

    def refresh(self):
        """Re-read the source matrix values (the matrix may be modified in place)."""
        _, _, data, cplx, _ = _csr_arrays(self.src)
        if bool(cplx) != self.cplx or data.shape[0] != self.nnz:
            raise ValueError("matrix pattern or scalar type changed; create a new object")
        check(self._lib.ssv_matrix_update_values(self.h, _capi.vptr(data)))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                self._lib.ssv_matrix_destroy(h)
            except Exception:
                pass
            self.h = None


# ---------------------------------------------------------------------------
# SparseSolvResult (sparsesolv_python_export.hpp:32-49)
# ---------------------------------------------------------------------------

class SparseSolvResult:
    """Result of a SparseSolv iterative solve (converged, iterations, final_residual, residual_history)."""

    __slots__ = ("converged", "iterations", "final_residual", "residual_history",
                 "actual_shift", "setup_seconds", "solve_seconds", "kernel_launches")

    def __init__(self, converged=False, iterations=0, final_residual=0.0, residual_history=(),
                 actual_shift=0.0, setup_seconds=0.0, solve_seconds=0.0, kernel_launches=0):
        self.converged = bool(converged)
        self.iterations = int(iterations)
        self.final_residual = float(final_residual)
        self.residual_history = list(residual_history)
        self.actual_shift = actual_shift
        self.setup_seconds = setup_seconds
        self.solve_seconds = solve_seconds
        self.kernel_launches = int(kernel_launches)

    def __repr__(self):
        return (f"SparseSolvResult(converged={'True' if self.converged else 'False'}, "
                f"iterations={self.iterations}, residual={self.final_residual:f})")


# ---------------------------------------------------------------------------
# SparseSolvSolver (ngsolve/sparsesolv_solvers.hpp:33-239)
# ---------------------------------------------------------------------------

class _SparseSolvSolverBase:
    _cplx = False

    def __init__(self, mat, method="ICCG", freedofs=None, tol=1e-10, maxiter=1000, shift=1.05,
                 save_best_result=True, save_residual_history=False, printrates=False):
        self._mat = _Matrix(mat)
        self._fd = _freedofs_array(freedofs, self._mat.n)
        self.method = method
        self._cfg = _capi.default_config(tolerance=tol, max_iterations=maxiter, shift_parameter=shift,
                                         save_best_result=save_best_result,
                                         save_residual_history=save_residual_history)
        self.printrates = bool(printrates)
        self._last = SparseSolvResult()
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.ssv_solver_create(self._mat.h, _capi.u8ptr(self._fd), ctypes.byref(h)))
        self._h = h
        self._lib = lib

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.ssv_solver_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- solve ----------------------------------------------------------------
    def Solve(self, rhs, sol):
        """Solve A x = b with sol as the initial guess; returns SparseSolvResult."""
        b = np.ascontiguousarray(_vec_view(rhs), dtype=self._mat.dtype)
        xv = _vec_view(sol)
        x = np.ascontiguousarray(xv, dtype=self._mat.dtype)
        if b.shape[0] != self._mat.n or x.shape[0] != self._mat.n:
            raise ValueError("vector size does not match the matrix")
        self._mat.refresh()
        cfg = _capi.ssv_config()
        ctypes.pointer(cfg)[0] = self._cfg
        if self.printrates:
            cfg.save_residual_history = 1
        cap = max(int(cfg.max_iterations), 0) + 2 if cfg.save_residual_history else 0
        hist = np.zeros(max(cap, 1))
        res = _capi.ssv_result()
        check(self._lib.ssv_solver_solve(self._h, str(self.method).encode(), ctypes.byref(cfg),
                                         _capi.vptr(b), _capi.vptr(x), ctypes.byref(res),
                                         hist.ctypes.data_as(_capi.PD), cap))
        if x is not xv:
            xv[...] = x
        r = SparseSolvResult(res.converged, res.iterations, res.final_residual,
                             hist[: res.history_len].tolist() if cfg.save_residual_history else [],
                             res.actual_shift, res.setup_seconds, res.solve_seconds, res.kernel_launches)
        if self.printrates and r.residual_history:
            for i, v in enumerate(r.residual_history):
                print(f"{self.method} iteration {i}, residual = {v}")
            state = "converged in" if r.converged else "NOT converged after"
            print(f"{self.method} {state} {r.iterations} iterations, residual = {r.final_residual}")
        self._last = r
        return r

    def Mult(self, x, y):
        """y = A^{-1} x with zero initial guess (BaseMatrix::Mult)."""
        yv = _vec_view(y)
        yv[...] = 0
        self.Solve(x, yv)

    def __mul__(self, vec):
        y = np.zeros(self._mat.n, dtype=self._mat.dtype)
        self.Mult(vec, y)
        return y

    def MultAdd(self, s, x, y):
        t = self * x
        yv = _vec_view(y)
        yv += s * t

    @property
    def height(self):
        return self._mat.n

    @property
    def width(self):
        return self._mat.m

    def IsComplex(self):
        return self._cplx

    @property
    def last_result(self):
        return self._last

    # -- properties (sparsesolv_python_export.hpp:101-156) ---------------------
    def _get(self, f):
        return getattr(self._cfg, f)

    def _set(self, f, v):
        setattr(self._cfg, f, v)

    tol = property(lambda s: s._cfg.tolerance, lambda s, v: s._set("tolerance", float(v)))
    maxiter = property(lambda s: s._cfg.max_iterations, lambda s, v: s._set("max_iterations", int(v)))
    shift = property(lambda s: s._cfg.shift_parameter, lambda s, v: s._set("shift_parameter", float(v)))
    save_best_result = property(lambda s: bool(s._cfg.save_best_result),
                                lambda s, v: s._set("save_best_result", int(bool(v))))
    save_residual_history = property(lambda s: bool(s._cfg.save_residual_history),
                                     lambda s, v: s._set("save_residual_history", int(bool(v))))
    auto_shift = property(lambda s: bool(s._cfg.auto_shift), lambda s, v: s._set("auto_shift", int(bool(v))))
    diagonal_scaling = property(lambda s: bool(s._cfg.diagonal_scaling),
                                lambda s, v: s._set("diagonal_scaling", int(bool(v))))
    divergence_check = property(lambda s: bool(s._cfg.divergence_check),
                                lambda s, v: s._set("divergence_check", int(bool(v))))
    divergence_threshold = property(lambda s: s._cfg.divergence_threshold,
                                    lambda s, v: s._set("divergence_threshold", float(v)))
    divergence_count = property(lambda s: s._cfg.divergence_count,
                                lambda s, v: s._set("divergence_count", int(v)))
    conjugate = property(lambda s: bool(s._cfg.conjugate), lambda s, v: s._set("conjugate", int(bool(v))))
    use_abmc = property(lambda s: bool(s._cfg.use_abmc), lambda s, v: s._set("use_abmc", int(bool(v))))
    abmc_block_size = property(lambda s: s._cfg.abmc_block_size, lambda s, v: s._set("abmc_block_size", int(v)))
    abmc_num_colors = property(lambda s: s._cfg.abmc_num_colors, lambda s, v: s._set("abmc_num_colors", int(v)))
    abmc_reorder_spmv = property(lambda s: bool(s._cfg.abmc_reorder_spmv),
                                 lambda s, v: s._set("abmc_reorder_spmv", int(bool(v))))
    abmc_use_rcm = property(lambda s: bool(s._cfg.abmc_use_rcm),
                            lambda s, v: s._set("abmc_use_rcm", int(bool(v))))
    # new knob: FP32 storage of the preconditioner ("fp64" | "fp32")
    precision = property(lambda s: "fp32" if s._cfg.precision == _capi.SSV_PREC_FP32 else "fp64",
                         lambda s, v: s._set("precision", _capi.SSV_PREC_FP32 if str(v).lower() == "fp32"
                                             else _capi.SSV_PREC_FP64))


class SparseSolvSolverD(_SparseSolvSolverBase):
    _cplx = False


class SparseSolvSolverC(_SparseSolvSolverBase):
    _cplx = True


def SparseSolvSolver(mat, method="ICCG", freedofs=None, tol=1e-10, maxiter=1000, shift=1.05,
                     save_best_result=True, save_residual_history=False, printrates=False, conjugate=False,
                     use_abmc=False, abmc_block_size=4, abmc_num_colors=4, abmc_reorder_spmv=False,
                     abmc_use_rcm=False):
    """Iterative solver (ICCG / SGSMRTR / CG / COCR). Auto-detects real/complex.

    Factory of sparsesolv_python_export.hpp:242-294 (same arguments and
    defaults); returns SparseSolvSolverD or SparseSolvSolverC.
    """
    ip, ix, data, cplx, shape = _csr_arrays(mat)
    cls = SparseSolvSolverC if cplx else SparseSolvSolverD
    s = cls(mat, method, freedofs, tol, maxiter, shift, save_best_result, save_residual_history, printrates)
    s.conjugate = conjugate
    s.use_abmc = use_abmc
    s.abmc_block_size = abmc_block_size
    s.abmc_num_colors = abmc_num_colors
    s.abmc_reorder_spmv = abmc_reorder_spmv
    s.abmc_use_rcm = abmc_use_rcm
    return s


# ---------------------------------------------------------------------------
# ICPreconditioner (ngsolve/sparsesolv_precond.hpp:177-224)
# ---------------------------------------------------------------------------

class _PrecondBase:
    """Common part of the preconditioner handles (BaseMatrix-like)."""

    _cplx = False

    def _init_handle(self, h):
        self._h = h
        self._lib = _capi.load()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.ssv_precond_destroy(h)
            except Exception:
                pass
            self._h = None

    def Mult(self, x, y):
        xv = np.ascontiguousarray(_vec_view(x), dtype=self._dtype)
        yv = _vec_view(y)
        out = np.empty(self._n, dtype=self._dtype)
        check(self._lib.ssv_precond_apply(self._h, _capi.vptr(xv), _capi.vptr(out)))
        yv[...] = out

    def MultTrans(self, x, y):
        self.Mult(x, y)

    def MultAdd(self, s, x, y):
        t = self * x
        yv = _vec_view(y)
        if self._fd is not None:
            yv += s * np.where(self._fd.astype(bool), t, 0)
        else:
            yv += s * t

    def __mul__(self, vec):
        y = np.zeros(self._n, dtype=self._dtype)
        self.Mult(vec, y)
        return y

    @property
    def height(self):
        return self._n

    @property
    def width(self):
        return self._n

    def IsComplex(self):
        return self._cplx


class _ICPreconditionerBase(_PrecondBase):
    def __init__(self, mat, freedofs=None, shift=1.05):
        self._mat = _Matrix(mat)
        self._n = self._mat.n
        self._dtype = self._mat.dtype
        self._fd = _freedofs_array(freedofs, self._n)
        self._shift = float(shift)
        self._cfg = _capi.default_config(shift_parameter=self._shift)
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.ssv_ic_create(self._mat.h, _capi.u8ptr(self._fd), self._shift, ctypes.byref(h)))
        self._init_handle(h)

    def _sync(self):
        self._cfg.shift_parameter = self._shift
        check(self._lib.ssv_ic_set_config(self._h, ctypes.byref(self._cfg)))

    def Update(self):
        """Re-read the matrix and refactorise (SparseSolvICPreconditioner::Update)."""
        self._mat.refresh()
        self._sync()
        check(self._lib.ssv_precond_update(self._h))

    @property
    def shift(self):
        return self._shift

    @shift.setter
    def shift(self, v):
        self._shift = float(v)
        self._sync()

    use_abmc = property(lambda s: bool(s._cfg.use_abmc),
                        lambda s, v: (setattr(s._cfg, "use_abmc", int(bool(v))), s._sync()))
    abmc_block_size = property(lambda s: s._cfg.abmc_block_size,
                               lambda s, v: (setattr(s._cfg, "abmc_block_size", int(v)), s._sync()))
    abmc_num_colors = property(lambda s: s._cfg.abmc_num_colors,
                               lambda s, v: (setattr(s._cfg, "abmc_num_colors", int(v)), s._sync()))
    diagonal_scaling = property(lambda s: bool(s._cfg.diagonal_scaling),
                                lambda s, v: (setattr(s._cfg, "diagonal_scaling", int(bool(v))), s._sync()))
    precision = property(lambda s: "fp32" if s._cfg.precision == _capi.SSV_PREC_FP32 else "fp64",
                         lambda s, v: (setattr(s._cfg, "precision", _capi.SSV_PREC_FP32
                                               if str(v).lower() == "fp32" else _capi.SSV_PREC_FP64), s._sync()))

    @property
    def actual_shift(self):
        v = ctypes.c_double()
        check(self._lib.ssv_ic_actual_shift(self._h, ctypes.byref(v)))
        return v.value


class ICPreconditionerD(_ICPreconditionerBase):
    _cplx = False


class ICPreconditionerC(_ICPreconditionerBase):
    _cplx = True


def ICPreconditioner(mat, freedofs=None, shift=1.05):
    """Incomplete Cholesky (IC) preconditioner; calls Update() (factory :176-207)."""
    _, _, _, cplx, _ = _csr_arrays(mat)
    p = (ICPreconditionerC if cplx else ICPreconditionerD)(mat, freedofs, shift)
    p.Update()
    return p


# ---------------------------------------------------------------------------
# SGSPreconditioner (sparsesolv_python_export.hpp:82-89,209-240)
# ---------------------------------------------------------------------------

class _SGSPreconditionerBase(_PrecondBase):
    def __init__(self, mat, freedofs=None):
        self._mat = _Matrix(mat)
        self._n = self._mat.n
        self._dtype = self._mat.dtype
        self._fd = _freedofs_array(freedofs, self._n)
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.ssv_sgs_create(self._mat.h, _capi.u8ptr(self._fd), ctypes.byref(h)))
        self._init_handle(h)

    def Update(self):
        """Re-read the matrix (FreeDofs view) and rebuild 1/a_ii
        (SparseSolvSGSPreconditioner::Update)."""
        self._mat.refresh()
        check(self._lib.ssv_precond_update(self._h))


class SGSPreconditionerD(_SGSPreconditionerBase):
    _cplx = False


class SGSPreconditionerC(_SGSPreconditionerBase):
    _cplx = True


def SGSPreconditioner(mat, freedofs=None):
    """Symmetric Gauss-Seidel preconditioner (D+U)^{-1} D (D+L)^{-1}; calls Update() (factory :209-230)."""
    _, _, _, cplx, _ = _csr_arrays(mat)
    p = (SGSPreconditionerC if cplx else SGSPreconditionerD)(mat, freedofs)
    p.Update()
    return p


# ---------------------------------------------------------------------------
# CompactAMGPreconditioner (sparsesolv_python_export.hpp:339-404)
# ---------------------------------------------------------------------------

class CompactAMGPreconditionerImpl(_PrecondBase):
    """CompactAMG (compact_amg.hpp:49-183): V-cycle preconditioner of a real H1 matrix."""

    _cplx = False

    def __init__(self, mat, freedofs=None, theta=0.25, max_levels=25, min_coarse=50, num_smooth=1,
                 print_level=0):
        self._mat = mat if isinstance(mat, _Matrix) else _Matrix(mat)
        if self._mat.cplx:
            raise TypeError("CompactAMGPreconditioner: expected real SparseMatrix<double>")
        self._n = self._mat.n
        self._dtype = np.float64
        self._fd = _freedofs_array(freedofs, self._n)
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.ssv_amg_create(self._mat.h, _capi.u8ptr(self._fd), float(theta), int(max_levels),
                                 int(min_coarse), int(num_smooth), ctypes.byref(h)))
        self._init_handle(h)
        if print_level > 0:
            lv = self.levels()
            print(f"  CompactAMG: {len(lv)} levels, coarsest = {lv[-1][0]} DOFs")

    def levels(self):
        """[(rows, nnz), ...] of the AMG hierarchy."""
        buf = np.zeros(256, np.int32)
        nl = ctypes.c_int32()
        check(self._lib.ssv_amg_levels(self._h, _capi.i32ptr(buf), 256, ctypes.byref(nl)))
        return [(int(buf[2 * l]), int(buf[2 * l + 1])) for l in range(nl.value)]


def CompactAMGPreconditioner(mat, freedofs=None, theta=0.25, max_levels=25, min_coarse=50, num_smooth=1,
                             print_level=0):
    """Compact algebraic multigrid (PMIS, direct interpolation, l1-Jacobi) for scalar H1 problems."""
    return CompactAMGPreconditionerImpl(mat, freedofs, theta, max_levels, min_coarse, num_smooth, print_level)


# ---------------------------------------------------------------------------
# COCRSolver (ngsolve/sparsesolv_solvers.hpp:255-396)
# ---------------------------------------------------------------------------

class _COCRSolverBase:
    _cplx = False

    def __init__(self, mat, pre, freedofs=None, maxiter=500, tol=1e-8, printrates=False):
        self._mat = mat if isinstance(mat, _Matrix) else _Matrix(mat)
        self._pre = pre
        self._fd = _freedofs_array(freedofs, self._mat.n)
        self.maxiter = int(maxiter)
        self.tol = float(tol)
        self.printrates = bool(printrates)
        self._iterations = 0
        self._lib = _capi.load()

    @property
    def iterations(self):
        return self._iterations

    def Mult(self, rhs, sol):
        b = np.ascontiguousarray(_vec_view(rhs), dtype=self._mat.dtype)
        sv = _vec_view(sol)
        x = np.zeros(self._mat.n, dtype=self._mat.dtype)
        it = ctypes.c_int32(0)
        pre_h = None
        if self._pre is not None:
            pre_h = self._pre._h
        self._mat.refresh()
        check(self._lib.ssv_cocr_solve(self._mat.h, pre_h, _capi.u8ptr(self._fd), self.maxiter, self.tol,
                                       1 if self.printrates else 0, _capi.vptr(b), _capi.vptr(x),
                                       ctypes.byref(it)))
        self._iterations = it.value
        _note_applies(self._pre, it.value + 1)
        sv[...] = x

    def __mul__(self, vec):
        y = np.zeros(self._mat.n, dtype=self._mat.dtype)
        self.Mult(vec, y)
        return y

    @property
    def height(self):
        return self._mat.n

    @property
    def width(self):
        return self._mat.m

    def IsComplex(self):
        return self._cplx


# ---------------------------------------------------------------------------
# GMRESSolver (ngsolve/sparsesolv_solvers.hpp:409-584, factory
# sparsesolv_python_export.hpp:643-697)
# ---------------------------------------------------------------------------

class _GMRESSolverBase(_COCRSolverBase):
    def __init__(self, mat, pre, freedofs=None, maxiter=500, tol=1e-8, restart=0, printrates=False):
        super().__init__(mat, pre, freedofs, maxiter, tol, printrates)
        self.restart = int(restart)

    def Mult(self, rhs, sol):
        b = np.ascontiguousarray(_vec_view(rhs), dtype=self._mat.dtype)
        sv = _vec_view(sol)
        x = np.zeros(self._mat.n, dtype=self._mat.dtype)
        it = ctypes.c_int32(0)
        pre_h = None if self._pre is None else self._pre._h
        self._mat.refresh()
        check(self._lib.ssv_gmres_solve(self._mat.h, pre_h, _capi.u8ptr(self._fd), self.maxiter, self.tol,
                                        self.restart, _capi.vptr(b), _capi.vptr(x), ctypes.byref(it)))
        self._iterations = it.value
        if self.printrates:
            print(f"GMRES: {it.value} iterations")
        sv[...] = x


class GMRESSolverD(_GMRESSolverBase):
    _cplx = False


class GMRESSolverC(_GMRESSolverBase):
    _cplx = True


def GMRESSolver(mat, pre, freedofs=None, maxiter=500, tol=1e-8, restart=0, printrates=False):
    """Right-preconditioned restarted GMRES (modified Gram-Schmidt, Givens); `.iterations`."""
    m = mat if isinstance(mat, _Matrix) else _Matrix(mat)
    cls = GMRESSolverC if m.cplx else GMRESSolverD
    return cls(m, pre, freedofs=freedofs, maxiter=maxiter, tol=tol, restart=restart, printrates=printrates)


class COCRSolverD(_COCRSolverBase):
    _cplx = False


class COCRSolverC(_COCRSolverBase):
    _cplx = True


def COCRSolver(mat, pre, freedofs=None, maxiter=500, tol=1e-8, printrates=False):
    """COCR for complex-symmetric systems with an external preconditioner (factory :577-599)."""
    m = mat if isinstance(mat, _Matrix) else _Matrix(mat)
    cls = COCRSolverC if m.cplx else COCRSolverD
    return cls(m, pre, freedofs, maxiter, tol, printrates)


class _MixedCOCRSolverBase(_COCRSolverBase):
    def __init__(self, mat, pre, freedofs=None, maxiter=500, tol=1e-8, restart_drop=1e-5, printrates=False):
        super().__init__(mat, pre, freedofs, maxiter, tol, printrates)
        self.restart_drop = float(restart_drop)
        self._info = _capi.ssv_refine_info()

    @property
    def cycles(self):
        return self._info.cycles

    @property
    def converged(self):
        return bool(self._info.converged)

    @property
    def true_residual(self):
        return self._info.true_residual

    def Mult(self, rhs, sol):
        b = np.ascontiguousarray(_vec_view(rhs), dtype=self._mat.dtype)
        sv = _vec_view(sol)
        x = np.zeros(self._mat.n, dtype=self._mat.dtype)
        pre_h = None if self._pre is None else self._pre._h
        self._mat.refresh()
        check(self._lib.ssv_cocr_refined_solve(self._mat.h, pre_h, _capi.u8ptr(self._fd), self.maxiter, self.tol,
                                               self.restart_drop, 1 if self.printrates else 0, _capi.vptr(b),
                                               _capi.vptr(x), ctypes.byref(self._info)))
        self._iterations = self._info.iterations
        _note_applies(self._pre, self._info.iterations + self._info.cycles)
        sv[...] = x

    def solve_dev(self, d_b, d_x, d_freedofs=None):
        """Device-pointer form (integers: addresses of n-vectors in HBM; d_freedofs a uint8 mask or None)."""
        pre_h = None if self._pre is None else self._pre._h
        check(self._lib.ssv_cocr_refined_solve_dev(self._mat.h, pre_h, ctypes.cast(d_freedofs or 0, _capi.PU8),
                                                   self.maxiter, self.tol, self.restart_drop,
                                                   1 if self.printrates else 0, ctypes.c_void_p(d_b),
                                                   ctypes.c_void_p(d_x), ctypes.byref(self._info)))
        self._iterations = self._info.iterations


class MixedCOCRSolverD(_MixedCOCRSolverBase):
    _cplx = False


class MixedCOCRSolverC(_MixedCOCRSolverBase):
    _cplx = True


def MixedCOCRSolver(mat, pre, freedofs=None, maxiter=500, tol=1e-8, restart_drop=1e-5, printrates=False):
    """COCR with FP64 defect correction (new: no reference counterpart): the
    Krylov driver of the mixed-precision form. Cycles of the COCRSolver
    recurrence, each restarted from the FP64 true residual once its residual
    has dropped by ``restart_drop``; it stops when the true relative residual
    is <= tol. Use it with a preconditioner in the FP32 form
    (``precision="fp32"``), which the plain COCR recurrence cannot drive to
    1e-10. ``.iterations`` (over all cycles), ``.cycles``, ``.converged``,
    ``.true_residual``."""
    m = mat if isinstance(mat, _Matrix) else _Matrix(mat)
    cls = MixedCOCRSolverC if m.cplx else MixedCOCRSolverD
    return cls(m, pre, freedofs, maxiter, tol, restart_drop, printrates)


def has_compact_ams():
    """True when Compact AMG/AMS support is available (sparsesolv_python_export.hpp:559-560)."""
    return True


# ---------------------------------------------------------------------------
# Compact AMS (preconditioners/compact_ams.hpp, complex_compact_ams.hpp)
# ---------------------------------------------------------------------------

def _coords(c, nh1):
    a = np.ascontiguousarray(np.asarray(c, dtype=np.float64).ravel())
    if a.shape[0] != nh1:  # compact_ams.hpp:71-74
        raise RuntimeError("CompactAMS: coordinate size mismatch with H1 DOFs")
    return a


class _AmsBase(_PrecondBase):
    _complex_form = 0

    def __init__(self, mat, grad_mat, freedofs, coord_x, coord_y, coord_z, cycle_type, num_smooth,
                 correction_weight, ndof_complex=0, print_level=0):
        import time
        t0 = time.perf_counter()
        self.print_level = int(print_level)
        self._cycle_type = int(cycle_type)
        self._mult_count = 0
        self._breakdown_done = False
        ip, ix, data, cplx, shape = _csr_arrays(mat)
        if cplx:
            raise TypeError("CompactAMSPreconditioner: expected real SparseMatrix<double>")
        _, _, gdata, gcplx, gshape = _csr_arrays(grad_mat)
        if gcplx:
            raise TypeError("CompactAMSPreconditioner: grad_mat must be real SparseMatrix<double>")
        self._mat = _Matrix(mat)
        self._grad = _Matrix(grad_mat)
        self._n = self._mat.n
        self._dtype = np.complex128 if self._complex_form else np.float64
        self._fd = _freedofs_array(freedofs, self._n)
        nh1 = self._grad.m
        self._cx, self._cy, self._cz = (_coords(c, nh1) for c in (coord_x, coord_y, coord_z))
        D = _capi.PD
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.ssv_ams_create(self._mat.h, self._grad.h, _capi.u8ptr(self._fd),
                                 self._cx.ctypes.data_as(D), self._cy.ctypes.data_as(D), self._cz.ctypes.data_as(D),
                                 int(cycle_type), int(num_smooth), 0.25, float(correction_weight),
                                 self._complex_form, int(ndof_complex), ctypes.byref(h)))
        self._init_handle(h)
        if self.print_level > 0:
            self._print_setup(nh1, int(ndof_complex) or self._n, time.perf_counter() - t0)

    def _print_setup(self, nh1, ndof_complex, seconds):
        """The set-up report of print_level >= 1 (compact_ams.hpp:247-271, 325-329;
        compact_amg.hpp:119-155; complex_compact_ams.hpp:86-88): sizes, each
        subspace hierarchy's coarsening, its coarsest level, the set-up time."""
        names = ("G", "Pix", "Piy", "Piz")
        print(f"CompactAMS setup: HC={self._n} H1={nh1}", end="")
        for sub in range(4):
            lv = self.levels(sub)
            print(f"\n  subspace {names[sub]}: A={lv[0][0]}x{lv[0][0]} nnz={lv[0][1]}")
            for l in range(len(lv) - 1):
                print(f"  CompactAMG level {l}: {lv[l][0]} -> {lv[l + 1][0]} (ratio {lv[l + 1][0] / lv[l][0]:g})")
            print(f"\n  CompactAMG: {len(lv)} levels, coarsest = {lv[-1][0]} DOFs", end="")
        print(f"\n  CompactAMS setup complete: {seconds:g}s total")
        if self._complex_form:
            print(f"  ComplexCompactAMS: fused Re/Im SpMV (ndof={ndof_complex})")

    def _note_applies(self, count):
        """print_level >= 1: after the 25th application, the per-phase breakdown of
        compact_ams.hpp:185-194. The phases run inside captured device graphs, so
        their times come from one profiled cycle (CUDA events), times 25."""
        self._mult_count += count
        if self.print_level < 1 or self._breakdown_done or self._mult_count < 25:
            return
        self._breakdown_done = True
        ph = {q["name"]: q["ms"] * 1e-3 for q in self.profile(nrhs=1, reps=5)}
        k = 25
        n_smooth = 3 if self._cycle_type == 7 else 1  # full fine sweeps (the first starts from x = 0)
        smooth = n_smooth * ph["fine_smooth"]
        grad = 2 * (ph["fine_residual"] + ph["grad_transfers"] + ph["grad_vcycle"])
        nodal = ph["fine_residual"] + ph["pi_transfers"] + ph["nodal_vcycles"]
        total = ph["ams_cycle"]
        bc = max(total - smooth - grad - nodal, 0.0)
        print(f"\n  AMS Mult x{k} breakdown: smooth={k * smooth:g}s grad={k * grad:g}s nodal={k * nodal:g}s "
              f"bc={k * bc:g}s total={k * total:g}s (device time: one profiled cycle x {k})")

    def Mult(self, x, y):
        super().Mult(x, y)
        self._note_applies(1)

    def Update(self, new_mat=None):
        """Rebuild with the current matrix values, or with new_mat (geometry kept)."""
        if new_mat is None:
            self._mat.refresh()
            check(self._lib.ssv_ams_update(self._h, None))
            return
        ip, ix, _, cplx, shape = _csr_arrays(new_mat)
        if cplx:
            raise TypeError("CompactAMS::Update: expected a real SparseMatrix<double>")
        oip, oix, _, _, oshape = _csr_arrays(self._mat.src)
        if tuple(shape) == tuple(oshape) and np.array_equal(ip, oip) and np.array_equal(ix, oix):
            # same pattern (a Newton step's Jacobian): new values into the same device matrix, so
            # the set-up keeps the layouts that depend only on the pattern
            self._mat.src = new_mat
            self._mat.refresh()
            check(self._lib.ssv_ams_update(self._h, None))
            return
        m = _Matrix(new_mat)
        check(self._lib.ssv_ams_update(self._h, m.h))
        self._mat = m  # the handle now refers to the new matrix

    @property
    def precision(self):
        """"fp64" (drop-in), "fp32" (new: FP32 hierarchies and cycle, FP64 coarsest solve and in/out) or
        "fp32_nodal" (new: the gradient hierarchy FP64, the three nodal ones FP32 -- the mixed form for
        COCR on eddy-current systems)."""
        v = ctypes.c_int32()
        check(self._lib.ssv_ams_get_precision(self._h, ctypes.byref(v)))
        return {_capi.SSV_PREC_FP32: "fp32", _capi.SSV_PREC_FP32_NODAL: "fp32_nodal"}.get(v.value, "fp64")

    @precision.setter
    def precision(self, value):
        v = str(value).lower()
        if v not in ("fp32", "fp64", "fp32_nodal"):
            raise ValueError("precision must be 'fp64', 'fp32' or 'fp32_nodal'")
        check(self._lib.ssv_ams_set_precision(self._h, {"fp32": _capi.SSV_PREC_FP32,
                                                        "fp32_nodal": _capi.SSV_PREC_FP32_NODAL}.get(v, _capi.SSV_PREC_FP64)))

    def subspace_apply(self, sub, r):
        """Parity hook: one subspace correction on its own from the residual r
        (sub 0 gradient, 1..3 Nedelec x, y, z): returns (b_s, x_s, corr) -- the
        restricted residual and the subspace V-cycle's result in the hierarchy's
        coordinates (diagonally scaled where it is FP32), and the prolonged
        correction w P_s x_s."""
        nv = 2 if self._cplx else 1
        rr = np.ascontiguousarray(np.asarray(r, dtype=self._dtype)).view(np.float64)
        n1 = self._grad.m * nv
        bs, xs = np.empty(n1), np.empty(n1)
        corr = np.empty(self._n * nv)
        check(self._lib.ssv_ams_subspace_apply(self._h, int(sub), _capi.vptr(rr), _capi.vptr(bs), _capi.vptr(xs),
                                               _capi.vptr(corr)))
        if nv == 2:
            return bs.view(np.complex128), xs.view(np.complex128), corr.view(np.complex128)
        return bs, xs, corr

    def MultBlock(self, X):
        """M^{-1} applied to the rows of X (shape (nrhs, n), nrhs 1 or 4) in one block
        cycle (new: the batched driver's apply); returns an array of X's shape."""
        X = np.asarray(X, dtype=self._dtype)
        if X.ndim != 2 or X.shape[1] != self._n or X.shape[0] not in (1, 4):
            raise ValueError(f"MultBlock: X must have shape (1 or 4, {self._n})")
        k = X.shape[0]
        xi = np.ascontiguousarray(X.T)  # [row][rhs]
        out = np.empty_like(xi)
        check(self._lib.ssv_precond_apply_block(self._h, k, _capi.vptr(xi), _capi.vptr(out)))
        self._note_applies(1)
        return np.ascontiguousarray(out.T)

    def profile(self, nrhs=1, reps=20, cold=False):
        """Per-phase device time (ms) and algorithmic bytes of one cycle (measurement hook);
        cold=True times each launch alone after evicting the L2."""
        prof = _capi.ssv_phase_profile()
        check(self._lib.ssv_ams_profile(self._h, int(nrhs), int(reps), _capi.SSV_PROFILE_COLD if cold else 0,
                                        ctypes.byref(prof)))
        return prof.as_list()

    def profile_levels(self, sub, reps=20):
        """Per-level device time (ms) of subspace sub's V-cycle (measurement hook): a list of
        (level, R ms, U ms, R shape, U shape) for the levels run one by one, and the last step's ms
        (dense tail or coarsest solve)."""
        cap = 32
        mr, mu = np.zeros(cap), np.zeros(cap)
        sr, su = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        last = ctypes.c_double()
        nl = ctypes.c_int32()
        check(self._lib.ssv_ams_profile_levels(self._h, int(sub), int(reps), _capi.vptr(mr), _capi.vptr(mu),
                                               _capi.vptr(sr), _capi.vptr(su), cap, ctypes.byref(last),
                                               ctypes.byref(nl)))
        rows = [(l, float(mr[l]), float(mu[l]), int(sr[l]), int(su[l])) for l in range(max(nl.value - 1, 0))]
        return rows, last.value

    @property
    def setup_times(self):
        """Wall seconds of the last set-up (construction, Update() or precision switch): total,
        host hierarchy, fused level products, launch-shape tuner, uploads (the rest)."""
        t = np.zeros(4)
        check(self._lib.ssv_ams_setup_times(self._h, t.ctypes.data_as(_capi.PD)))
        return {"total": t[0], "host_hierarchy": t[1], "fused_products": t[2], "tuner": t[3],
                "uploads": max(t[0] - t[1] - t[2] - t[3], 0.0)}

    def level_matrix(self, subspace, level, what=0):
        """Level matrix (what=0) or interpolation (what=1) of a subspace hierarchy as set up
        (FP64, unscaled), as scipy CSR; ``.on_device`` tells whether the set-up ran on the GPU."""
        import scipy.sparse as sp
        nnz, dev = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.ssv_ams_level_matrix(self._h, subspace, level, what, None, None, None, 0, ctypes.byref(nnz),
                                             ctypes.byref(dev)))
        sizes = self.levels(subspace)
        n = sizes[level][0]
        m = n if what == 0 else sizes[level + 1][0]
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(max(nnz.value, 1), np.int32)
        v = np.zeros(max(nnz.value, 1))
        check(self._lib.ssv_ams_level_matrix(self._h, subspace, level, what, _capi.i32ptr(rp), _capi.i32ptr(ci),
                                             v.ctypes.data_as(_capi.PD), nnz.value, ctypes.byref(nnz), None))
        self.on_device = bool(dev.value)
        return sp.csr_matrix((v[: nnz.value], ci[: nnz.value], rp), shape=(n, m))

    def levels(self, subspace):
        """AMG hierarchy of a subspace (0 gradient, 1..3 Nedelec x/y/z): [(rows, nnz), ...]."""
        buf = np.zeros(256, np.int32)
        nl = ctypes.c_int32()
        check(self._lib.ssv_ams_levels(self._h, subspace, _capi.i32ptr(buf), 256, ctypes.byref(nl)))
        return [(int(buf[2 * l]), int(buf[2 * l + 1])) for l in range(nl.value)]


class CompactAMSPreconditionerImpl(_AmsBase):
    _cplx = False
    _complex_form = 0


class ComplexCompactAMSPreconditionerImpl(_AmsBase):
    _cplx = True
    _complex_form = 1


def CompactAMSPreconditioner(mat, grad_mat, freedofs=None, coord_x=(), coord_y=(), coord_z=(), cycle_type=1,
                             print_level=0, subspace_solver=0, num_smooth=1, precision="fp64"):
    """Compact AMS preconditioner for real HCurl curl-curl + mass systems (factory :410-474).

    ``precision="fp32"`` (new keyword, default the drop-in "fp64") selects the FP32-preconditioner form."""
    if subspace_solver != 0:
        raise ValueError("subspace_solver=1 (sparse Cholesky subspace solves, diagnostic) is not provided")
    p = CompactAMSPreconditionerImpl(mat, grad_mat, freedofs, coord_x, coord_y, coord_z, cycle_type,
                                     num_smooth, 1.0, print_level=print_level)
    if str(precision).lower() != "fp64":
        p.precision = precision
    return p


def ComplexCompactAMSPreconditioner(a_real_mat, grad_mat, freedofs=None, coord_x=(), coord_y=(), coord_z=(),
                                    ndof_complex=0, cycle_type=1, print_level=0, correction_weight=1.0,
                                    subspace_solver=0, num_smooth=1, precision="fp64"):
    """Complex Compact AMS: one real AMS hierarchy on a_real applied to Re and Im in fused passes
    (factory :476-557; complex_compact_ams.hpp). ``precision`` as in CompactAMSPreconditioner."""
    if subspace_solver != 0:
        raise ValueError("subspace_solver=1 (sparse Cholesky subspace solves, diagnostic) is not provided")
    p = ComplexCompactAMSPreconditionerImpl(a_real_mat, grad_mat, freedofs, coord_x, coord_y, coord_z,
                                            cycle_type, num_smooth, correction_weight, ndof_complex,
                                            print_level=print_level)
    if str(precision).lower() != "fp64":
        p.precision = precision
    return p


# ---------------------------------------------------------------------------
# PCGSolver -- CG with an external preconditioner and an initial guess (new:
# the reference's AMS scripts use NGSolve's krylovspace.CGSolver here)
# ---------------------------------------------------------------------------

class PCGSolver:
    """CG (sparsesolv::CGSolver recurrence) with any preconditioner of this module.

    ``Solve(rhs, sol)`` uses ``sol`` as the initial guess and returns a
    SparseSolvResult; ``inv * rhs`` starts from zero. Convergence rule of
    sparsesolv::CGSolver: ||r||/||b|| < tol or ||r|| < 1e-12.
    """

    def __init__(self, mat, pre=None, freedofs=None, maxiter=1000, tol=1e-10, printrates=False,
                 save_residual_history=False, conjugate=False):
        self._mat = mat if isinstance(mat, _Matrix) else _Matrix(mat)
        self._pre = pre
        self._fd = _freedofs_array(freedofs, self._mat.n)
        self._cfg = _capi.default_config(tolerance=tol, max_iterations=maxiter,
                                         save_residual_history=save_residual_history, conjugate=conjugate)
        self.printrates = bool(printrates)
        self._lib = _capi.load()
        self._last = SparseSolvResult()

    tol = property(lambda s: s._cfg.tolerance, lambda s, v: setattr(s._cfg, "tolerance", float(v)))
    maxiter = property(lambda s: s._cfg.max_iterations, lambda s, v: setattr(s._cfg, "max_iterations", int(v)))

    @property
    def iterations(self):
        return self._last.iterations

    @property
    def last_result(self):
        return self._last

    def Solve(self, rhs, sol):
        b = np.ascontiguousarray(_vec_view(rhs), dtype=self._mat.dtype)
        sv = _vec_view(sol)
        x = np.ascontiguousarray(sv, dtype=self._mat.dtype)
        cfg = _capi.ssv_config()
        ctypes.pointer(cfg)[0] = self._cfg
        if self.printrates:
            cfg.save_residual_history = 1
        cap = max(int(cfg.max_iterations), 0) + 2 if cfg.save_residual_history else 0
        hist = np.zeros(max(cap, 1))
        res = _capi.ssv_result()
        self._mat.refresh()
        check(self._lib.ssv_pcg_solve(self._mat.h, None if self._pre is None else self._pre._h,
                                      _capi.u8ptr(self._fd), ctypes.byref(cfg), _capi.vptr(b), _capi.vptr(x),
                                      ctypes.byref(res), hist.ctypes.data_as(_capi.PD), cap))
        if x is not sv:
            sv[...] = x
        r = SparseSolvResult(res.converged, res.iterations, res.final_residual,
                             hist[: res.history_len].tolist() if cfg.save_residual_history else [],
                             0.0, res.setup_seconds, res.solve_seconds, res.kernel_launches)
        if self.printrates:
            for i, v in enumerate(r.residual_history):
                print(f"CG iteration {i}, residual = {v}")
        self._last = r
        _note_applies(self._pre, res.iterations + 1)
        return r

    def Mult(self, rhs, sol):
        sv = _vec_view(sol)
        sv[...] = 0
        self.Solve(rhs, sv)

    def __mul__(self, vec):
        y = np.zeros(self._mat.n, dtype=self._mat.dtype)
        self.Mult(vec, y)
        return y


# ---------------------------------------------------------------------------
# BatchedCOCRSolver -- many frequencies x right-hand sides in one launch graph
# (new: no reference counterpart; each column runs COCRSolver's recurrence)
# ---------------------------------------------------------------------------

class BatchedCOCRSolver:
    """COCR on the family A_f = K + 1j*omegas[f]*M for every frequency f and
    ``nrhs`` right-hand sides per frequency, advanced together.

    K, M: real sparse matrices of one size (patterns merged). ``pres``: one
    ComplexCompactAMSPreconditioner per frequency (or None = identity), FP64 or
    FP32 form. ``Solve(B)`` takes B of shape (F, nrhs, n) complex and returns X
    of the same shape; ``iterations``, ``converged`` and ``residuals`` are then
    (F, nrhs) arrays with the COCRSolver meaning per column. The SpMM launch
    shape is autotuned at construction (``tuning``). ``residual_replacement``:
    every k-th step recomputes the preconditioned residual (None = automatic,
    k = 10 with FP32 preconditioners; 0 = never). ``restart_drop`` (new, the
    mixed-precision form's driver): each column runs cycles restarted from its
    FP64 true residual once its residual has dropped by this factor, and is
    done when its true relative residual is <= tol (``residuals`` then hold
    true residuals); None keeps the plain recurrence.
    """

    def __init__(self, K, M, omegas, pres, nrhs=1, freedofs=None, maxiter=500, tol=1e-8,
                 residual_replacement=None, restart_drop=None):
        self._K = K if isinstance(K, _Matrix) else _Matrix(K)
        self._M = M if isinstance(M, _Matrix) else _Matrix(M)
        if self._K.cplx or self._M.cplx:
            raise TypeError("BatchedCOCRSolver: K and M must be real")
        self._om = np.ascontiguousarray(np.asarray(omegas, dtype=np.float64).ravel())
        self.F = int(self._om.shape[0])
        self.nrhs = int(nrhs)
        self.n = self._K.n
        pres = list(pres) if pres is not None else [None] * self.F
        if len(pres) != self.F:
            raise ValueError("BatchedCOCRSolver: one preconditioner (or None) per frequency")
        self._pres = pres  # the batch keeps raw handles: hold the objects
        self._fd = _freedofs_array(freedofs, self.n)
        self.maxiter = int(maxiter)
        self.tol = float(tol)
        self._lib = _capi.load()
        harr = (ctypes.c_void_p * self.F)(*[(p._h.value if p is not None else None) for p in pres])
        h = ctypes.c_void_p()
        check(self._lib.ssv_batch_create(self._K.h, self._M.h, self.F, self._om.ctypes.data_as(_capi.PD),
                                         ctypes.cast(harr, _capi.PP), self.nrhs, _capi.u8ptr(self._fd),
                                         ctypes.byref(h)))
        self._h = h
        if residual_replacement is not None:
            check(self._lib.ssv_batch_set_replacement(self._h, int(residual_replacement)))
        self.restart_drop = None if restart_drop is None else float(restart_drop)
        if self.restart_drop:
            check(self._lib.ssv_batch_set_refinement(self._h, self.restart_drop))
        shape = (self.F, self.nrhs)
        self.iterations = np.zeros(shape, np.int32)
        self.converged = np.zeros(shape, np.int32)
        self.residuals = np.zeros(shape)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.ssv_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def Solve(self, B):
        b = np.ascontiguousarray(np.asarray(B, dtype=np.complex128))
        if b.shape != (self.F, self.nrhs, self.n):
            raise ValueError(f"BatchedCOCRSolver: right-hand sides must have shape {(self.F, self.nrhs, self.n)}")
        x = np.empty_like(b)
        check(self._lib.ssv_batch_cocr_solve(self._h, self.maxiter, self.tol, _capi.vptr(b), _capi.vptr(x),
                                             _capi.i32ptr(self.iterations), _capi.i32ptr(self.converged),
                                             self.residuals.ctypes.data_as(_capi.PD)))
        its = int(self.iterations.max()) if self.iterations.size else 0
        for p in {id(p): p for p in self._pres if p is not None}.values():
            _note_applies(p, its + 1)
        return x

    def solve_dev(self, d_b, d_x):
        """Device-pointer form (integers: addresses of (F, nrhs, n) complex128 arrays in HBM)."""
        check(self._lib.ssv_batch_cocr_solve_dev(self._h, self.maxiter, self.tol, ctypes.c_void_p(d_b),
                                                 ctypes.c_void_p(d_x), _capi.i32ptr(self.iterations),
                                                 _capi.i32ptr(self.converged),
                                                 self.residuals.ctypes.data_as(_capi.PD)))

    @property
    def tuning(self):
        """{"candidates": [(freq_tile, lanes, grid_x, us), ...], "chosen": (freq_tile, lanes, grid_x, us)}"""
        cap = 64
        arr = (_capi.ssv_batch_tune_entry * cap)()
        cnt, ch = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.ssv_batch_tuning(self._h, arr, cap, ctypes.byref(cnt), ctypes.byref(ch)))
        rows = [(e.freq_tile, e.lanes, e.grid_x, e.microseconds) for e in arr[: min(cnt.value, cap)]]
        return {"candidates": rows, "chosen": rows[ch.value] if 0 <= ch.value < len(rows) else None}

    @property
    def last_timing(self):
        """Device time of the last solve: {"device_ms", "loop_ms", "loops", "kernel_launches"}."""
        ms, lms = ctypes.c_double(), ctypes.c_double()
        loops, nk = ctypes.c_int32(), ctypes.c_int64()
        check(self._lib.ssv_batch_last_timing(self._h, ctypes.byref(ms), ctypes.byref(lms), ctypes.byref(loops),
                                              ctypes.byref(nk)))
        cyc = ctypes.c_int32()
        check(self._lib.ssv_batch_last_cycles(self._h, ctypes.byref(cyc)))
        return {"device_ms": ms.value, "loop_ms": lms.value, "loops": loops.value, "kernel_launches": nk.value,
                "cycles": cyc.value}
