"""Generate the edge-input fixtures from the reference itself.

Runs the reference's own headers (compiled by oracle/build_oracle.py into
oracle/_ref/libssv_ref.so) single-threaded on right-hand sides and initial
guesses the main fixtures do not cover -- a NaN entry in b, a zero b -- with a
nonzero initial guess, and stores inputs and outputs in
tests/golden/golden_edge.npz: solutions, iteration counts, convergence flags,
final residuals and residual histories (NaN where the reference produces NaN).

    python tests/golden/gen_golden_edge.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "ngsolve-sparsesolv_b200"))

from oracle import oracle as O  # noqa: E402
from sparsesolv_ngsolve import problems as P  # noqa: E402


def _real():
    return P.laplacian_7pt(6)


def _cplx():
    return P.complex_shifted(P.laplacian_7pt(6), 0.3 + 0.5j)


def _rhs(A, kind, seed):
    n = A.shape[0]
    if kind == "zero":
        return np.zeros(n, dtype=A.dtype)
    b = P.random_rhs(n, seed=seed, dtype=A.dtype)
    if kind == "nan":
        b[n // 3] = np.nan
    return b


def _x0(A, kind):
    n = A.shape[0]
    if kind == "zeros":
        return np.zeros(n, dtype=A.dtype)
    return np.linspace(0.5, 1.5, n).astype(A.dtype)


# (case, matrix, method, rhs, initial guess, config overrides)
CASES = [
    ("nan_cg_best", _real, "CG", "nan", "ramp", dict(max_iterations=12)),
    ("nan_cg_nobest", _real, "CG", "nan", "ramp", dict(max_iterations=12, save_best_result=0)),
    ("nan_iccg_level_best", _real, "ICCG", "nan", "ramp", dict(max_iterations=12)),
    ("nan_iccg_abmc_nobest", _real, "ICCG", "nan", "ramp", dict(max_iterations=12, use_abmc=1, save_best_result=0)),
    ("nan_sgsmrtr_best", _real, "SGSMRTR", "nan", "ramp", dict(max_iterations=12)),
    ("nan_cplx_cocr_best", _cplx, "COCR", "nan", "ramp", dict(max_iterations=12)),
    ("nan_cplx_iccg_nobest", _cplx, "ICCG", "nan", "ramp", dict(max_iterations=12, save_best_result=0)),
    ("zero_rhs_cg_guess", _real, "CG", "zero", "ramp", dict(max_iterations=200)),
    ("zero_rhs_iccg_zero_guess", _real, "ICCG", "zero", "zeros", dict(max_iterations=200)),
    ("zero_rhs_cplx_cocr_guess", _cplx, "COCR", "zero", "ramp", dict(max_iterations=200)),
]


def main():
    ref = O.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libssv_ref.so is not built (needs the reference checkout)")
    ref.ref_set_threads(1)
    out = {}
    for k, (case, build, method, rhs, guess, over) in enumerate(CASES):
        A = build()
        b = _rhs(A, rhs, seed=10 + k)
        x0 = _x0(A, guess)
        over = dict(over)
        cfg = O.default_config(save_residual_history=1, tolerance=1e-10,
                               max_iterations=over.pop("max_iterations"), **over)
        x, res, hist = O.solve(A, b, method, cfg, x0=x0, which="ref")
        out[f"{case}/indptr"] = A.indptr.astype(np.int32)
        out[f"{case}/indices"] = A.indices.astype(np.int32)
        out[f"{case}/data"] = A.data
        out[f"{case}/b"] = b
        out[f"{case}/x0"] = x0
        out[f"{case}/x"] = x
        out[f"{case}/hist"] = hist
        out[f"{case}/meta"] = np.array([res.converged, res.iterations, res.final_residual], dtype=np.float64)
        out[f"{case}/info"] = np.array([method, repr(sorted((f, getattr(cfg, f)) for f, _ in cfg._fields_))])
        print(f"{case:26s} {method:8s} it={res.iterations:4d} conv={res.converged} res={res.final_residual:.3e} "
              f"nan(x)={int(np.isnan(x).sum())}")
    np.savez_compressed(os.path.join(HERE, "golden_edge.npz"), **out)


if __name__ == "__main__":
    main()
