"""Generate golden fixtures from the reference itself.

Runs the reference's own headers (ksugahar/ngsolve-sparsesolv,
include/sparsesolv, compiled by oracle/build_oracle.py into
oracle/_ref/libssv_ref.so) single-threaded on small synthetic systems and
stores inputs and outputs in tests/golden/golden_small.npz:
solutions, iteration counts, residual histories, ABMC schedules, RCM
orderings, level schedules and one IC and one SGS preconditioner application per
system.

    python tests/golden/gen_golden.py [--rewrite]
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

# (name, builder) -- small systems the whole suite can afford on the CPU
SYSTEMS = {
    "lap3d_6": lambda: (P.laplacian_7pt(6), P.random_rhs(216, 0), None),
    "lap3d_8_fd": lambda: (P.laplacian_7pt(8), P.random_rhs(512, 1), P.boundary_freedofs_7pt(8)),
    "lap2d_12": lambda: (P.laplacian_5pt(12), P.random_rhs(144, 2), None),
    "cplx3d_6": lambda: (P.complex_shifted(P.laplacian_7pt(6), 0.3 + 0.5j),
                         P.random_rhs(216, 3, np.complex128), None),
    "cplx3d_8_fd": lambda: (P.complex_shifted(P.laplacian_7pt(8), 0.2 + 1.0j),
                            P.random_rhs(512, 4, np.complex128), P.boundary_freedofs_7pt(8)),
}

# (case name, system, method, config overrides)
CASES = [
    ("iccg_abmc", "lap3d_6", "ICCG", dict(use_abmc=1)),
    ("iccg_level", "lap3d_6", "ICCG", dict()),
    ("iccg_abmc_fd", "lap3d_8_fd", "ICCG", dict(use_abmc=1)),
    ("iccg_abmc_bs2", "lap2d_12", "ICCG", dict(use_abmc=1, abmc_block_size=2, abmc_num_colors=3)),
    ("iccg_abmc_bs8", "lap3d_8_fd", "ICCG", dict(use_abmc=1, abmc_block_size=8)),
    ("iccg_reorder", "lap3d_8_fd", "ICCG", dict(use_abmc=1, abmc_reorder_spmv=1)),
    ("iccg_scaled", "lap3d_8_fd", "ICCG", dict(diagonal_scaling=1)),
    ("iccg_abmc_scaled", "lap3d_8_fd", "ICCG", dict(use_abmc=1, diagonal_scaling=1)),
    ("iccg_autoshift", "lap3d_6", "ICCG", dict(shift_parameter=0.3, auto_shift=1, min_diagonal_threshold=2.0)),
    ("cg", "lap3d_8_fd", "CG", dict()),
    ("cg_2d", "lap2d_12", "CG", dict()),
    ("cocr_real", "lap3d_6", "COCR", dict()),
    ("sgsmrtr", "lap3d_8_fd", "SGSMRTR", dict()),
    ("sgsmrtr_2d", "lap2d_12", "SGSMRTR", dict()),
    ("cplx_iccg_abmc", "cplx3d_6", "ICCG", dict(use_abmc=1)),
    ("cplx_iccg_level_fd", "cplx3d_8_fd", "ICCG", dict()),
    ("cplx_cocr", "cplx3d_8_fd", "COCR", dict()),
    ("cplx_cg", "cplx3d_6", "CG", dict()),
    ("cplx_sgsmrtr", "cplx3d_6", "SGSMRTR", dict()),
    ("maxiter_best", "lap3d_8_fd", "CG", dict(max_iterations=7)),
    ("maxiter_nobest", "lap3d_8_fd", "CG", dict(max_iterations=7, save_best_result=0)),
    ("divergence", "lap3d_6", "CG", dict(divergence_check=1, divergence_threshold=1e-30, divergence_count=3)),
    # Path 2: RCM pre-ordering, ABMC on the RCM-reordered pattern (sparsesolv.hpp:80-97)
    ("iccg_rcm", "lap3d_8_fd", "ICCG", dict(use_abmc=1, abmc_use_rcm=1)),
    ("iccg_rcm_2d", "lap2d_12", "ICCG", dict(use_abmc=1, abmc_use_rcm=1, abmc_block_size=2, abmc_num_colors=3)),
    ("iccg_rcm_bs8", "lap3d_6", "ICCG", dict(use_abmc=1, abmc_use_rcm=1, abmc_block_size=8)),
    ("iccg_rcm_scaled", "lap3d_8_fd", "ICCG", dict(use_abmc=1, abmc_use_rcm=1, diagonal_scaling=1)),
    ("cplx_iccg_rcm", "cplx3d_8_fd", "ICCG", dict(use_abmc=1, abmc_use_rcm=1)),
]


def main():
    ref = O.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libssv_ref.so is not built (needs the reference checkout)")
    ref.ref_set_threads(1)
    out = {}
    for name, build in SYSTEMS.items():
        A, b, fd = build()
        out[f"sys/{name}/indptr"] = A.indptr.astype(np.int32)
        out[f"sys/{name}/indices"] = A.indices.astype(np.int32)
        out[f"sys/{name}/data"] = A.data
        out[f"sys/{name}/b"] = b
        if fd is not None:
            out[f"sys/{name}/fd"] = fd
        sched = O.abmc(A, 4, 4, which="ref")
        for k, v in sched.items():
            out[f"abmc/{name}/{k}"] = np.asarray(v)
        od, rv = O.rcm(A, which="ref")
        out[f"rcm/{name}/ordering"] = od
        out[f"rcm/{name}/reverse"] = rv
        L = __import__("scipy.sparse", fromlist=["tril"]).tril(A, format="csr")
        L.sort_indices()
        lev, nl = O.level_schedule(L.indptr, L.indices, A.shape[0], upper=False, which="ref")
        out[f"levels/{name}/lower"] = lev
        y, sh = O.ic_mult(A, b, O.default_config(use_abmc=1), freedofs=fd, which="ref")
        out[f"icmult/{name}/abmc"] = y
        y, sh = O.ic_mult(A, b, O.default_config(), freedofs=fd, which="ref")
        out[f"icmult/{name}/level"] = y
        y, sh = O.ic_mult(A, b, O.default_config(use_abmc=1, abmc_use_rcm=1), freedofs=fd, which="ref")
        out[f"icmult/{name}/abmc_rcm"] = y
        out[f"sgsmult/{name}"] = O.sgs_mult(A, b, freedofs=fd, which="ref")
    for case, sysname, method, over in CASES:
        A, b, fd = SYSTEMS[sysname]()
        cfg = O.default_config(save_residual_history=1, max_iterations=over.pop("max_iterations", 2000), **over)
        x, res, hist = O.solve(A, b, method, cfg, freedofs=fd, which="ref")
        out[f"case/{case}/x"] = x
        out[f"case/{case}/hist"] = hist
        out[f"case/{case}/meta"] = np.array([res.converged, res.iterations, res.final_residual], dtype=np.float64)
        out[f"case/{case}/info"] = np.array([sysname, method, repr(sorted(cfg_items(cfg)))])
        print(f"{case:20s} {sysname:12s} {method:8s} it={res.iterations:4d} conv={res.converged} "
              f"res={res.final_residual:.3e}")
    path = os.path.join(HERE, "golden_small.npz")
    if os.path.exists(path) and "--rewrite" not in sys.argv:
        # entries already committed keep their bytes (a rebuild of the reference
        # library may move the last bits of some results); new entries are added
        old = np.load(path)
        for k in old.files:
            out[k] = old[k]
    np.savez_compressed(path, **out)


def cfg_items(cfg):
    return [(f, getattr(cfg, f)) for f, _ in cfg._fields_]


if __name__ == "__main__":
    main()
