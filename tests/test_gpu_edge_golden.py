"""The sm_100a path on edge inputs against the reference's own outputs
(tests/golden/golden_edge.npz): a NaN in b runs to maxiter and returns what
the reference returns (DBL_MAX and the zero vector with save_best_result, NaN
without; a NaN history), a zero b converges from an initial guess as the
reference does, and from a zero guess at once. Through SparseSolvSolver with
the fixture's configuration and initial guess."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_outcome, edge_cases

pytestmark = pytest.mark.gpu

CASES = edge_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["case"] for c in CASES])
def test_gpu_edge_case(case):
    import sparsesolv_ngsolve as ss
    d = dict(case["items"])
    s = ss.SparseSolvSolver(case["A"], method=case["method"], tol=d["tolerance"], maxiter=d["max_iterations"],
                            shift=d["shift_parameter"], save_best_result=bool(d["save_best_result"]),
                            save_residual_history=bool(d["save_residual_history"]),
                            conjugate=bool(d["conjugate"]), use_abmc=bool(d["use_abmc"]),
                            abmc_block_size=d["abmc_block_size"], abmc_num_colors=d["abmc_num_colors"])
    x = np.array(case["x0"], copy=True)
    r = s.Solve(case["b"], x)
    assert_same_outcome(case, r.converged, r.iterations, r.final_residual, x, r.residual_history)
