"""The oracle (C restatement) on edge inputs against the reference's own
outputs (tests/golden/golden_edge.npz, made by gen_golden_edge.py): a NaN in b
(the solve runs to maxiter, reports DBL_MAX and the zero vector with
save_best_result, NaN without) and a zero b with and without an initial guess."""
from __future__ import annotations

import pytest

from conftest import assert_same_outcome, edge_cases
from oracle import oracle as O

CASES = edge_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["case"] for c in CASES])
def test_oracle_edge_case(case):
    cfg = O.default_config()
    for k, v in case["items"]:
        setattr(cfg, k, v)
    x, res, hist = O.solve(case["A"], case["b"], case["method"], cfg, x0=case["x0"], which="port")
    assert_same_outcome(case, res.converged, res.iterations, res.final_residual, x, hist)
