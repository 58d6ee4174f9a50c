"""print_level of the AMS factories (compact_ams.hpp:185-194, 247-271;
compact_amg.hpp:119-155; complex_compact_ams.hpp:86-88): the set-up report
at construction and, once 25 applications have been made (direct Mult calls
or the applications a solve makes inside its device graph), one per-phase
breakdown line; nothing at print_level 0."""
from __future__ import annotations

import numpy as np
import pytest

from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu


def _make(d, complex_form, print_level):
    import sparsesolv_ngsolve as ss
    kw = dict(freedofs=d["freedofs"], coord_x=d["coords"][0], coord_y=d["coords"][1], coord_z=d["coords"][2],
              print_level=print_level)
    if complex_form:
        return ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], **kw)
    return ss.CompactAMSPreconditioner(d["A"], d["G"], **kw)


def test_setup_report_and_breakdown_after_25_mults(capsys):
    d = H.magnetostatic(10)  # 1,331 vertices: more than one AMG level
    p = _make(d, False, 1)
    out = capsys.readouterr().out
    assert f"CompactAMS setup: HC={d['A'].shape[0]} H1={d['G'].shape[1]}" in out
    assert "CompactAMG level 0:" in out and "levels, coarsest =" in out
    assert "CompactAMS setup complete:" in out
    lv = p.levels(0)
    assert f"CompactAMG level 0: {lv[0][0]} -> {lv[1][0]}" in out
    b = np.random.default_rng(0).standard_normal(d["A"].shape[0])
    for k in range(24):
        p * b
    assert "breakdown" not in capsys.readouterr().out
    p * b
    out = capsys.readouterr().out
    assert out.count("AMS Mult x25 breakdown: smooth=") == 1 and "total=" in out
    for k in range(30):
        p * b
    assert "breakdown" not in capsys.readouterr().out  # printed once, as the reference does


def test_breakdown_counts_applications_inside_a_solve(capsys):
    import sparsesolv_ngsolve as ss
    d = H.eddy_current(6)
    p = _make(d, True, 1)
    assert "ComplexCompactAMS: fused Re/Im SpMV" in capsys.readouterr().out
    inv = ss.COCRSolver(d["A"], p, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    inv * d["f"]
    assert inv.iterations >= 25
    assert "AMS Mult x25 breakdown" in capsys.readouterr().out


def test_print_level_zero_is_silent(capsys):
    d = H.magnetostatic(6)
    p = _make(d, False, 0)
    b = np.ones(d["A"].shape[0])
    for _ in range(26):
        p * b
    assert capsys.readouterr().out == ""
