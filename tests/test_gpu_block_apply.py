"""Block form of the AMS apply (ssv_precond_apply_block, MultBlock): four
right-hand sides in one cycle against four single applies of the same
preconditioner (ssv_precond_apply), and the FP64 form against the AMS oracle.

Bars: the FP64 form gives each column the single apply's result up to the
reduction order of the shape tuner's picks: 1e-10 relative (of max|y|) on
the well-conditioned family (cond ~ 3e3), 1e-7 on the SI family (iron
nu_r 1e-3, mass weight 1e-6: cond 1e8..1e11, where a 1e-16 difference in a
sum grows to ~1e-8 of max|y| in one apply; the oracle comparison uses the
same two bars). The FP32 forms agree with their own single applies to 1e-5
relative (one FP32 cycle's rounding, taken twice). The hierarchies at 6^3
are one level deep (a direct coarsest solve at level 0); at 10^3 they have
two or more levels."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu

WELL = dict(nu_r_core=1.0, mass_eps=1.0, sigma=1e5)


def _family(nc, si):
    return H.eddy_family(nc, freqs=[1e2, 1e4], nrhs=4) if si else H.eddy_family(nc, freqs=[1e2, 1e4], nrhs=4, **WELL)


def _pre(d, f, precision):
    import sparsesolv_ngsolve as ss
    return ss.ComplexCompactAMSPreconditioner(d["a_real"][f], d["G"], freedofs=d["freedofs"],
                                              coord_x=d["coords"][0], coord_y=d["coords"][1],
                                              coord_z=d["coords"][2], precision=precision)


def _rhs(d, seed):
    rng = np.random.default_rng(seed)
    n = d["A"][0].shape[0]
    X = rng.standard_normal((4, n)) + 1j * rng.standard_normal((4, n))
    return X * d["freedofs"][None, :]


@pytest.mark.parametrize("nc", [6, 10])
@pytest.mark.parametrize("precision", ["fp64", "fp32_nodal", "fp32"])
@pytest.mark.parametrize("si", [False, True])
def test_block_equals_single(nc, precision, si):
    d = _family(nc, si)
    X = _rhs(d, 3)
    tol = (1e-7 if si else 1e-10) if precision == "fp64" else 1e-5
    for f in range(2):
        p = _pre(d, f, precision)
        Y1 = np.stack([p * X[c] for c in range(4)])
        Y4 = p.MultBlock(X)
        for c in range(4):
            err = np.abs(Y4[c] - Y1[c]).max() / np.abs(Y1[c]).max()
            assert err <= tol, (f, c, err)
        Yb = p.MultBlock(X[:1])
        assert np.abs(Yb[0] - Y1[0]).max() <= tol * np.abs(Y1[0]).max()


@pytest.mark.parametrize("nc", [6, 10])
@pytest.mark.parametrize("si", [False, True])
def test_block_fp64_matches_oracle(nc, si):
    d = _family(nc, si)
    X = _rhs(d, 5)
    tol = 1e-7 if si else 1e-11
    for f in range(2):
        p = _pre(d, f, "fp64")
        o = O.AmsOracle(d["a_real"][f], d["G"], d["freedofs"], *d["coords"])
        Y4 = p.MultBlock(X)
        for c in range(4):
            yo = o.apply_complex(X[c])
            err = np.abs(Y4[c] - yo).max() / np.abs(yo).max()
            assert err <= tol, (f, c, err)


def test_block_rejects_bad_nrhs_and_kind():
    import sparsesolv_ngsolve as ss
    d = _family(6, False)
    p = _pre(d, 0, "fp64")
    with pytest.raises(ValueError):
        p.MultBlock(np.zeros((3, d["A"][0].shape[0]), dtype=np.complex128))
    ic = ss.ICPreconditioner(d["A"][0], freedofs=d["freedofs"])
    ic.Update()
    n = d["A"][0].shape[0]
    x = np.zeros(4 * n, dtype=np.complex128)
    y = np.zeros_like(x)
    from sparsesolv_ngsolve import _capi
    rc = ic._lib.ssv_precond_apply_block(ic._h, 4, _capi.vptr(x), _capi.vptr(y))
    assert rc == _capi.SSV_ERR_TYPE
