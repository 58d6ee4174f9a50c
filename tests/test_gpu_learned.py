"""Learned initial guess (new form): the device MLP kernels against the CPU
oracle (forward values and gradients), training on the GPU, and the Newton
sequence showing what the trained network gains over the previous-step guess
(total CG iterations on the same trajectory)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def _net(D=12, H=64, seed=1):
    from sparsesolv_ngsolve.learned import EdgeMLP
    return EdgeMLP(D, H, seed=seed)


def test_forward_matches_oracle():
    net = _net()
    rng = np.random.default_rng(0)
    X = rng.standard_normal((3000, 12)).astype(np.float32)
    p = net.params.astype(np.float64)
    ref = MO.forward(p, X, 12, 64)
    out = net.predict(X)
    assert np.abs(out - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n", [1, 257, 5000])
def test_gradients_match_oracle(n):
    net = _net(D=7, H=33, seed=3)
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, 7)).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    loss, g = net.gradients(X, y)
    lo, go = MO.loss_and_grad(net.params.astype(np.float64), X.astype(np.float64), y.astype(np.float64), 7, 33)
    # FP32 kernels against the FP64 oracle
    assert abs(loss - lo) <= 1e-5 * max(1.0, lo)
    assert np.abs(g - go).max() <= 1e-4 * max(1e-3, np.abs(go).max())


def test_set_params_roundtrip_and_shape_check():
    net = _net(D=5, H=9)
    p = np.arange(net.num_params, dtype=np.float32) * 1e-3
    net.params = p
    np.testing.assert_array_equal(net.params, p)
    with pytest.raises(ValueError):
        net.params = p[:-1]


def test_training_reduces_loss():
    net = _net(D=4, H=32, seed=5)
    rng = np.random.default_rng(7)
    X = rng.uniform(-1, 1, (20000, 4)).astype(np.float32)
    y = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] - 0.5 * X[:, 3] ** 2).astype(np.float32)
    l0, _ = net.gradients(X, y)
    net.train(X, y, epochs=30, batch=1024, lr=3e-3, seed=1)
    l1, _ = net.gradients(X, y)
    assert l1 < 0.05 * l0


def test_learned_guess_saves_iterations():
    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import newton as NW
    prob = NW.NonlinearMagnetostatic(8)
    amps = np.random.default_rng(2).uniform(0.5, 2.0, 14)

    def make_pre(J):
        return ss.CompactAMSPreconditioner(J, prob.G, freedofs=prob.freedofs, coord_x=prob.coords[0],
                                           coord_y=prob.coords[1], coord_z=prob.coords[2])

    def solver(J, pre):
        return ss.PCGSolver(J, pre, freedofs=prob.freedofs, maxiter=500, tol=1e-10)

    tr = NW.run_loads(prob, amps[:10], 5, make_pre, solver, collect=True)
    net, ys, _ = NW.train_predictor(tr)
    ev = NW.run_loads(prob, amps[9:], 5, make_pre, solver, predictor=net, scale=tr["scale"], yscale=ys)
    prev = sum(sum(x) for x in ev["iters_prev"][1:])
    mlp = sum(sum(x) for x in ev["iters_mlp"][1:])
    # the prediction is closer to the new load's solution than the previous load's
    assert np.mean(ev["start_err_mlp"]) < 0.5 * np.mean(ev["start_err_prev"])
    # and the learned guesses cut the CG iterations of the same Newton steps
    assert mlp < prev, (prev, mlp)
