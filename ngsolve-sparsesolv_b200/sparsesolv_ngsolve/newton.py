"""Nonlinear magnetostatic Newton sequences with Update() + Compact AMS + CG,
and the learned initial guess (new: no reference counterpart).

Problem: the Kuhn-mesh HCurl system of the magnetostatic configuration with
an iron reluctivity depending on the flux density, nu(|B|) = nu0 (k1 + k2
|B|^2) in the iron block (nu0 = 1, k1 = 1e-3, k2 = 5e-3), nu = 1 in air, plus
a 1e-6 M mass regularisation, Dirichlet on the boundary; B = curl u is constant
per tetrahedron. A sequence of loads f_l = a_l f (a_l ~ U[0.5, 2]) is solved
by Newton's method, each load starting from the previous load's solution.
Every Newton step solves J(u_k) u_{k+1} = J(u_k) u_k - F(u_k) with the
Jacobian J = K(nu) + 1e-6 M + 2 k2 nu0 (B . curl w_i)(B . curl w_j) on iron,
after ``pre.Update(J)``, by PCG to 1e-10. The unknown of each linear solve is
the new iterate, so the previous-step guess is u_k.

The learned guess: between loads, a per-edge MLP (``EdgeMLP``, 64 hidden
units, FP32, trained and run by the library's own kernels) predicts the next
load's solution u*_l from the previous one. Its features per edge are the
midpoint, the direction, u*_{l-1}[e] / (a_{l-1} S), log10 nu(u*_{l-1}) on the
edge, a_l, a_{l-1}, a_l / a_{l-1} - 1 and the nonlinear residual of the
previous solution under the new load, F(u*_{l-1}; a_l f)[e] / (a_l |f|_inf);
its target is the change of the
solution per unit amplitude, (u*_l / a_l - u*_{l-1} / a_{l-1})[e] / (S Ys), S a
fixed solution scale and Ys the training targets' standard deviation. The
Newton trajectory is the baseline's (each load starts from the previous
load's solution); the prediction only sets the initial guesses of its linear
solves: at step k the guess is u_k + beta (p - u_k), p the prediction and
beta in [0, 1.5] the step along p - u_k that minimises the J-norm of the
guess's error (one SpMV and two dot products), so beta = 0 -- the
previous-step guess u_k, the fallback -- is taken whenever the prediction
does not help. Trained on the first loads of a sequence; judged on the
remaining ones by the total CG iterations of their Newton steps against the
previous-step guesses on the same trajectory.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import hcurl as H

class NonlinearMagnetostatic:
    def __init__(self, nc, k1=1e-3, k2=5e-3, mass_eps=1e-6):
        m = H.kuhn_mesh(nc)
        self.m = m
        self.k1, self.k2, self.eps = k1, k2, mass_eps
        self.Ke, self.Me = H.element_matrices(m)
        ga = m.grads[:, H._LE[:, 0], :]
        gb = m.grads[:, H._LE[:, 1], :]
        self.curl = 2.0 * np.cross(ga, gb) * m.tet_signs[:, :, None]  # (nt, 6, 3)
        self.iron = H._inside(m.centroids, 0.3, 0.7)
        ne = m.ne
        rows = np.repeat(m.tet_edges, 6, axis=1).ravel()
        cols = np.tile(m.tet_edges, (1, 6)).ravel()
        key = rows * ne + cols
        ukey, inv = np.unique(key, return_inverse=True)
        self.map = inv
        self.indices = (ukey % ne).astype(np.int32)
        counts = np.bincount(ukey // ne, minlength=ne)
        self.indptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        self.nnz = ukey.shape[0]
        self.G = H.gradient_matrix(m)
        self.freedofs = H.boundary_freedofs(m)
        self.fd = self.freedofs.astype(bool)
        self.coords = (m.coords[:, 0].copy(), m.coords[:, 1].copy(), m.coords[:, 2].copy())
        self.f_unit = H.loop_source(m, z_levels=(0.5,), squares=((0.15, 0.85), (0.2, 0.8))) * self.freedofs
        # per-edge geometry features
        p0, p1 = m.coords[m.edges[:, 0]], m.coords[m.edges[:, 1]]
        d = p1 - p0
        self.edge_mid = 0.5 * (p0 + p1) - 0.5
        self.edge_dir = d / np.linalg.norm(d, axis=1)[:, None]
        self.tets_per_edge = np.bincount(m.tet_edges.ravel(), minlength=ne).astype(np.float64)

    # B per tetrahedron and nu
    def fields(self, u):
        ue = u[self.m.tet_edges]
        B = np.einsum("ti,tie->te", ue, self.curl)
        b2 = (B * B).sum(axis=1)
        nu = np.where(self.iron, self.k1 + self.k2 * b2, 1.0)
        return B, nu

    def _csr(self, vals):
        data = np.bincount(self.map, weights=vals.ravel(), minlength=self.nnz)
        A = sp.csr_matrix((data, self.indices, self.indptr), shape=(self.m.ne, self.m.ne))
        A.indptr = A.indptr.astype(np.int32)
        A.indices = A.indices.astype(np.int32)
        return A

    def jacobian(self, u):
        B, nu = self.fields(u)
        vals = nu[:, None, None] * self.Ke + self.eps * self.Me
        bc = np.einsum("te,tie->ti", B[self.iron], self.curl[self.iron])
        vals[self.iron] += (2.0 * self.k2 * self.m.vol[self.iron])[:, None, None] * bc[:, :, None] * bc[:, None, :]
        return self._csr(vals)

    def residual(self, u, f):
        """F(u) = K(nu(u)) u + eps M u - f on the free edges (0 on constrained ones)."""
        _, nu = self.fields(u)
        ue = u[self.m.tet_edges]
        loc = np.einsum("tij,tj->ti", nu[:, None, None] * self.Ke + self.eps * self.Me, ue)
        F = np.bincount(self.m.tet_edges.ravel(), weights=loc.ravel(), minlength=self.m.ne) - f
        return np.where(self.fd, F, 0.0)

    def edge_nu(self, nu):
        s = np.bincount(self.m.tet_edges.ravel(), weights=np.repeat(nu, 6), minlength=self.m.ne)
        return s / self.tets_per_edge


N_FEATURES = 12


def load_features(prob, u_prev, a_prev, a, scale):
    """Per-edge features (ne x 12, float32) for predicting load a from the solution of load a_prev."""
    _, nu = prob.fields(u_prev)
    f = a * prob.f_unit
    res = prob.residual(u_prev, f) / max(float(np.abs(f).max()), 1e-300)
    X = np.empty((prob.m.ne, N_FEATURES), np.float32)
    X[:, 0:3] = prob.edge_mid
    X[:, 3:6] = prob.edge_dir
    X[:, 6] = u_prev / (a_prev * scale)
    X[:, 7] = np.log10(np.maximum(prob.edge_nu(nu), 1e-12)) / 3.0
    X[:, 8] = a / 2.0
    X[:, 9] = a_prev / 2.0
    X[:, 10] = a / a_prev - 1.0
    X[:, 11] = res
    return X


def newton_load(prob, u0, a, nsteps, state, make_pre, solver_factory, target=None):
    """nsteps Newton steps of load a from u0 (Update() + AMS + PCG per step);
    returns (u, CG iterations per step, betas). With `target` (a predicted
    solution), each linear solve starts from u_k + beta (target - u_k) with the
    J-norm-optimal beta in [0, 1.5]; otherwise from u_k."""
    f = a * prob.f_unit
    fd = prob.fd
    u = u0.copy()
    its, betas = [], []
    for _ in range(nsteps):
        J = prob.jacobian(u)
        F = prob.residual(u, f)
        rhs = np.where(fd, J @ u - F, 0.0)
        if state.get("pre") is None:
            state["pre"] = make_pre(J)
        else:
            state["pre"].Update(J)
        x = u.copy()
        if target is not None:
            d = np.where(fd, target - u, 0.0)
            Jd = np.where(fd, J @ d, 0.0)
            den = float(d @ Jd)
            beta = float(np.clip(d @ (-F) / den, 0.0, 1.5)) if den > 0 else 0.0
            x = u + beta * d
            betas.append(beta)
        r = solver_factory(J, state["pre"]).Solve(rhs, x)
        its.append(r.iterations)
        u = x
    return u, its, betas


def run_loads(prob, amps, nsteps, make_pre, solver_factory, predictor=None, scale=None, yscale=1.0,
              collect=False):
    """Newton over the loads `amps`, each starting from the previous load's
    solution (u = 0 for the first). With a predictor, every load after the
    first is solved a second time on the same trajectory with the learned
    guesses. collect=True gathers (X, Y) samples."""
    ne = prob.m.ne
    state = {}
    out = {"iters_prev": [], "iters_mlp": [], "X": [], "Y": [], "scale": scale, "betas": [], "loads": 0,
           "start_err_prev": [], "start_err_mlp": []}
    u_prev = np.zeros(ne)
    a_prev = 0.0
    for a in amps:
        u, its, _ = newton_load(prob, u_prev, a, nsteps, state, make_pre, solver_factory)
        out["iters_prev"].append(its)
        if out["scale"] is None:
            out["scale"] = max(float(np.abs(u).max()) / a, 1e-30)
        if a_prev > 0:
            if predictor is not None:
                X = load_features(prob, u_prev, a_prev, a, out["scale"])
                pred = a * (u_prev / a_prev + out["scale"] * yscale * predictor.predict(X).astype(np.float64))
                pred = np.where(prob.fd, pred, 0.0)
                _, its_m, betas = newton_load(prob, u_prev, a, nsteps, state, make_pre, solver_factory, target=pred)
                out["iters_mlp"].append(its_m)
                out["betas"].append(betas)
                nrm = max(float(np.abs(u).max()), 1e-300)
                out["start_err_prev"].append(float(np.abs(u_prev - u).max()) / nrm)
                out["start_err_mlp"].append(float(np.abs(pred - u).max()) / nrm)
                out["loads"] += 1
            if collect:
                X = load_features(prob, u_prev, a_prev, a, out["scale"])
                out["X"].append(X[prob.fd])
                out["Y"].append(((u / a - u_prev / a_prev) / out["scale"])[prob.fd].astype(np.float32))
        elif predictor is not None:
            out["iters_mlp"].append(its)
        u_prev, a_prev = u, a
    return out


def train_predictor(samples, hidden=64, epochs=150, batch=1024, lr=1e-3, seed=0):
    """Standardise the targets and train an EdgeMLP on the GPU; returns (net, yscale, last loss)."""
    from .learned import EdgeMLP
    X = np.concatenate(samples["X"])
    Y = np.concatenate(samples["Y"])
    ys = float(Y.std()) or 1.0
    net = EdgeMLP(N_FEATURES, hidden, seed=seed)
    loss = net.train(X, Y / ys, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return net, ys, loss
