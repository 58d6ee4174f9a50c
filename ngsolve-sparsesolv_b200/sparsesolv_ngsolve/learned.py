"""Learned initial guess for Update()-driven Newton sequences (new: no
reference counterpart).

``EdgeMLP`` is a 2-layer per-edge MLP (FP32, ``hidden`` units) whose training
and inference run in the library's own CUDA kernels (csrc/mlp.cu) through the
C ABI: ``train`` (minibatch Adam on device-resident samples), ``predict``,
and ``gradients`` (the hook the CPU gradient check uses).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import check


class EdgeMLP:
    def __init__(self, in_dim, hidden=64, seed=0):
        self._lib = _capi.load()
        h = ctypes.c_void_p()
        check(self._lib.ssv_mlp_create(int(in_dim), int(hidden), int(seed), ctypes.byref(h)))
        self._h = h
        self.in_dim = int(in_dim)
        self.hidden = int(hidden)
        n = ctypes.c_int32()
        check(self._lib.ssv_mlp_num_params(self._h, ctypes.byref(n)))
        self.num_params = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.ssv_mlp_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def params(self):
        p = np.empty(self.num_params, np.float32)
        check(self._lib.ssv_mlp_get_params(self._h, p.ctypes.data_as(_capi.PF)))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (self.num_params,):
            raise ValueError(f"EdgeMLP: expected {self.num_params} parameters")
        check(self._lib.ssv_mlp_set_params(self._h, p.ctypes.data_as(_capi.PF)))

    def gradients(self, X, y):
        """(loss, gradient) of the mean squared error on host arrays (device kernels)."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        if X.ndim != 2 or X.shape[1] != self.in_dim or y.shape != (X.shape[0],):
            raise ValueError("EdgeMLP.gradients: X must be (n, in_dim) and y (n,)")
        g = np.empty(self.num_params, np.float32)
        loss = ctypes.c_float()
        check(self._lib.ssv_mlp_gradients(self._h, X.ctypes.data_as(_capi.PF), y.ctypes.data_as(_capi.PF),
                                          X.shape[0], g.ctypes.data_as(_capi.PF), ctypes.byref(loss)))
        return float(loss.value), g

    @staticmethod
    def _device(a):
        import torch
        if isinstance(a, torch.Tensor):
            return a.to(device="cuda", dtype=torch.float32).contiguous()
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to("cuda")

    def train(self, X, y, epochs=10, batch=8192, lr=1e-3, seed=0):
        """Minibatch Adam on the GPU; returns the last batch's loss."""
        dX, dy = self._device(X), self._device(y)
        if dX.ndim != 2 or dX.shape[1] != self.in_dim or dy.shape != (dX.shape[0],):
            raise ValueError("EdgeMLP.train: X must be (n, in_dim) and y (n,)")
        loss = ctypes.c_float()
        check(self._lib.ssv_mlp_train_dev(self._h, ctypes.c_void_p(dX.data_ptr()), ctypes.c_void_p(dy.data_ptr()),
                                          dX.shape[0], int(epochs), int(batch), float(lr), int(seed),
                                          ctypes.byref(loss)))
        return float(loss.value)

    def predict(self, X):
        """MLP(X) for X (n, in_dim): numpy in, numpy out (the kernel runs on the GPU)."""
        import torch
        dX = self._device(X)
        out = torch.empty(dX.shape[0], dtype=torch.float32, device="cuda")
        check(self._lib.ssv_mlp_predict_dev(self._h, ctypes.c_void_p(dX.data_ptr()), dX.shape[0],
                                            ctypes.c_void_p(out.data_ptr())))
        return out.cpu().numpy()
