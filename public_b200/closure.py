"""Learned subgrid closure: the tensor-core MLP of libcruna_b200.so (cruna_mlp_*) behind a small
Python class, with device arrays passed as torch CUDA tensors (PyTorch is plumbing here: memory and
streams; the arithmetic runs in the library's tcgen05 kernels).

No counterpart in the reference (CRUNA has no learned component).  Features per point (12): the nine
velocity-gradient components du_i/dx_j ordered (u_x, u_y, u_z, v_x, v_y, v_z, w_x, w_y, w_z), density,
temperature and the filter width; targets (6): the subgrid stresses tau_11, tau_22, tau_33, tau_12,
tau_13, tau_23.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from .cruna import CrunaError, load_library

NPARAMS = 5382
NIN, NOUT = 12, 6


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


class ClosureMLP:
    """One MLP (parameters, Adam state and its own CUDA stream) on one device."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.cruna_mlp_create(int(device), int(seed), C.byref(h))
        if rc != 0:
            raise CrunaError(rc, "cruna_mlp_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.cruna_mlp_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.cruna_mlp_last_error(self.h)
            raise CrunaError(rc, msg.decode() if msg else "")

    @property
    def params(self) -> np.ndarray:
        p = np.empty(NPARAMS, np.float32)
        self._check(self.lib.cruna_mlp_get_params(self.h, p.ctypes.data_as(C.c_void_p)))
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        if p.size != NPARAMS:
            raise ValueError(f"expected {NPARAMS} parameters")
        self._check(self.lib.cruna_mlp_set_params(self.h, p.ctypes.data_as(C.c_void_p)))

    def set_scaling(self, in_mean: Sequence[float], in_scale: Sequence[float], out_scale: Sequence[float]):
        a, b, c = _f32(in_mean), _f32(in_scale), _f32(out_scale)
        self._check(self.lib.cruna_mlp_set_scaling(self.h, a.ctypes.data_as(C.c_void_p),
                                                   b.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p)))

    @staticmethod
    def _dev(t, cols: int):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise TypeError("expected a contiguous float32 CUDA tensor")
        if t.ndim != 2 or t.shape[1] != cols:
            raise ValueError(f"expected shape (n, {cols})")
        return C.c_void_p(t.data_ptr())

    def forward(self, X, out=None):
        """Stresses (n, 6) of features X (n, 12), both float32 CUDA tensors."""
        import torch
        n = X.shape[0]
        Y = out if out is not None else torch.empty((n, NOUT), dtype=torch.float32, device=X.device)
        torch.cuda.current_stream(X.device).synchronize()
        self._check(self.lib.cruna_mlp_forward_dev(self.h, self._dev(X, NIN), self._dev(Y, NOUT), int(n)))
        return Y

    def grad(self, X, Y):
        """(loss, gradient) of the mean squared error on the n samples (n a multiple of 128)."""
        import torch
        g = np.empty(NPARAMS, np.float32)
        loss = C.c_float()
        torch.cuda.current_stream(X.device).synchronize()
        self._check(self.lib.cruna_mlp_grad_dev(self.h, self._dev(X, NIN), self._dev(Y, NOUT), int(X.shape[0]),
                                                g.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return float(loss.value), g

    def train(self, X, Y, batch: int, steps: int, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        """Adam over `steps` mini-batches; returns the loss of every step."""
        import torch
        hist = np.empty(max(steps, 1), np.float32)
        torch.cuda.current_stream(X.device).synchronize()
        self._check(self.lib.cruna_mlp_train_dev(self.h, self._dev(X, NIN), self._dev(Y, NOUT), int(X.shape[0]),
                                                 int(batch), int(steps), float(lr), int(seed),
                                                 hist.ctypes.data_as(C.c_void_p)))
        return hist[:steps]
