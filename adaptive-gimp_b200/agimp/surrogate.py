"""Surrogate return-map MLP on the tensor cores (libagimp.so agimp_mlp_*).

The network maps 7 normalised features of a particle's trial elastic state to
4 normalised outputs (projected singular values and the new log Jp); the
feature definitions live with the simulator integration.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi

IN, H, OUT = 7, 64, 4


class MLP:
    def __init__(self, device=0, params=None, seed=0):
        self._L = _capi.load()
        self.device = device
        self.nparam = int(self._L.agimp_mlp_num_params())
        h = ctypes.c_void_p()
        _capi.check(self._L.agimp_mlp_create(device, ctypes.byref(h)), None, "agimp_mlp_create")
        self._h = h
        if params is None:
            params = self.default_init(seed)
        self.set_params(params)

    def default_init(self, seed=0):
        rng = np.random.default_rng(seed)
        out = []
        for fan_in, shape in [(IN, (IN, H)), (None, (H,)), (H, (H, H)), (None, (H,)), (H, (H, OUT)), (None, (OUT,))]:
            out.append(rng.normal(0, np.sqrt(1.0 / fan_in), shape).ravel() if fan_in else np.zeros(shape[0]))
        return np.concatenate(out).astype(np.float32)

    def close(self):
        if getattr(self, "_h", None):
            self._L.agimp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.nparam
        _capi.check(self._L.agimp_mlp_set_params(self._h, ctypes.c_void_p(p.ctypes.data), 1, None), None, "set params")

    def params(self):
        p = np.zeros(self.nparam, np.float32)
        _capi.check(self._L.agimp_mlp_get_params(self._h, ctypes.c_void_p(p.ctypes.data), 1, None), None, "get params")
        return p

    def forward(self, X):
        """X: CUDA float32 tensor [n, 7] -> CUDA float32 tensor [n, 4]."""
        import torch
        X = X.contiguous().float()
        Y = torch.empty((X.shape[0], OUT), dtype=torch.float32, device=X.device)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _capi.check(self._L.agimp_mlp_forward(self._h, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(Y.data_ptr()),
                                              X.shape[0], st), None, "mlp forward")
        return Y

    def errors(self, clear=True):
        b = ctypes.c_uint32()
        _capi.check(self._L.agimp_mlp_errors(self._h, ctypes.byref(b), 1 if clear else 0), None, "mlp errors")
        return b.value
