"""Surrogate return-map MLP on the tensor cores (libagimp.so agimp_mlp_*).

The network maps 7 normalised features of a particle's trial elastic state to
4 normalised outputs (the return map's change of the singular values and of
log Jp, which decode to the projected singular values and the new log Jp);
the feature definitions live with the simulator integration
(csrc/common.cuh snow_features).
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


# ---------------------------------------------------------------------------
# training pipeline
SIG, LJ, HSC = 0.05, 0.5, 5.0  # input scales (csrc/common.cuh snow_features)
DSIG, DLJ = 0.02, 0.02  # output scales: changes of sig and log Jp


def record_pairs(scene, capacity, stride=1, max_substeps=400, device=0, **sim_over):
    """Run the plain (SVD) return map on `scene` and record up to `capacity`
    (features, projected state) pairs; returns CUDA tensors X [n, 7], T [n, 4]."""
    import torch
    sim = scene.build(device=device, **sim_over)
    X = torch.empty((capacity, IN), dtype=torch.float32, device="cuda:%d" % device)
    T = torch.empty((capacity, OUT), dtype=torch.float32, device="cuda:%d" % device)
    sim.set_recorder(X, T, stride)
    for i in range(max_substeps):
        if scene.refine_every and i % scene.refine_every == 0:
            sim.refine_levels(scene.refine_band)
        sim.substep(scene.dt)
        if i % 20 == 19 and sim.recorded() >= capacity:
            break
    n = min(sim.recorded(), capacity)
    sim.close()
    return X[:n], T[:n]


def trained_range(X, margin=1.05, floor=1e-3):
    """Per-feature bound |x_k| <= xmax_k of the training inputs."""
    import torch
    m = X.abs().amax(dim=0).float().cpu().numpy()
    return np.maximum(m * margin, floor).astype(np.float32)


def train(mlp, X, T, steps=2000, batch=65536, lr=3e-3, lr_final=3e-4, seed=0, log_every=0):
    """Adam on random minibatches (tensor-core gradients); returns the loss history."""
    import torch
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    loss = torch.zeros(1, dtype=torch.float32, device=X.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = mlp._L
    L.agimp_mlp_reset_optimizer(mlp._h)
    hist = []
    n = X.shape[0]
    for it in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), generator=g, device=X.device)
        xb, tb = X[idx].contiguous(), T[idx].contiguous()
        a = it / max(steps - 1, 1)
        rate = lr * (lr_final / lr) ** a  # geometric decay
        _capi.check(L.agimp_mlp_train_step(mlp._h, ctypes.c_void_p(xb.data_ptr()), ctypes.c_void_p(tb.data_ptr()),
                                           xb.shape[0], ctypes.c_float(rate), ctypes.c_void_p(loss.data_ptr()), st),
                    None, "train step")
        if log_every and (it % log_every == 0 or it == steps - 1):
            hist.append((it, float(loss.item())))
    return hist


def evaluate(mlp, X, T):
    """Mean squared error and max abs error of the MLP on (X, T)."""
    Y = mlp.forward(X)
    d = (Y - T).abs()
    return float((d ** 2).sum(1).mean().item()), float(d.max().item())


def save(path, mlp, xmax, meta=None):
    np.savez(path, params=mlp.params(), xmax=np.asarray(xmax, np.float32), **(meta or {}))


def load(path, device=0):
    z = np.load(path)
    return MLP(device=device, params=z["params"]), z["xmax"]


def bench(rows=2_000_000, reps=10, device=0):
    """Throughput of the tensor-core forward pass and of one training step on
    `rows` random samples (CUDA events); returns a dict."""
    import torch
    m = MLP(device=device)
    X = torch.randn((rows, IN), device="cuda:%d" % device)
    T = torch.randn((rows, OUT), device="cuda:%d" % device)
    for _ in range(3):
        m.forward(X)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        m.forward(X)
    e1.record()
    torch.cuda.synchronize()
    fwd = e0.elapsed_time(e1) / reps
    train(m, X, T, steps=3, batch=min(rows, 1 << 20))
    torch.cuda.synchronize()
    e0.record()
    train(m, X, T, steps=reps, batch=min(rows, 1 << 20))
    e1.record()
    torch.cuda.synchronize()
    step = e0.elapsed_time(e1) / reps
    flop = 2 * (IN * H + H * H + H * OUT)
    return {"rows": rows, "forward_ms": fwd, "forward_tflops": rows * flop / (fwd * 1e-3) / 1e12,
            "train_step_ms": step, "train_batch": min(rows, 1 << 20), "errors": m.errors()}


if __name__ == "__main__":
    import json
    import sys
    print(json.dumps(bench(int(sys.argv[1]) if len(sys.argv) > 1 else 2_000_000)))
