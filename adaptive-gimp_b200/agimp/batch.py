"""Batches of independent scenes stepped by shared launches (libagimp.so
agimp_batch_*).  No counterpart in the reference: it runs one AdaptiveGIMP at a
time.

    sims = [scene.build() for scene in scenes]
    batch = SceneBatch(sims)
    batch.autotune(dt)          # optional: pick launch sizes by measurement
    batch.substep(dt, 100)      # every simulator advances 100 substeps
    x0 = sims[0].x_p.to_numpy() # readback stays per simulator
"""
from __future__ import annotations

import ctypes

from . import _capi
from .simulator import _torch_stream


class SceneBatch:
    def __init__(self, sims, graphs=True):
        self._L = _capi.load()
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s._h for s in self.sims])
        h = ctypes.c_void_p()
        _capi.check(self._L.agimp_batch_create(arr, len(self.sims), ctypes.byref(h)), None, "agimp_batch_create")
        self._h = h
        self._L.agimp_batch_set_graphs(self._h, 1 if graphs else 0)

    def close(self):
        if getattr(self, "_h", None):
            self._L.agimp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.sims)

    @property
    def n_particles(self):
        return sum(s.n_particles for s in self.sims)

    def substep(self, dt0, n=1, stream=None):
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_batch_substep(self._h, float(dt0), int(n), st), self._h, "batch substep", batch=True)

    @property
    def tuning(self):
        t = _capi.Tuning()
        _capi.check(self._L.agimp_batch_get_tuning(self._h, ctypes.byref(t)), self._h, "get tuning", batch=True)
        return t.as_dict()

    def set_tuning(self, chunk=256, ctas_per_sm=8):
        t = _capi.Tuning(int(chunk), int(ctas_per_sm), 0.0)
        _capi.check(self._L.agimp_batch_set_tuning(self._h, ctypes.byref(t)), self._h, "set tuning", batch=True)

    def autotune(self, dt0, trials=5, stream=None):
        t = _capi.Tuning()
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_batch_autotune(self._h, float(dt0), int(trials), ctypes.byref(t), st), self._h,
                    "batch autotune", batch=True)
        return t.as_dict()

    def profile_substep(self, dt0, stream=None):
        """One substep of the whole batch with per-phase CUDA-event timing; {phase: ms}."""
        ms = (ctypes.c_float * len(_capi.PHASES))()
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_batch_profile_substep(self._h, float(dt0), ms, len(ms), st), self._h,
                    "batch profile", batch=True)
        return dict(zip(_capi.PHASES, list(ms)))

    def positions(self, out=None, blocking=True, stream=None):
        """x_p of every scene, concatenated in batch order ([sum of N][dim]).
        blocking=False returns at once (out required, pinned for overlap); the
        copy has landed once `stream` has run it."""
        import numpy as np
        dim = self.sims[0].dim if self.sims else 2
        shape = (self.n_particles, dim)
        if out is None:
            if not blocking:
                raise ValueError("an asynchronous copy needs `out`")
            out = np.empty(shape, np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape %s" % (shape,))
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_batch_positions_async(self._h, ctypes.c_void_p(out.ctypes.data), st), self._h,
                    "batch positions", batch=True)
        if blocking:
            import torch
            torch.cuda.synchronize()
        return out

    def set_particles(self, x=None, v=None, F=None, C=None, m=None, g=None, Jp=None):
        """Upload every scene's particles in one call: each array holds all
        scenes' particles concatenated in batch order (as positions() returns
        them), host arrays (pinned for the fastest copy) or CUDA tensors."""
        import numpy as np
        vals = [x, v, F, C, m, g, Jp]
        dtypes = [np.float32] * 5 + [np.int32, np.float32]
        try:
            import torch
            is_t = [isinstance(a, torch.Tensor) for a in vals if a is not None]
        except ImportError:
            is_t = []
        if is_t and all(is_t):
            args = [ctypes.c_void_p(a.contiguous().data_ptr()) if a is not None else None for a in vals]
            mem, st = _capi.AGIMP_MEM_DEVICE, _torch_stream()
        else:
            arrs = [np.ascontiguousarray(a, dt) if a is not None else None for a, dt in zip(vals, dtypes)]
            n = self.n_particles
            for a in arrs:
                if a is not None and a.shape[0] != n:
                    raise ValueError("batch arrays hold all %d particles of the batch, got %d" % (n, a.shape[0]))
            args = [ctypes.c_void_p(a.ctypes.data) if a is not None else None for a in arrs]
            mem, st = _capi.AGIMP_MEM_HOST, None
        # argument order of the C entry point: x, v, F, C, m, g, Jp
        _capi.check(self._L.agimp_batch_set_particles(self._h, *args, mem, st), self._h, "batch upload", batch=True)

    def kernels_per_substep(self):
        return int(self._L.agimp_batch_kernels_per_substep(self._h))

    # -- surrogate return map over the batch (extension) ------------------------
    def set_surrogate(self, mlp, xmax=None, tol=0.02):
        """Snow scenes of the batch take their return map from `mlp`
        (agimp.surrogate.MLP) with the exact map as fallback; one MLP launch per
        substep serves every scene.  None switches it off."""
        if mlp is None:
            _capi.check(self._L.agimp_batch_set_surrogate(self._h, None, None, 0.0), self._h, "batch surrogate",
                        batch=True)
            return
        xm = (ctypes.c_float * 7)(*[float(v) for v in xmax])
        self._mlp = mlp  # the parameters must outlive their use
        _capi.check(self._L.agimp_batch_set_surrogate(self._h, mlp._h, xm, float(tol)), self._h, "batch surrogate",
                    batch=True)

    def surrogate_stats(self):
        """{'handed_off', 'rejected', 'errors'} of the last substep over the batch."""
        h, r, e = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_uint32()
        _capi.check(self._L.agimp_batch_surrogate_stats(self._h, ctypes.byref(h), ctypes.byref(r), ctypes.byref(e)),
                    self._h, "batch surrogate stats", batch=True)
        return {"handed_off": h.value, "rejected": r.value, "errors": e.value}
