"""AdaptiveGIMP: the reference's simulator class over the B200 C ABI.

Mirrors ``AdaptiveGIMP`` of adaptive_gimp.py (g1n0st/adaptive-gimp): the same
constructor arguments and call order (storage, constants, then
``particle_initializer(self)``, then ``grid_initializer``), the same attribute
and field names, ``substep(dt0)``, and the node predicates.  The state lives in
device memory owned by libagimp.so; fields are views with Taichi's
``to_numpy`` / ``from_numpy`` plus ``to_torch`` / ``from_torch``.

Differences a caller of the reference should know (each is forced by the
reference relying on Taichi JIT features):

* ``grid_initializer`` is tabulated once over the finest cells (plus a halo)
  at construction.  A plain function ``f(sim, I) -> level`` that calls
  ``sim.activate_cell(level, I)`` (the reference's form, init.py:34-98) is
  evaluated per cell in Python; a function with attribute ``vectorized = True``
  receives an int array ``I[..., dim]`` and returns ``(level, activate)``
  arrays.  It must activate nothing or exactly the cell of the returned level
  that contains ``I``.
* Physical constants that the reference hard-codes (adaptive_gimp.py:48-53) are
  keyword overrides with the reference's values as defaults.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import AGIMP_MEM_DEVICE, AGIMP_MEM_HOST

UNACTIVATED, ACTIVATED, GHOST, T_JUNCTION, CULLING = 0, 1, 2, 4, 8


def align_size(x, align):
    """utils.py:44-45"""
    return (x + (align - 1)) & ~(align - 1)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _torch_stream():
    try:
        import torch
        if torch.cuda.is_available():
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    except ImportError:
        pass
    return None


class ParticleField:
    """One particle field (x_p, v_p, F_p, C_p, m_p, g_p, fl_p, Jp)."""

    _ORDER = ("x", "v", "F", "C", "m", "g", "fl", "Jp")

    def __init__(self, sim, name, shape, dtype, writable=True):
        self.sim, self.name, self.shape, self.dtype, self.writable = sim, name, shape, dtype, writable

    def _args(self, buf):
        args = [None] * 8
        args[self._ORDER.index(self.name)] = buf
        return args

    def to_numpy(self, out=None, blocking=True, stream=None):
        """Copy to host memory (into `out` when given, e.g. a pinned buffer).

        blocking=False enqueues the copy on `stream` (a CUDA stream handle;
        default the current torch stream) and returns at once: `out` (required,
        pinned for the copy to overlap) holds the state once that stream has
        run the copy.  The next substep may run meanwhile; the library orders
        whatever would overwrite this state after the copy."""
        if out is None:
            if not blocking:
                raise ValueError("an asynchronous copy needs `out`")
            out = np.empty(self.shape, self.dtype)
        elif out.shape != self.shape or out.dtype != self.dtype or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous %s array of shape %s" % (np.dtype(self.dtype), self.shape))
        a = self._args(_ptr(out))
        s = self.sim
        if blocking:
            _capi.check(s._L.agimp_get_particles(s._h, *a, AGIMP_MEM_HOST, stream), s._h, "get " + self.name)
        else:
            st = stream if stream is not None else _torch_stream()
            _capi.check(s._L.agimp_get_particles_async(s._h, *a, st), s._h, "get " + self.name)
        return out

    def from_numpy(self, arr):
        if not self.writable:
            raise AttributeError("%s is computed by the substep and cannot be written" % self.name)
        a = np.ascontiguousarray(np.asarray(arr).reshape(self.shape), self.dtype)
        s = self.sim
        args = self._args(_ptr(a))
        set_args = args[:6] + [args[7]]  # set_particles has no fl_p
        _capi.check(s._L.agimp_set_particles(s._h, *set_args, AGIMP_MEM_HOST, None), s._h, "set " + self.name)

    def to_torch(self, device=None):
        import torch
        s = self.sim
        dt = torch.float32 if self.dtype == np.float32 else torch.int32
        out = torch.empty(self.shape, dtype=dt, device=device or "cuda:%d" % s.device)
        a = self._args(ctypes.c_void_p(out.data_ptr()))
        _capi.check(s._L.agimp_get_particles(s._h, *a, AGIMP_MEM_DEVICE, _torch_stream()), s._h, "get " + self.name)
        return out

    def from_torch(self, t):
        import torch
        if not self.writable:
            raise AttributeError("%s is computed by the substep and cannot be written" % self.name)
        s = self.sim
        dt = torch.float32 if self.dtype == np.float32 else torch.int32
        t = t.to(device="cuda:%d" % s.device, dtype=dt).reshape(self.shape).contiguous()
        args = self._args(ctypes.c_void_p(t.data_ptr()))
        set_args = args[:6] + [args[7]]
        _capi.check(s._L.agimp_set_particles(s._h, *set_args, AGIMP_MEM_DEVICE, _torch_stream()), s._h,
                    "set " + self.name)

    def __getitem__(self, i):
        return self.to_numpy()[i]

    def __setitem__(self, i, val):
        a = self.to_numpy()
        a[i] = val
        self.from_numpy(a)


class GridField:
    """cell_mask[l], ad_grid_m[l] or ad_grid_v[l] (adaptive_gimp.py:35-42)."""

    def __init__(self, sim, l, kind):
        self.sim, self.l, self.kind = sim, l, kind
        lsz = sim.coarsest_size << l
        self.shape = (4 * align_size(lsz // sim.leaf_size + 1, 4),) * sim.dim

    def read(self, lo=0, n=None):
        """Dense box [lo, lo+n)^dim (the library stores [-4, size+8))."""
        s = self.sim
        n = self.shape[0] if n is None else n
        shp = (n,) * s.dim
        m = np.zeros(shp, np.float32) if self.kind == "m" else None
        v = np.zeros(shp + (s.dim,), np.float32) if self.kind == "v" else None
        c = np.zeros(shp, np.int32) if self.kind == "cell" else None
        _capi.check(s._L.agimp_get_grid(s._h, self.l, lo, n, _ptr(m), _ptr(v), _ptr(c), AGIMP_MEM_HOST, None),
                    s._h, "get grid")
        return {"m": m, "v": v, "cell": c}[self.kind]

    def to_numpy(self):
        return self.read(0, self.shape[0])


class NodeMaskField:
    """node_mask on the finest lattice (adaptive_gimp.py:23-26)."""

    def __init__(self, sim):
        self.sim = sim
        self.shape = (4 * align_size(sim.finest_size // 4 + 1, 4),) * sim.dim

    def read_lattice(self):
        """node_mask over [0, finest]^dim."""
        s = self.sim
        out = np.zeros((s.finest_size + 1,) * s.dim, np.int32)
        _capi.check(s._L.agimp_get_node_mask(s._h, _ptr(out), AGIMP_MEM_HOST, None), s._h, "get node mask")
        return out

    def to_numpy(self):
        full = np.zeros(self.shape, np.int32)
        lat = self.read_lattice()
        full[tuple(slice(0, k) for k in lat.shape)] = lat
        return full


class _MapRecorder:
    """Stand-in passed to a scalar grid_initializer while it is tabulated."""

    def __init__(self, dim, level, coarsest_size):
        self.dim, self.level, self.coarsest_size = dim, level, coarsest_size
        self.finest_size = coarsest_size << (level - 1)
        self.calls = []

    def activate_cell(self, l, I):
        self.calls.append((int(l), tuple(int(e) for e in I)))


def tabulate_level_map(grid_initializer, dim, level, coarsest_size):
    """Tabulate a grid_initializer over finest cells [-H, finest+H)^dim.

    Returns (table int8, H).  Entry: returned level in the low 4 bits, bit 6
    set when the call activates nothing.
    """
    sz = coarsest_size << (level - 1)
    H = max(2, 1 << (level - 1))
    n = sz + 2 * H
    if getattr(grid_initializer, "vectorized", False):
        axes = np.meshgrid(*[np.arange(-H, sz + H)] * dim, indexing="ij")
        I = np.stack(axes, axis=-1)
        lv, act = grid_initializer(_MapRecorder(dim, level, coarsest_size), I)
        lv = np.asarray(lv, np.int64)
        act = np.asarray(act, bool)
        if lv.min() < 0 or lv.max() >= level:
            raise ValueError("grid_initializer returned a level outside [0, level)")
        return (lv | np.where(act, 0, 64)).astype(np.int8), H

    rec = _MapRecorder(dim, level, coarsest_size)
    table = np.zeros((n,) * dim, np.int8)
    for idx in np.ndindex(*table.shape):
        I = np.array([i - H for i in idx])
        rec.calls.clear()
        lv = int(grid_initializer(rec, I))
        if not 0 <= lv < level:
            raise ValueError("grid_initializer returned level %d" % lv)
        if not rec.calls:
            table[idx] = lv | 64
        elif rec.calls == [(lv, tuple(I))]:
            table[idx] = lv
        else:
            raise ValueError("grid_initializer at %s must activate nothing or the level-%d cell containing it; "
                             "it called %s" % (tuple(I), lv, rec.calls))
    return table, H


class AdaptiveGIMP:
    """Drop-in for adaptive_gimp.AdaptiveGIMP backed by libagimp.so."""

    def __init__(self, dim, level, coarsest_size, n_particles, particle_initializer, grid_initializer=None, *,
                 device=0, radius=0.5, p_mass=1.0, gravity=None, E=5e3, nu=0.2, boundary_gap=4,
                 boundary_mode="ref_slip", plasticity=None, theta_c=2.5e-2, theta_s=7.5e-3, hardening=10.0,
                 colliders=(), invalid_nodes="raw", graphs=True):
        self._L = _capi.load()
        self.dim = dim
        self.level = level
        self.coarsest_size = coarsest_size
        self.coarsest_dx = 1 / self.coarsest_size
        self.finest_size = self.coarsest_size * (2 ** (self.level - 1))
        self.boundary_gap = boundary_gap
        self.leaf_size = 4
        self.radius = radius
        self.p_mass = p_mass
        self.gravity = np.array(gravity if gravity is not None else [-100.0 if _ == 1 else 0.0 for _ in range(dim)],
                                np.float32)
        self.n_particles = n_particles
        self.E, self.nu = E, nu
        self.mu, self.la = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
        self.device = device
        self.plasticity = plasticity
        p = _capi.Params()
        self._L.agimp_default_params(ctypes.byref(p), dim, level, coarsest_size, n_particles)
        p.radius = radius
        for i in range(3):
            p.gravity[i] = float(self.gravity[i]) if i < dim else 0.0
        p.E, p.nu = E, nu
        p.boundary_gap = boundary_gap
        p.boundary_mode = {"ref_slip": 0, "sticky": 1}[boundary_mode]
        p.plasticity = {None: 0, "none": 0, "snow": 1}[plasticity]
        p.theta_c, p.theta_s, p.hardening = theta_c, theta_s, hardening
        # "raw": the reference's grid update (unactivated nodes keep raw P2G
        # momentum); "normalize": extension that divides them by their mass
        p.invalid_nodes = {"raw": 0, "normalize": 1}[invalid_nodes]
        p.n_colliders = len(colliders)
        for k, box in enumerate(colliders):
            for j in range(6):
                p.colliders[k][j] = float(box[j])
        h = ctypes.c_void_p()
        _capi.check(self._L.agimp_create(ctypes.byref(p), device, ctypes.byref(h)), None, "agimp_create")
        self._h = h
        self._params = p
        self._L.agimp_set_graphs(self._h, 1 if graphs else 0)
        d = dim
        n = n_particles
        self.x_p = ParticleField(self, "x", (n, d), np.float32)
        self.v_p = ParticleField(self, "v", (n, d), np.float32)
        self.F_p = ParticleField(self, "F", (n, d, d), np.float32)
        self.C_p = ParticleField(self, "C", (n, d, d), np.float32)
        self.m_p = ParticleField(self, "m", (n,), np.float32)
        self.g_p = ParticleField(self, "g", (n,), np.int32)
        self.fl_p = ParticleField(self, "fl", (n,), np.int32, writable=False)
        self.Jp = ParticleField(self, "Jp", (n,), np.float32)
        self.c_p = np.zeros((n, 3), np.float32)  # particle colour: host-side only (GUI data)
        self.cell_mask = [GridField(self, l, "cell") for l in range(level)]
        self.ad_grid_m = [GridField(self, l, "m") for l in range(level)]
        self.ad_grid_v = [GridField(self, l, "v") for l in range(level)]
        self.node_mask = NodeMaskField(self)
        particle_initializer(self)
        self.grid_initializer = grid_initializer
        self.static_adaptivity = grid_initializer is not None
        if self.static_adaptivity:
            # initializers that describe themselves are tabulated on the device
            # (init.py's masks by rule number, maps constant per coarsest cell);
            # any other Python callable is tabulated here
            rule = getattr(grid_initializer, "device_rule", None)
            coarse = getattr(grid_initializer, "coarse_levels", None)
            if rule is not None and (rule != 3 or level >= 3) and (rule in (1, 3) or level >= 4):
                self.set_level_map_rule(rule)
            elif coarse is not None and np.shape(coarse) == (coarsest_size,) * dim:
                self.set_coarse_level_map(coarse)
            else:
                table, H = tabulate_level_map(grid_initializer, dim, level, coarsest_size)
                self.set_level_map(table, H)

    # -- lifetime ----------------------------------------------------------
    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.agimp_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference API ------------------------------------------------------
    def substep(self, dt0, n=1, stream=None):
        """adaptive_gimp.py:323-352; asynchronous on `stream` (default: torch's current stream)."""
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_substep(self._h, float(dt0), int(n), st), self._h, "substep")

    def activate_cell(self, l, I):
        raise RuntimeError("activate_cell is only meaningful inside a grid_initializer, which is tabulated at "
                           "construction")

    def set_level_map(self, table, halo):
        t = np.ascontiguousarray(table, np.int8)
        _capi.check(self._L.agimp_set_level_map(self._h, _ptr(t), int(halo), AGIMP_MEM_HOST, None), self._h,
                    "set level map")
        self.static_adaptivity = True

    def set_level_map_rule(self, rule, stream=None):
        """initialize_mask<rule> of init.py:34-98, tabulated on the device."""
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_set_level_map_rule(self._h, int(rule), st), self._h, "level map rule")
        self.static_adaptivity = True

    def set_coarse_level_map(self, coarse_levels, stream=None):
        """A level map constant per coarsest cell (coarsest_size^dim levels),
        expanded to the finest cells on the device."""
        c = np.ascontiguousarray(coarse_levels, np.int8)
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_set_coarse_level_map(self._h, _ptr(c), AGIMP_MEM_HOST, st), self._h,
                    "coarse level map")
        self.static_adaptivity = True

    def get_level_map(self):
        """The selected level map: (table int8 [(finest + 2 halo)]*dim, halo)."""
        H = ctypes.c_int32()
        _capi.check(self._L.agimp_get_level_map(self._h, None, ctypes.byref(H), AGIMP_MEM_HOST, None), self._h,
                    "level map")
        n = self.finest_size + 2 * H.value
        t = np.empty((n,) * self.dim, np.int8)
        _capi.check(self._L.agimp_get_level_map(self._h, _ptr(t), None, AGIMP_MEM_HOST, None), self._h, "level map")
        return t, H.value

    def clear_level_map(self):
        _capi.check(self._L.agimp_clear_level_map(self._h), self._h, "clear level map")
        self.static_adaptivity = False

    def refine_levels(self, band=3, stream=None):
        """Extension: recompute g_p from the free surface (see include/agimp.h)."""
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_refine_levels(self._h, int(band), st), self._h, "refine levels")

    def set_particles(self, x=None, v=None, F=None, C=None, m=None, g=None, Jp=None):
        """Upload several particle fields in one call (host arrays or CUDA tensors)."""
        vals = [x, v, F, C, m, g, Jp]
        dtypes = [np.float32] * 5 + [np.int32, np.float32]
        try:
            import torch
            is_t = [isinstance(a, torch.Tensor) for a in vals if a is not None]
        except ImportError:
            is_t = []
        if is_t and all(is_t):
            args = [ctypes.c_void_p(a.contiguous().data_ptr()) if a is not None else None for a in vals]
            _capi.check(self._L.agimp_set_particles(self._h, *args, AGIMP_MEM_DEVICE, _torch_stream()), self._h,
                        "set particles")
            return
        arrs = [np.ascontiguousarray(a, dt) if a is not None else None for a, dt in zip(vals, dtypes)]
        _capi.check(self._L.agimp_set_particles(self._h, *[_ptr(a) for a in arrs], AGIMP_MEM_HOST, None), self._h,
                    "set particles")

    def errors(self, clear=True):
        bits = ctypes.c_uint32()
        _capi.check(self._L.agimp_errors(self._h, ctypes.byref(bits), 1 if clear else 0), self._h, "errors")
        return bits.value

    def bin_keys(self):
        """The bins of the last substep, one uint64 key per particle (the
        reference's pid[l] lists, adaptive_gimp.py:208-216): level in bits
        60-63, floor(base / 4) + 1 per axis in 20-bit fields (first axis
        highest), all ones for particles without a level."""
        out = np.zeros(self.n_particles, np.uint64)
        _capi.check(self._L.agimp_get_bins(self._h, _ptr(out), AGIMP_MEM_HOST, None), self._h, "get bins")
        return out

    def stats(self):
        st = _capi.Stats()
        _capi.check(self._L.agimp_get_stats(self._h, ctypes.byref(st)), self._h, "stats")
        return dict(active_blocks=list(st.active_blocks)[: self.level], n_binned=st.n_binned, n_chunks=st.n_chunks,
                    substeps=st.substeps, n_surrogate=st.n_surrogate, n_fallback=st.n_fallback)

    # -- surrogate return map (extension) ---------------------------------------
    def set_surrogate(self, mlp, xmax=None, tol=0.02):
        """Use `mlp` (agimp.surrogate.MLP) for the snow return map; None switches it off."""
        if mlp is None:
            _capi.check(self._L.agimp_set_surrogate(self._h, None, None, 0.0), self._h, "set surrogate")
            return
        xm = (ctypes.c_float * 7)(*[float(v) for v in xmax])
        _capi.check(self._L.agimp_set_surrogate(self._h, mlp._h, xm, float(tol)), self._h, "set surrogate")
        self._surrogate = mlp

    def set_recorder(self, X=None, T=None, stride=1):
        """Record (features, projected state) pairs into CUDA tensors X [cap, 7], T [cap, 4]."""
        if X is None:
            _capi.check(self._L.agimp_set_recorder(self._h, None, None, 0, 1), self._h, "set recorder")
            return
        _capi.check(self._L.agimp_set_recorder(self._h, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(T.data_ptr()),
                                               X.shape[0], int(stride)), self._h, "set recorder")
        self._rec = (X, T)

    def recorded(self, reset=False):
        n = ctypes.c_int64()
        _capi.check(self._L.agimp_recorded(self._h, ctypes.byref(n), 1 if reset else 0), self._h, "recorded")
        return n.value

    # -- launch tuning -----------------------------------------------------------
    @property
    def tuning(self):
        t = _capi.Tuning()
        _capi.check(self._L.agimp_get_tuning(self._h, ctypes.byref(t)), self._h, "get tuning")
        return t.as_dict()

    def set_tuning(self, chunk=256, ctas_per_sm=8):
        """P2G work-item size (64, 128, 256, 512) and grid-stride CTAs per SM."""
        t = _capi.Tuning(int(chunk), int(ctas_per_sm), 0.0)
        _capi.check(self._L.agimp_set_tuning(self._h, ctypes.byref(t)), self._h, "set tuning")

    def autotune(self, dt0, trials=5, stream=None):
        """Time every launch choice on the current state (restored afterwards),
        keep the fastest and return it."""
        t = _capi.Tuning()
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_autotune(self._h, float(dt0), int(trials), ctypes.byref(t), st), self._h,
                    "autotune")
        return t.as_dict()

    def profile_substep(self, dt0, stream=None):
        """One substep with per-phase CUDA-event timing; returns {phase: ms}."""
        ms = (ctypes.c_float * len(_capi.PHASES))()
        st = stream if stream is not None else _torch_stream()
        _capi.check(self._L.agimp_profile_substep(self._h, float(dt0), ms, len(ms), st), self._h, "profile")
        return dict(zip(_capi.PHASES, list(ms)))

    def kernels_per_substep(self):
        return int(self._L.agimp_kernels_per_substep(self._h))

    # -- predicates (adaptive_gimp.py:126-140), vectorised over I[..., dim] --
    def _map(self, l, I):
        return np.asarray(I) * (2 ** (self.level - 1 - l))

    def _nm(self, l, I, nm=None):
        nm = self.node_mask.read_lattice() if nm is None else nm
        P = self._map(l, I)
        return nm[tuple(np.moveaxis(P, -1, 0))]

    def is_valid(self, l, I, nm=None):
        return self._nm(l, I, nm) > 0

    def is_activated(self, l, I, nm=None):
        return (self._nm(l, I, nm) & (ACTIVATED | T_JUNCTION)) == ACTIVATED

    def is_T_junction(self, l, I, nm=None):
        return (self._nm(l, I, nm) & T_JUNCTION) == T_JUNCTION

    def is_ghost(self, l, I, nm=None):
        return (self._nm(l, I, nm) & (ACTIVATED | GHOST | T_JUNCTION)) == GHOST
