"""ctypes binding of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: the oracle is the parity checker and the timed CPU
baseline.  Nothing on the product path imports this module.

Array conventions follow the reference's field readback (Taichi ``to_numpy``):
particle vectors are ``[N, d]``, matrices ``[N, d, d]`` (row-major), grid
readback is a dense box of node/cell indices ``[lo, lo + n)`` per axis with the
first axis slowest (the reference's ``ti.ij`` / ``ti.ijk`` ordering).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile next to this file."""
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("level", ctypes.c_int32), ("coarsest_size", ctypes.c_int32),
        ("boundary_gap", ctypes.c_int32), ("boundary_mode", ctypes.c_int32), ("plasticity", ctypes.c_int32),
        ("radius", ctypes.c_double), ("gravity", ctypes.c_double * 3), ("E", ctypes.c_double), ("nu", ctypes.c_double),
        ("theta_c", ctypes.c_double), ("theta_s", ctypes.c_double), ("hardening", ctypes.c_double),
        ("n_colliders", ctypes.c_int32), ("colliders", (ctypes.c_double * 6) * 4), ("invalid_nodes", ctypes.c_int32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int32, ctypes.c_int64]
        L.orc_destroy.argtypes = [P]
        L.orc_set_particles.argtypes = [P, dp, dp, dp, dp, dp, ip, dp]
        L.orc_set_g.argtypes = [P, ip]
        L.orc_set_level_map.argtypes = [P, ctypes.POINTER(ctypes.c_int8), ctypes.c_int32]
        L.orc_substep.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.c_int32]
        L.orc_refine_levels.argtypes = [P, ctypes.c_int32]
        L.orc_get_particles.argtypes = [P, dp, dp, dp, dp, dp, ip, ip, dp]
        L.orc_get_grid.argtypes = [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, dp, dp, ip]
        L.orc_get_node_mask.argtypes = [P, ip]
        L.orc_errors.restype = ctypes.c_uint32
        L.orc_errors.argtypes = [P]
        L.orc_clear_errors.argtypes = [P]
        L.orc_weight_stencil.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, dp, dp]
        L.orc_stress.argtypes = [ctypes.c_int32, ctypes.c_int32, dp, ctypes.c_double, ctypes.c_double, dp]
        L.orc_svd.argtypes = [ctypes.c_int32, dp, dp, dp, dp]
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


REF_DEFAULTS = dict(radius=0.5, gravity=(0.0, -100.0, 0.0), E=5e3, nu=0.2, boundary_gap=4, boundary_mode=0,
                    plasticity=0, theta_c=2.5e-2, theta_s=7.5e-3, hardening=10.0, colliders=(),
                    invalid_nodes=0)


class Oracle:
    """One restated simulator instance (f32 or f64)."""

    def __init__(self, dim, level, coarsest_size, n_particles, f64=False, **kw):
        cfg = dict(REF_DEFAULTS)
        cfg.update(kw)
        p = OrcParams()
        p.dim, p.level, p.coarsest_size = dim, level, coarsest_size
        p.boundary_gap, p.boundary_mode, p.plasticity = cfg["boundary_gap"], cfg["boundary_mode"], cfg["plasticity"]
        p.radius = cfg["radius"]
        g = list(cfg["gravity"]) + [0.0] * 3
        for i in range(3):
            p.gravity[i] = g[i]
        p.E, p.nu = cfg["E"], cfg["nu"]
        p.theta_c, p.theta_s, p.hardening = cfg["theta_c"], cfg["theta_s"], cfg["hardening"]
        cols = list(cfg["colliders"])
        p.invalid_nodes = int(cfg["invalid_nodes"])
        p.n_colliders = len(cols)
        for k, c in enumerate(cols):
            for j in range(6):
                p.colliders[k][j] = c[j]
        self.dim, self.level, self.coarsest_size, self.n = dim, level, coarsest_size, n_particles
        self.finest_size = coarsest_size << (level - 1)
        self.f64 = f64
        self._h = lib().orc_create(ctypes.byref(p), 1 if f64 else 0, n_particles)
        if not self._h:
            raise ValueError("invalid oracle parameters")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    def set_particles(self, x, v, F, C, m, g, Jp=None):
        n, d = self.n, self.dim
        x, v = _d(x).reshape(n, d), _d(v).reshape(n, d)
        F, C = _d(F).reshape(n, d, d), _d(C).reshape(n, d, d)
        m = _d(m).reshape(n)
        g = np.ascontiguousarray(g, dtype=np.int32).reshape(n)
        Jp = None if Jp is None else _d(Jp).reshape(n)
        lib().orc_set_particles(self._h, _p(x), _p(v), _p(F), _p(C), _p(m), _p(g, ctypes.c_int32), _p(Jp))

    def set_g(self, g):
        g = np.ascontiguousarray(g, dtype=np.int32).reshape(self.n)
        lib().orc_set_g(self._h, _p(g, ctypes.c_int32))

    def set_level_map(self, table, halo):
        t = np.ascontiguousarray(table, dtype=np.int8)
        lib().orc_set_level_map(self._h, _p(t, ctypes.c_int8), int(halo))

    def substep(self, dt, n=1, nthreads=0):
        lib().orc_substep(self._h, float(dt), int(n), int(nthreads))

    def refine_levels(self, band=3):
        lib().orc_refine_levels(self._h, int(band))

    def particles(self):
        n, d = self.n, self.dim
        out = dict(x=np.zeros((n, d)), v=np.zeros((n, d)), F=np.zeros((n, d, d)), C=np.zeros((n, d, d)),
                   m=np.zeros(n), g=np.zeros(n, np.int32), fl=np.zeros(n, np.int32), Jp=np.zeros(n))
        lib().orc_get_particles(self._h, _p(out["x"]), _p(out["v"]), _p(out["F"]), _p(out["C"]), _p(out["m"]),
                                _p(out["g"], ctypes.c_int32), _p(out["fl"], ctypes.c_int32), _p(out["Jp"]))
        return out

    def grid(self, l, lo=0, n=None):
        """(m, v, cell_mask) of level l over indices [lo, lo+n) per axis."""
        if n is None:
            n = (self.coarsest_size << l) + 2
        shp = (n,) * self.dim
        m = np.zeros(shp)
        v = np.zeros(shp + (self.dim,))
        c = np.zeros(shp, np.int32)
        lib().orc_get_grid(self._h, int(l), int(lo), int(n), _p(m), _p(v), _p(c, ctypes.c_int32))
        return m, v, c

    def node_mask(self):
        n = self.finest_size + 1
        out = np.zeros((n,) * self.dim, np.int32)
        lib().orc_get_node_mask(self._h, _p(out, ctypes.c_int32))
        return out

    def errors(self):
        return int(lib().orc_errors(self._h))

    def clear_errors(self):
        lib().orc_clear_errors(self._h)


def weight_stencil(tc, radius=0.5, f64=True):
    tc = _d(tc)
    d = tc.shape[0]
    out = np.zeros((3 ** d, d + 1))
    lib().orc_weight_stencil(d, 1 if f64 else 0, float(radius), _p(tc), _p(out))
    return out


def stress(F, mu, la, f64=True):
    F = _d(F)
    d = F.shape[0]
    out = np.zeros((d, d))
    lib().orc_stress(d, 1 if f64 else 0, _p(F), float(mu), float(la), _p(out))
    return out


def svd(A):
    A = _d(A)
    d = A.shape[0]
    U, S, V = np.zeros((d, d)), np.zeros(d), np.zeros((d, d))
    lib().orc_svd(d, _p(A), _p(U), _p(S), _p(V))
    return U, S, V
