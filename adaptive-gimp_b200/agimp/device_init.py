"""Scene initialisers that run on the GPU (agimp_lattice_* / agimp_random_fill).

The reference fills its particle fields with Taichi kernels passed to
``AdaptiveGIMP`` as ``particle_initializer`` (init.py:3-32, run_3d.py:14-32).
The functions here build the same kind of initializer for this library: the
particle state is generated in device memory from a few shapes and a seed, so a
scene of millions of particles needs no host arrays and no upload.

* ``box`` / ``sphere``: shapes of a jittered sub-lattice (the benchmark
  scenes: ``per_axis`` points per finest cell and axis, each moved by up to
  half a sub-spacing).  ``lattice_count`` gives the particle count (needed to
  create the simulator), ``lattice_initializer`` the initializer, and
  ``lattice_simulator`` both in one call.
* ``random_box`` and ``reference_boxes_2d`` / ``reference_boxes_3d``: uniform
  particles in boxes with init.py's level bands (``random_initializer``).

Random numbers come from Philox4x32-10 keyed by the seed; the same seed gives
the same particles on any GPU and launch configuration.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi


def _shape(kind, level, velocity, mass, lo=(0.0,) * 3, hi=(0.0,) * 3, centre=(0.0,) * 3, radius=0.0):
    s = _capi.Shape()
    s.kind = kind
    s.level = int(level)
    for d in range(3):
        s.lo[d] = float(lo[d]) if d < len(lo) else 0.0
        s.hi[d] = float(hi[d]) if d < len(hi) else 0.0
        s.centre[d] = float(centre[d]) if d < len(centre) else 0.0
        s.velocity[d] = float(velocity[d]) if d < len(velocity) else 0.0
    s.radius = float(radius)
    s.mass = float(mass)
    return s


def box(lo, hi, level, velocity=(0.0, 0.0, 0.0), mass=1.0):
    """Lattice points with lo <= x < hi (per axis, after the jitter)."""
    return _shape(_capi.SHAPE_BOX, level, velocity, mass, lo=lo, hi=hi)


def sphere(centre, radius, level, velocity=(0.0, 0.0, 0.0), mass=1.0):
    """Lattice points with |x - centre|^2 < radius^2 (after the jitter)."""
    return _shape(_capi.SHAPE_SPHERE, level, velocity, mass, centre=centre, radius=radius)


def _shape_array(shapes):
    arr = (_capi.Shape * max(1, len(shapes)))()
    for i, s in enumerate(shapes):
        arr[i] = s
    return arr


def lattice_count(dim, finest, shapes, seed=0, per_axis=2, jitter=True, device=0):
    """Number of particles the shapes hold (computed on the GPU)."""
    L = _capi.load()
    n = ctypes.c_int64()
    _capi.check(L.agimp_lattice_count(int(dim), int(finest), int(per_axis), 1 if jitter else 0, int(seed),
                                      _shape_array(shapes), len(shapes), ctypes.byref(n), int(device)),
                None, "lattice count")
    return int(n.value)


def lattice_initializer(shapes, seed=0, per_axis=2, jitter=True):
    """particle_initializer(sim) that fills the simulator's particles on the GPU."""
    arr = _shape_array(shapes)

    def init(sim):
        _capi.check(sim._L.agimp_lattice_fill(sim._h, int(per_axis), 1 if jitter else 0, int(seed), arr, len(shapes),
                                              None), sim._h, "lattice fill")

    return init


def lattice_simulator(dim, level, coarsest_size, shapes, seed=0, per_axis=2, jitter=True, grid_initializer=None,
                      **kw):
    """An AdaptiveGIMP whose particles are generated on the GPU."""
    from .simulator import AdaptiveGIMP
    finest = coarsest_size << (level - 1)
    n = lattice_count(dim, finest, shapes, seed, per_axis, jitter, kw.get("device", 0))
    return AdaptiveGIMP(dim, level, coarsest_size, n, lattice_initializer(shapes, seed, per_axis, jitter),
                        grid_initializer, **kw)


def random_box(count, lo, size, level, velocity=(0.0, 0.0, 0.0), mass=1.0, bands=()):
    """`count` particles at x = u * size + lo (u uniform in [0, 1)^dim, float
    arithmetic); g_p is the level of the first band (lo_u, hi_u, level) with
    lo_u <= u <= hi_u on every axis, else `level`."""
    b = _capi.RandomBox()
    b.count = int(count)
    for d in range(3):
        b.lo[d] = float(lo[d]) if d < len(lo) else 0.0
        b.size[d] = float(size[d]) if d < len(size) else 0.0
        b.velocity[d] = float(velocity[d]) if d < len(velocity) else 0.0
    b.mass = float(mass)
    if len(bands) > 4:
        raise ValueError("at most 4 bands")
    b.n_bands = len(bands)
    for k, (blo, bhi, blev) in enumerate(bands):
        b.band_lo[k], b.band_hi[k], b.band_level[k] = float(blo), float(bhi), int(blev)
    b.level = int(level)
    return b


def reference_boxes_2d(n_particles, case=0, p_mass=1.0):
    """init.py:3-32 (initialize_particle): the first n // 2 particles in
    [0.2, 0.6] x [0.1, 0.5] moving up at 20, the rest in [0.4, 0.8] x
    [0.55, 0.95] moving down; case 0 puts g_p on levels 0..3 by the position
    inside the box (bands 0.2-0.8, 0.1-0.9, 0.03-0.97), any other case -1."""
    half = n_particles // 2
    bands = ((0.2, 0.8, 0), (0.1, 0.9, 1), (0.03, 0.97, 2)) if case == 0 else ()
    lev = 3 if case == 0 else -1
    return [random_box(half, (0.2, 0.1), (0.4, 0.4), lev, (0.0, 20.0), p_mass, bands),
            random_box(n_particles - half, (0.4, 0.55), (0.4, 0.4), lev, (0.0, -20.0), p_mass, bands)]


def reference_boxes_3d(n_particles, p_mass=1.0, first=25000):
    """run_3d.py:14-32 (init_p): particles with i // 25000 == 0 in
    [0.2, 0.5] x [0.1, 0.4] x [0.2, 0.5] moving up at 20, the rest 0.4 higher
    moving down; g_p 0 / 1 / 2 by the bands 0.05-0.95 and 0.01-0.99."""
    a = min(first, n_particles)
    bands = ((0.05, 0.95, 0), (0.01, 0.99, 1))
    return [random_box(a, (0.2, 0.1, 0.2), (0.3, 0.3, 0.3), 2, (0.0, 20.0, 0.0), p_mass, bands),
            random_box(n_particles - a, (0.2, 0.5, 0.2), (0.3, 0.3, 0.3), 2, (0.0, -20.0, 0.0), p_mass, bands)]


def random_initializer(boxes, seed=0):
    """particle_initializer(sim) drawing the boxes' particles on the GPU."""
    arr = (_capi.RandomBox * len(boxes))(*boxes)

    def init(sim):
        _capi.check(sim._L.agimp_random_fill(sim._h, int(seed), arr, len(boxes), None), sim._h, "random fill")

    return init


def band_colours(g, case=0):
    """init.py:19-32's particle colours from g_p (host side: GUI data)."""
    table = np.array([[0.93, 0.33, 0.23], [0.95, 0.80, 0.43], [0.80, 0.49, 0.80], [0.34, 0.51, 0.44]], np.float32)
    g = np.asarray(g)
    if case != 0:
        return np.tile(table[0], (len(g), 1))
    return table[np.clip(g, 0, 3)]
