"""Scene generators and level maps.

* ``initialize_mask1`` .. ``initialize_mask5``: the reference's static level
  maps (init.py:34-98) restated as vectorised grid initializers: given finest
  cell indices ``I[..., dim]`` they return ``(level, activate)``.
* ``make_config(k)``: seeded synthetic scenes with the shapes, sizes and
  materials of the benchmark configurations (numpy PCG64, seed 0 by default).
  Particles fill boxes / spheres on a sub-lattice of the finest cells (2 per
  axis per cell: 4 per cell in 2D, 8 in 3D) with uniform jitter of +-0.5
  sub-spacing.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def _vec(fn):
    fn.vectorized = True
    return fn


def _inner(I, sz):
    return np.all((I >= 8) & (I < sz - 8), axis=-1)


@_vec
def initialize_mask1(sim, I):
    """init.py:34-37: every cell at the finest level."""
    lv = np.full(I.shape[:-1], sim.level - 1)
    return lv, np.ones(lv.shape, bool)


@_vec
def initialize_mask2(sim, I):
    """init.py:39-49: level 0 in the left half (8-cell margin), else level 3."""
    sz = sim.finest_size
    left = (I[..., 0] < sz / 2) & _inner(I, sz)
    return np.where(left, 0, 3), np.ones(left.shape, bool)


@_vec
def initialize_mask3(sim, I):
    """init.py:51-64: levels 0 / 1 / 2 in vertical bands."""
    sz = sim.finest_size
    inner = _inner(I, sz)
    lv = np.where((I[..., 0] < sz / 4) & inner, 0, np.where((I[..., 0] < sz / 2) & inner, 1, 2))
    return lv, np.ones(lv.shape, bool)


@_vec
def initialize_mask4(sim, I):
    """init.py:66-80: levels 1 / 2 in the left half, 3 elsewhere in range;
    out-of-range cells return 3 without activating."""
    sz = sim.finest_size
    left = (I[..., 0] < sz / 2) & _inner(I, sz)
    inr = np.all((I >= 0) & (I < sz), axis=-1)
    lv = np.where(left, np.where(I[..., 1] < sz / 2, 1, 2), 3)
    return lv, left | inr


@_vec
def initialize_mask5(sim, I):
    """init.py:82-98: levels 0 / 1 / 2 in the left half, 3 elsewhere in range."""
    sz = sim.finest_size
    left = (I[..., 0] < sz / 2) & _inner(I, sz)
    inr = np.all((I >= 0) & (I < sz), axis=-1)
    lv = np.where(left, np.where(I[..., 1] < sz / 4, 0, np.where(I[..., 1] < sz / 2, 1, 2)), 3)
    return lv, left | inr


REFERENCE_MASKS = {1: initialize_mask1, 2: initialize_mask2, 3: initialize_mask3, 4: initialize_mask4,
                   5: initialize_mask5}
for _k, _f in REFERENCE_MASKS.items():
    _f.device_rule = _k  # the library tabulates these on the device (agimp_set_level_map_rule)


def band_level_map(boxes, dim, level, coarsest_size, near=2, mid=4, floor_y=0.25):
    """Static level map aligned to coarsest cells: the finest level within
    `near` coarsest cells (Chebyshev) of any box or below `floor_y`, level
    level-2 within `mid` cells, level 0 elsewhere; halo cells return level-1
    without activating."""
    nc = coarsest_size
    cov = np.zeros((nc,) * dim, bool)
    for lo, hi in boxes:
        sl = tuple(slice(int(np.floor(a * nc)), int(np.ceil(b * nc))) for a, b in zip(lo, hi))
        cov[sl] = True
    # Chebyshev distance <= k from a covered cell <=> inside a (2k+1)^dim box
    from scipy.ndimage import maximum_filter
    within_near = maximum_filter(cov, size=2 * near + 1, mode="constant", cval=False)
    within_mid = maximum_filter(cov, size=2 * mid + 1, mode="constant", cval=False)
    y_center = (np.arange(nc) + 0.5) / nc
    ylow = np.broadcast_to(y_center.reshape((1, nc) + (1,) * (dim - 2)), cov.shape) < floor_y
    coarse_lv = np.where(within_near | ylow, level - 1, np.where(within_mid, max(level - 2, 0), 0))
    sz = nc << (level - 1)
    s = level - 1

    @_vec
    def grid_initializer(sim, I):
        inr = np.all((I >= 0) & (I < sz), axis=-1)
        C = np.clip(I >> s, 0, nc - 1)
        lv = coarse_lv[tuple(np.moveaxis(C, -1, 0))]
        return np.where(inr, lv, level - 1), inr

    grid_initializer.coarse_levels = coarse_lv.astype(np.int8)  # expanded on the device
    return grid_initializer


# ---------------------------------------------------------------------------
def fill_lattice(rng, dim, finest, inside, lo, hi, per_axis=2, jitter=True):
    """Points on the sub-lattice (per_axis per finest cell and axis) inside the
    region lo..hi that satisfy inside(points)."""
    h = 1.0 / (finest * per_axis)
    axes = [np.arange(np.floor(a / h), np.ceil(b / h)) * h + 0.5 * h for a, b in zip(lo, hi)]
    mesh = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, dim)
    if jitter:
        mesh = mesh + rng.uniform(-0.5 * h, 0.5 * h, mesh.shape)
    return mesh[inside(mesh)].astype(np.float32)


def box_region(lo, hi):
    lo, hi = np.asarray(lo), np.asarray(hi)
    return lambda p: np.all((p >= lo) & (p < hi), axis=1), lo, hi


def sphere_region(c, r):
    c = np.asarray(c)
    return lambda p: ((p - c) ** 2).sum(1) < r * r, c - r, c + r


@dataclass
class Scene:
    name: str
    dim: int
    level: int
    coarsest: int
    x: np.ndarray
    v: np.ndarray
    g: np.ndarray
    m: np.ndarray
    dt: float
    steps: int
    sim_kwargs: dict = field(default_factory=dict)
    grid_initializer: object = None
    refine_every: int = 0
    refine_band: int = 3
    description: str = ""

    @property
    def n(self):
        return len(self.x)

    def build(self, **over):
        """Construct an AdaptiveGIMP for this scene."""
        from .simulator import AdaptiveGIMP
        kw = dict(self.sim_kwargs)
        kw.update(over)
        d = self.dim
        n = self.n
        F = np.tile(np.eye(d, dtype=np.float32), (n, 1, 1))

        def pinit(sim):
            sim.set_particles(x=self.x, v=self.v, F=F, C=np.zeros((n, d, d), np.float32), m=self.m, g=self.g,
                              Jp=np.ones(n, np.float32))

        return AdaptiveGIMP(d, self.level, self.coarsest, n, pinit, self.grid_initializer, **kw)


# Units.  The reference's P2G stress term carries no particle volume
# (adaptive_gimp.py:240, i.e. V_p = 1) and its particle mass is p_mass = 1
# (adaptive_gimp.py:49): the density is 1 and only E/rho enters the dynamics.
# The scenes keep that convention (m_p = 1) and pass E/rho as the modulus, so
# the wave speed sqrt(E/rho) is the configuration's.  The configurations'
# (E, dt) with rho = 1 violate the explicit CFL limit (sqrt(E/rho) dt/dx > 1),
# so each uses a density that keeps the CFL number near 0.3: 100 for config 1,
# 400 (snow, Stomakhin et al. 2013) for configs 3 and 5, 1000 for config 2.
# Scaling the mass instead would break the reference's scheme: invalid odd
# nodes keep raw P2G momentum through G2P (adaptive_gimp.py:281 converts only
# activated nodes), which stays of the order of a velocity only when m_p = 1.
RHO = {1: 100.0, 2: 1000.0, 3: 400.0, 5: 400.0}
#
# Grid update of the dynamic scenes.  The refinement rule puts the interior of
# a body on coarse levels.  There, a particle's 3^d stencil reaches nodes of
# edge- and corner-adjacent cells that the reference marks neither activated,
# ghost nor T-junction (ghost marking covers face neighbours only,
# adaptive_gimp.py:159-181), and the reference's grid update leaves their P2G
# momentum undivided (adaptive_gimp.py:280).  On a coarse level that momentum
# sums hundreds of particles, so G2P accelerates them: the 3D scenes blow up
# within ten substeps.  The dynamic scenes therefore use invalid_nodes =
# "normalize" (those nodes are divided by their mass); the parity tests cover
# both forms.


def _unit_mass(n):
    return np.ones(n, np.float32)


def make_config(k, seed=0, scale=1.0):
    """Benchmark configurations 1..5 (scale < 1 shrinks the bodies for tests)."""
    rng = np.random.default_rng(seed)
    if k == 1:
        L, c = 3, 64
        fin = c << (L - 1)
        boxes = [((0.3 - 0.1 * scale, 0.5 - 0.1 * scale), (0.3 + 0.1 * scale, 0.5 + 0.1 * scale)),
                 ((0.6 - 0.1 * scale, 0.7 - 0.1 * scale), (0.6 + 0.1 * scale, 0.7 + 0.1 * scale))]
        xs = [fill_lattice(rng, 2, fin, *box_region(lo, hi)) for lo, hi in boxes]
        x = np.concatenate(xs)
        n = len(x)
        return Scene("config1_2d_static", 2, L, c, x, np.zeros((n, 2), np.float32), np.full(n, L - 1, np.int32),
                     _unit_mass(n), 1e-4, 1000,
                     dict(E=1e4 / RHO[1], nu=0.2, gravity=(0.0, -9.8), boundary_mode="sticky"),
                     grid_initializer=band_level_map(boxes, 2, L, c),
                     description="2D static 3-level quadtree 64^2..256^2, two elastic boxes 0.2x0.2, 4 ppc, E=1e4 rho=100")
    if k == 2:
        L, c = 4, 64
        fin = c << (L - 1)
        xs, vs = [], []
        for _ in range(3):
            side = rng.uniform(0.1, 0.25, 2) * scale
            lo = rng.uniform(0.1, 0.9 - side)
            pts = fill_lattice(rng, 2, fin, *box_region(lo, lo + side))
            xs.append(pts)
            vs.append(np.tile(rng.uniform(-1, 1, 2).astype(np.float32), (len(pts), 1)))
        x, v = np.concatenate(xs), np.concatenate(vs)
        n = len(x)
        return Scene("config2_2d_dynamic", 2, L, c, x, v, np.full(n, L - 1, np.int32),
                     _unit_mass(n), 5e-5, 2000,
                     dict(E=1.4e5 / RHO[2], nu=0.2, gravity=(0.0, -9.8), boundary_mode="sticky", plasticity="snow",
                          theta_c=2.5e-2, theta_s=7.5e-3, hardening=10.0, invalid_nodes="normalize"),
                     refine_every=10, refine_band=3,
                     description="2D dynamic 4 levels 64^2..512^2, 3 random snow boxes, 4 ppc, E=1.4e5 rho=1000, re-refined every 10")
    if k == 3:
        L, c = 3, 64
        fin = c << (L - 1)
        r = 0.15 * scale
        x = fill_lattice(rng, 3, fin, *sphere_region((0.5, 0.6, 0.5), r))
        n = len(x)
        v = np.tile(np.array([0.0, -3.0, 0.0], np.float32), (n, 1))
        slab = (0.3, 0.2, 0.3, 0.7, 0.3, 0.7)
        return Scene("config3_3d_dynamic", 3, L, c, x, v, np.full(n, L - 1, np.int32),
                     _unit_mass(n), 5e-5, 1000,
                     dict(E=1e5 / RHO[3], nu=0.25, gravity=(0.0, -9.8, 0.0), boundary_mode="sticky", plasticity="snow",
                          theta_c=2.5e-2, theta_s=7.5e-3, hardening=10.0, colliders=(slab,),
                          invalid_nodes="normalize"),
                     refine_every=10, refine_band=3,
                     description="3D dynamic 3 levels 64^3..256^3, snow sphere r=0.15 at y=0.6 moving down at 3 "
                                 "onto a 0.4x0.1x0.4 static slab collider, 8 ppc, E=1e5 rho=400, re-refined every 10")
    if k == 5:
        L, c = 4, 64
        fin = c << (L - 1)
        r = 0.12 * scale
        a = fill_lattice(rng, 3, fin, *sphere_region((0.35, 0.5, 0.5), r))
        b = fill_lattice(rng, 3, fin, *sphere_region((0.65, 0.5, 0.5), r))
        x = np.concatenate([a, b])
        v = np.concatenate([np.tile(np.array([2.0, 0, 0], np.float32), (len(a), 1)),
                            np.tile(np.array([-2.0, 0, 0], np.float32), (len(b), 1))])
        n = len(x)
        return Scene("config5_3d_two_spheres", 3, L, c, x, v, np.full(n, L - 1, np.int32),
                     _unit_mass(n), 3e-5, 1000,
                     dict(E=1.4e5 / RHO[5], nu=0.2, gravity=(0.0, -9.8, 0.0), boundary_mode="sticky", plasticity="snow",
                          invalid_nodes="normalize"),
                     refine_every=10, refine_band=3,
                     description="3D 4 levels 64^3..512^3, two colliding snow spheres r=0.12 at +-2, E=1.4e5 rho=400")
    if k == 4:
        raise ValueError("config 4 is a batch of scenes: use make_batch_config()")
    raise ValueError("unknown config %r" % k)


def _place_boxes(rng, sides, tries=200):
    """Non-overlapping axis-aligned 2D boxes with the given (w, h) sides inside
    [0.1, 0.9]^2 (rejection sampling; later boxes shrink if they do not fit)."""
    placed = []
    for w, h in sides:
        for t in range(tries):
            f = 1.0 if t < tries // 2 else 0.7
            ww, hh = w * f, h * f
            lo = rng.uniform([0.1, 0.1], [0.9 - ww, 0.9 - hh])
            hi = lo + [ww, hh]
            if all(np.any(hi <= a) or np.any(lo >= b) for a, b in placed):
                placed.append((lo, hi))
                break
    return placed


SNOW_BATCH = dict(E=1.4e5 / RHO[2], nu=0.2, gravity=(0.0, -9.8), boundary_mode="sticky", plasticity="snow",
                  theta_c=2.5e-2, theta_s=7.5e-3, hardening=10.0)


def make_batch_config(seed=0, n_scenes=256, scale=1.0, device=False, material="elastic"):
    """Config 4: independent 2D scenes for one batch.  Each scene draws its
    level count from {2, 3, 4}, its finest resolution from {256, 512}, 1-3
    boxes and a particle count from a lognormal clipped to [2k, 60k] (times
    `scale`); the boxes share that count at 4 particles per finest cell.
    Material, time step and level maps are config 1's (elastic, E=1e4 with
    rho=100, sticky walls, dt=1e-4, static map: the finest level within 2
    coarsest cells of a box or below y = 0.25).  material="snow" keeps the
    scenes and gives them config 2's snow material and time step (5e-5), with
    each box thrown at a velocity drawn uniformly from [-2, 2]^2 (a generator
    of its own, so the scenes' shapes are the elastic batch's)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        L = int(rng.integers(2, 5))
        fin = int(rng.choice([256, 512]))
        c = fin >> (L - 1)
        nbox = int(rng.integers(1, 4))
        target = float(np.clip(rng.lognormal(np.log(12000.0), 0.8), 2000, 60000)) * scale
        area = target / (4.0 * fin * fin)  # 4 particles per finest cell
        shares = rng.dirichlet(np.ones(nbox)) * area
        sides = []
        for a in shares:
            r = rng.uniform(0.5, 2.0)
            w = float(np.sqrt(a * r))
            sides.append((min(w, 0.7), min(a / w, 0.7)))
        boxes = _place_boxes(rng, sides)
        if device:
            from . import device_init as di
            out.append(DeviceScene(
                "config4_scene%03d" % i, 2, L, c, [di.box(lo, hi, L - 1) for lo, hi in boxes],
                seed * 100003 + i, 1e-4, 1000, dict(E=1e4 / RHO[1], nu=0.2, gravity=(0.0, -9.8), boundary_mode="sticky"),
                grid_initializer=band_level_map([(tuple(lo), tuple(hi)) for lo, hi in boxes], 2, L, c),
                description="%d levels %d^2..%d^2, %d boxes" % (L, c, fin, len(boxes))))
            continue
        xs = [fill_lattice(rng, 2, fin, *box_region(lo, hi)) for lo, hi in boxes]
        x = np.concatenate(xs) if xs else np.zeros((0, 2), np.float32)
        n = len(x)
        if material == "snow":
            vrng = np.random.default_rng(1000003 * (seed + 1) + i)
            v = np.concatenate([np.tile(vrng.uniform(-2, 2, 2).astype(np.float32), (len(p), 1)) for p in xs]) \
                if xs else np.zeros((0, 2), np.float32)
            kw, dt = dict(SNOW_BATCH), 5e-5
        else:
            v, kw, dt = np.zeros((n, 2), np.float32), dict(E=1e4 / RHO[1], nu=0.2, gravity=(0.0, -9.8),
                                                           boundary_mode="sticky"), 1e-4
        out.append(Scene("config4_scene%03d" % i, 2, L, c, x, v,
                         np.full(n, L - 1, np.int32), _unit_mass(n), dt, 1000, kw,
                         grid_initializer=band_level_map([(tuple(lo), tuple(hi)) for lo, hi in boxes], 2, L, c),
                         description="%d levels %d^2..%d^2, %d boxes, %d particles" % (L, c, fin, len(boxes), n)))
    return out


# ---------------------------------------------------------------------------
# The same configurations generated on the GPU (agimp_lattice_fill): shapes and
# materials as above, lattice jitter from Philox keyed by the seed instead of
# numpy's generator, so the particles are another draw of the same scene.
# (Config 2's random boxes use the same numpy draws for their sizes, places and
# velocities, minus the jitter draws the host version makes between them.)


@dataclass
class DeviceScene:
    name: str
    dim: int
    level: int
    coarsest: int
    shapes: list
    seed: int
    dt: float
    steps: int
    sim_kwargs: dict = field(default_factory=dict)
    grid_initializer: object = None
    refine_every: int = 0
    refine_band: int = 3
    description: str = ""
    per_axis: int = 2
    _n: int = -1

    @property
    def n(self):
        if self._n < 0:
            from . import device_init as di
            self._n = di.lattice_count(self.dim, self.coarsest << (self.level - 1), self.shapes, self.seed,
                                       self.per_axis)
        return self._n

    def build(self, **over):
        """Construct an AdaptiveGIMP whose particles are generated on the GPU."""
        from . import device_init as di
        from .simulator import AdaptiveGIMP
        kw = dict(self.sim_kwargs)
        kw.update(over)
        return AdaptiveGIMP(self.dim, self.level, self.coarsest, self.n,
                            di.lattice_initializer(self.shapes, self.seed, self.per_axis), self.grid_initializer, **kw)


def make_device_config(k, seed=0, scale=1.0):
    """Configurations 1, 2, 3 and 5 with their particles generated on the GPU."""
    from . import device_init as di
    host = make_config(k, seed, scale=min(scale, 1e-3)) if k in (1, 2, 3, 5) else None
    if host is None:
        raise ValueError("device scenes: configs 1, 2, 3 and 5 (config 4: make_batch_config(device=True))")
    L, c = host.level, host.coarsest
    if k == 1:
        shapes = [di.box((0.3 - 0.1 * scale, 0.5 - 0.1 * scale), (0.3 + 0.1 * scale, 0.5 + 0.1 * scale), L - 1),
                  di.box((0.6 - 0.1 * scale, 0.7 - 0.1 * scale), (0.6 + 0.1 * scale, 0.7 + 0.1 * scale), L - 1)]
        boxes = [((0.3 - 0.1 * scale, 0.5 - 0.1 * scale), (0.3 + 0.1 * scale, 0.5 + 0.1 * scale)),
                 ((0.6 - 0.1 * scale, 0.7 - 0.1 * scale), (0.6 + 0.1 * scale, 0.7 + 0.1 * scale))]
        gi = band_level_map(boxes, 2, L, c)
    elif k == 2:
        rng = np.random.default_rng(seed)
        shapes = []
        for _ in range(3):
            side = rng.uniform(0.1, 0.25, 2) * scale
            lo = rng.uniform(0.1, 0.9 - side)
            vel = rng.uniform(-1, 1, 2).astype(np.float32)
            shapes.append(di.box(lo, lo + side, L - 1, velocity=vel))
        gi = None
    elif k == 3:
        shapes = [di.sphere((0.5, 0.6, 0.5), 0.15 * scale, L - 1, velocity=(0.0, -3.0, 0.0))]
        gi = None
    else:
        r = 0.12 * scale
        shapes = [di.sphere((0.35, 0.5, 0.5), r, L - 1, velocity=(2.0, 0.0, 0.0)),
                  di.sphere((0.65, 0.5, 0.5), r, L - 1, velocity=(-2.0, 0.0, 0.0))]
        gi = None
    return DeviceScene(host.name + "_device", host.dim, L, c, shapes, seed, host.dt, host.steps, dict(host.sim_kwargs),
                       grid_initializer=gi, refine_every=host.refine_every, refine_band=host.refine_band,
                       description=host.description + " (particles generated on the GPU)")
