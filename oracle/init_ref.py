"""CPU restatement of the device scene initialisers (test infrastructure only:
the tests compare agimp_lattice_fill, agimp_random_fill and the device level
maps of libagimp.so against it).

* philox: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
  as easy as 1, 2, 3", SC 2011), vectorised over counters.  Pinned by the
  generator's published known-answer vectors (tests/test_init_cpu.py).
* lattice_fill: the jittered sub-lattice of the library's lattice fill, in
  float64 numpy arithmetic (one rounding per operation, as on the device) and
  rounded to float32 once.  With jitter off it equals the host scene
  generator's lattice (scenes.fill_lattice, jitter=False), which pins the
  lattice geometry and order.
* random_fill: init.py:3-32 / run_3d.py:14-32's uniform particles in boxes
  with level bands (x = u * size + lo in float32, the first matching band).
* The level-map rules are init.py:34-98's masks, which the host tabulation
  (simulator.tabulate_level_map over scenes.initialize_mask1..5) already
  states; the tests compare the device tables with that tabulation.
"""
import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57  # round multipliers
W0, W1 = 0x9E3779B9, 0xBB67AE85  # key increments (Weyl sequence)
_M32 = np.uint64(0xFFFFFFFF)


def philox(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 of counters (c0, c1, c2, c3) under key (k0, k1); arrays
    broadcast; returns four uint32 arrays."""
    x, y, z, w = [np.asarray(v, np.uint64) & _M32 for v in (c0, c1, c2, c3)]
    k0 = np.uint64(int(k0) & 0xFFFFFFFF)
    k1 = np.uint64(int(k1) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(M0) * x
        p1 = np.uint64(M1) * z
        x, y, z, w = ((p1 >> np.uint64(32)) ^ y ^ k0) & _M32, p1 & _M32, ((p0 >> np.uint64(32)) ^ w ^ k1) & _M32, \
            p0 & _M32
        k0 = (k0 + np.uint64(W0)) & _M32
        k1 = (k1 + np.uint64(W1)) & _M32
    return [v.astype(np.uint32) for v in (x, y, z, w)]


def u53(a, b):
    """Uniform float64 in [0, 1) from two words (a high, b low): 53 bits."""
    v = (a.astype(np.uint64) << np.uint64(32) | b.astype(np.uint64)) >> np.uint64(11)
    return v.astype(np.float64) * 2.0 ** -53


def u24(a):
    """Uniform float32 in [0, 1) from one word: 24 bits."""
    return (a >> np.uint32(8)).astype(np.float32) * np.float32(2.0 ** -24)


def box(lo, hi, level, velocity=(0.0, 0.0, 0.0), mass=1.0):
    return dict(kind="box", lo=tuple(lo), hi=tuple(hi), level=level, velocity=tuple(velocity), mass=mass)


def sphere(centre, radius, level, velocity=(0.0, 0.0, 0.0), mass=1.0):
    return dict(kind="sphere", centre=tuple(centre), radius=radius, level=level, velocity=tuple(velocity), mass=mass)


def lattice_fill(dim, finest, shapes, seed=0, per_axis=2, jitter=True):
    """Particles of the jittered sub-lattice inside the shapes: dict of x
    [N][dim] f32, v [N][dim] f32, g [N] i32, m [N] f32, in generation order."""
    h = 1.0 / (finest * per_axis)
    hh = 0.5 * h
    k0, k1 = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    xs, vs, gs, ms = [], [], [], []
    for j, s in enumerate(shapes):
        if s["kind"] == "box":
            a, b = np.asarray(s["lo"][:dim], np.float64), np.asarray(s["hi"][:dim], np.float64)
        else:
            c = np.asarray(s["centre"][:dim], np.float64)
            a, b = c - s["radius"], c + s["radius"]
        start = np.floor(a / h)
        n = np.maximum(0, np.ceil(b / h) - start).astype(np.int64)
        k = np.arange(int(np.prod(n)), dtype=np.int64)
        idx = np.stack(np.unravel_index(k, tuple(n)), -1) if len(k) else np.zeros((0, dim), np.int64)
        cen = (start + idx.astype(np.float64)) * h + hh
        if jitter and len(k):
            r = philox(k & 0xFFFFFFFF, k >> 32, np.full(len(k), j), np.zeros(len(k)), k0, k1)
            u = [u53(r[0], r[1]), u53(r[2], r[3])]
            if dim == 3:
                r2 = philox(k & 0xFFFFFFFF, k >> 32, np.full(len(k), j), np.ones(len(k)), k0, k1)
                u.append(u53(r2[0], r2[1]))
            off = np.stack([-hh + h * u[d] for d in range(dim)], -1)
            x = cen + off
        else:
            x = cen
        if s["kind"] == "box":
            inside = np.all((x >= a) & (x < b), axis=1)
        else:
            e = x - np.asarray(s["centre"][:dim], np.float64)
            s2 = e[:, 0] * e[:, 0]
            for d in range(1, dim):
                s2 = s2 + e[:, d] * e[:, d]
            inside = s2 < s["radius"] * s["radius"]
        x = x[inside].astype(np.float32)
        cnt = len(x)
        xs.append(x)
        vs.append(np.tile(np.asarray(s["velocity"][:dim], np.float32), (cnt, 1)))
        gs.append(np.full(cnt, s["level"], np.int32))
        ms.append(np.full(cnt, s["mass"], np.float32))
    cat = (lambda a, shp, t: np.concatenate(a) if a else np.zeros(shp, t))
    return dict(x=cat(xs, (0, dim), np.float32), v=cat(vs, (0, dim), np.float32), g=cat(gs, (0,), np.int32),
                m=cat(ms, (0,), np.float32))


def random_box(count, lo, size, level, velocity=(0.0, 0.0, 0.0), mass=1.0, bands=()):
    return dict(count=count, lo=tuple(lo), size=tuple(size), level=level, velocity=tuple(velocity), mass=mass,
                bands=tuple(bands))


def random_fill(dim, boxes, seed=0):
    """init.py:3-32-style particles: box after box, x = u * size + lo (f32),
    g = the level of the first band holding u on every axis, else the box's."""
    k0, k1 = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    n = sum(b["count"] for b in boxes)
    p = np.arange(n, dtype=np.int64)
    r = philox(p & 0xFFFFFFFF, p >> 32, np.zeros(n), np.zeros(n), k0, k1)
    u = np.stack([u24(r[d]) for d in range(dim)], -1)
    x = np.zeros((n, dim), np.float32)
    v = np.zeros((n, dim), np.float32)
    g = np.zeros(n, np.int32)
    m = np.zeros(n, np.float32)
    first = 0
    for b in boxes:
        sl = slice(first, first + b["count"])
        ub = u[sl]
        x[sl] = ub * np.asarray(b["size"][:dim], np.float32) + np.asarray(b["lo"][:dim], np.float32)
        v[sl] = np.asarray(b["velocity"][:dim], np.float32)
        gb = np.full(b["count"], b["level"], np.int32)
        done = np.zeros(b["count"], bool)
        for blo, bhi, blev in b["bands"]:
            hit = ~done & np.all((np.float32(blo) <= ub) & (ub <= np.float32(bhi)), axis=1)
            gb[hit] = blev
            done |= hit
        g[sl] = gb
        m[sl] = b["mass"]
        first += b["count"]
    return dict(x=x, v=v, g=g, m=m)
