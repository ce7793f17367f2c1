"""Generate golden vectors by running the reference's own source.

Runs the reference project's adaptive_gimp.py, utils.py and init.py (read from
a checkout of g1n0st/adaptive-gimp given by --ref or the AGIMP_REFERENCE
environment variable) under the
Taichi-semantics shim in tests/golden/taichi_shim, on small seeded scenes, and
writes one compressed .npz per scene into tests/golden/.

    python tests/golden/make_golden.py --ref PATH [--only NAME]

The fixtures hold the inputs (particle state, prescribed levels, the level
map tabulated from the reference's grid_initializer), and after every substep
the particle state, fl_p, every level's cell_mask / ad_grid_m / ad_grid_v over
indices [-4, size+8) and node_mask over the finest lattice [0, finest].
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LO = -4


def load_reference(ref):
    sys.path.insert(0, os.path.join(HERE, "taichi_shim"))
    sys.path.insert(0, ref)
    import taichi as ti  # the shim
    import utils
    import adaptive_gimp
    import init
    for mod in (utils, adaptive_gimp, init):
        mod.float = ti._FloatCast
    return ti, adaptive_gimp, init


def tabulate_map(ti, mask_fn, dim, level, coarsest):
    """Tabulate a reference grid_initializer over finest cells [-H, sz+H)^d.

    Entry = returned level; bit 6 set when the call activated nothing.  The
    call must activate either nothing or exactly the cell of the returned
    level that contains I (true of every initializer in init.py).
    """
    sz = coarsest << (level - 1)
    H = max(2, 1 << (level - 1))
    n = sz + 2 * H

    class Rec:
        pass

    rec = Rec()
    rec.level, rec.finest_size, rec.coarsest_size = level, sz, coarsest
    calls = []
    rec.activate_cell = lambda l, I: calls.append((int(l), tuple(int(e) for e in I.a)))
    table = np.zeros((n,) * dim, np.int8)
    for idx in np.ndindex(*table.shape):
        I = tuple(i - H for i in idx)
        calls.clear()
        lv = int(mask_fn(rec, ti.Mat._wrap(np.array(I, np.int64))))
        if not calls:
            table[idx] = lv | 64
        else:
            assert calls == [(lv, I)], (I, lv, calls)
            table[idx] = lv
    return table, H


def dense_level(f, lsize, dim, comps=None):
    n = lsize + 12
    shp = (n,) * dim + ((comps,) if comps else ())
    out = np.zeros(shp, np.float32 if f.dt is np.float32 else np.int32)
    for k, v in f.store.items():
        idx = tuple(i - LO for i in k)
        assert all(0 <= i < n for i in idx), ("out of fixture range", k)
        out[idx] = v
    return out


def snapshot(sim, dim):
    L = sim.level
    d = dict(x=sim.x_p.to_numpy(), v=sim.v_p.to_numpy(), F=sim.F_p.to_numpy(), C=sim.C_p.to_numpy(),
             fl=sim.fl_p.to_numpy())
    for l in range(L):
        ls = sim.coarsest_size << l
        d["cell%d" % l] = dense_level(sim.cell_mask[l], ls, dim)
        d["m%d" % l] = dense_level(sim.ad_grid_m[l], ls, dim)
        d["v%d" % l] = dense_level(sim.ad_grid_v[l], ls, dim, dim)
    sz = sim.finest_size
    nm = np.zeros((sz + 1,) * dim, np.int32)
    dropped = 0
    for k, v in sim.node_mask.store.items():
        if all(0 <= i <= sz for i in k):
            nm[k] = v
        elif v:
            dropped += 1
    d["node_mask"] = nm
    d["node_mask_outside"] = np.int32(dropped)
    return d


def scene_boxes(rng, n, boxes, vel):
    """n particles split evenly over axis-aligned boxes (lo, hi) with velocities."""
    dim = len(boxes[0][0])
    per = [n // len(boxes)] * len(boxes)
    per[-1] += n - sum(per)
    xs, vs, us = [], [], []
    for (lo, hi), vv, k in zip(boxes, vel, per):
        u = rng.random((k, dim)).astype(np.float32)
        xs.append(np.asarray(lo, np.float32) + u * (np.asarray(hi, np.float32) - np.asarray(lo, np.float32)))
        vs.append(np.tile(np.asarray(vv, np.float32), (k, 1)))
        us.append(u)
    return np.concatenate(xs).astype(np.float32), np.concatenate(vs).astype(np.float32), np.concatenate(us)


def band_levels(u, bands):
    """Prescribed level from the relative position u in its box, init.py:17-29 /
    run_3d.py:151-156 style: innermost band -> level 0, outer bands finer."""
    g = np.full(u.shape[0], len(bands), np.int32)
    for lvl in reversed(range(len(bands))):
        lo = bands[lvl]
        inside = np.all((u >= lo) & (u <= 1 - lo), axis=1)
        g[inside] = lvl
    return g


SCENES = {}


def scene(name):
    def deco(fn):
        SCENES[name] = fn
        return fn
    return deco


def _common_2d(seed, n):
    rng = np.random.default_rng(seed)
    x, v, u = scene_boxes(rng, n, [((0.2, 0.1), (0.45, 0.35)), ((0.4, 0.5), (0.65, 0.75))],
                          [(0.0, 20.0), (0.0, -20.0)])
    # a deterministic perturbation so C and F are not trivial from the start
    v = v + (rng.standard_normal(v.shape) * 2.0).astype(np.float32)
    return x, v, u


for _k in range(1, 6):
    def _mk(k):
        @scene("static2d_mask%d" % k)
        def _s(ti, ag, init):
            x, v, u = _common_2d(100 + k, 300)
            return dict(dim=2, level=4, coarsest=8, x=x, v=v, g=np.zeros(len(x), np.int32),
                        mask=getattr(init, "initialize_mask%d" % k), dt=2e-5, steps=3)
        return _s
    _mk(_k)


@scene("dynamic2d")
def _dyn2(ti, ag, init):
    x, v, u = _common_2d(7, 400)
    g = band_levels(u, [0.2, 0.1, 0.03])  # init.py:17-29 thresholds
    return dict(dim=2, level=4, coarsest=8, x=x, v=v, g=g, mask=None, dt=2e-5, steps=3)


@scene("dynamic2d_l3")
def _dyn2b(ti, ag, init):
    x, v, u = _common_2d(8, 300)
    g = band_levels(u, [0.25, 0.08])
    return dict(dim=2, level=3, coarsest=16, x=x, v=v, g=g, mask=None, dt=2e-5, steps=3)


@scene("dynamic3d")
def _dyn3(ti, ag, init):
    rng = np.random.default_rng(11)
    x, v, u = scene_boxes(rng, 160, [((0.25, 0.15, 0.25), (0.5, 0.4, 0.5)), ((0.3, 0.5, 0.3), (0.55, 0.75, 0.55))],
                          [(0.0, 20.0, 0.0), (0.0, -20.0, 0.0)])
    v = v + (rng.standard_normal(v.shape) * 2.0).astype(np.float32)
    g = band_levels(u, [0.3, 0.1])  # run_3d.py:151-156 style, widened for a small scene
    return dict(dim=3, level=3, coarsest=8, x=x, v=v, g=g, mask=None, dt=1e-4, steps=2)


@scene("dynamic3d_large")
def _dyn3_large(ti, ag, init):
    # a few thousand particles on a 3-level octree (16^3 .. 64^3): a wide block
    # whose core is prescribed the coarsest level (several coarse cells
    # across, so some survive the culling), hit by a smaller falling block
    rng = np.random.default_rng(13)
    x, v, u = scene_boxes(rng, 3000, [((0.18, 0.08, 0.18), (0.82, 0.6, 0.82)), ((0.35, 0.66, 0.35), (0.6, 0.9, 0.6))],
                          [(0.0, 2.0, 0.0), (1.0, -8.0, 0.5)])
    v = v + (rng.standard_normal(v.shape) * 1.0).astype(np.float32)
    g = band_levels(u, [0.22, 0.08])
    return dict(dim=3, level=3, coarsest=16, x=x, v=v, g=g, mask=None, dt=5e-5, steps=3)


def run_scene(ti, ag, init, name, spec, out_dir):
    dim, L, c = spec["dim"], spec["level"], spec["coarsest"]
    x, v, g = spec["x"], spec["v"], spec["g"]
    n = len(x)
    F = np.tile(np.eye(dim, dtype=np.float32), (n, 1, 1))
    C = np.zeros((n, dim, dim), np.float32)
    m = np.ones(n, np.float32)

    def pinit(sim):
        sim.x_p.from_numpy(x)
        sim.v_p.from_numpy(v)
        sim.F_p.from_numpy(F)
        sim.C_p.from_numpy(C)
        sim.m_p.from_numpy(m * np.float32(sim.p_mass))
        sim.g_p.from_numpy(g)

    sim = ag.AdaptiveGIMP(dim, L, c, n, pinit, spec["mask"])
    rec = dict(dim=np.int32(dim), level=np.int32(L), coarsest=np.int32(c), dt=np.float64(spec["dt"]),
               steps=np.int32(spec["steps"]), x0=x, v0=v, F0=F, C0=C, m0=m, g0=g)
    if spec["mask"] is not None:
        table, H = tabulate_map(ti, spec["mask"], dim, L, c)
        rec["level_map"] = table
        rec["map_halo"] = np.int32(H)
    for s in range(spec["steps"]):
        t0 = time.time()
        sim.substep(spec["dt"])
        snap = snapshot(sim, dim)
        for k, val in snap.items():
            rec["s%d_%s" % (s, k)] = val
        print("  %s step %d: %.1fs (binned %d/%d)" % (name, s, time.time() - t0, int((snap["fl"] >= 0).sum()), n))
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), **rec)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("AGIMP_REFERENCE"),
                    help="checkout of the reference (default: $AGIMP_REFERENCE)")
    ap.add_argument("--only", default=None)
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the reference checkout with --ref or AGIMP_REFERENCE")
    ti, ag, init = load_reference(a.ref)
    for name, fn in SCENES.items():
        if a.only and name != a.only:
            continue
        print(name)
        run_scene(ti, ag, init, name, fn(ti, ag, init), a.out)


if __name__ == "__main__":
    main()
