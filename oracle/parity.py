"""Long-horizon parity of a simulator run against the oracle.

TEST INFRASTRUCTURE ONLY (the checker): used by the GPU tests and by the
benchmark's CPU leg, never by the product path.

The oracle restates the reference's substep (adaptive_gimp.py:323-352, with
the refinement extension every `refine_every` substeps).  A run is compared
with the f32 oracle and the f64 oracle after the same substeps from the same
initial state; the f32-vs-f64 difference is the noise floor of f32
arithmetic.  Quantities, as the error report of the hot path defines them:

* positions: relative L2 error normalised by the RMS displacement from the
  initial state, plus the largest absolute error in domain units;
* velocities: relative L2 error;
* grid momentum m v per level at the last substep: relative L2 error over a
  box of nodes that covers every particle.
"""
from __future__ import annotations

import time

import numpy as np

import oracle as O


def oracle_params(sim_kwargs, dim):
    """AdaptiveGIMP keyword overrides -> oracle parameters."""
    out = {}
    if "gravity" in sim_kwargs:
        out["gravity"] = tuple(sim_kwargs["gravity"]) + (0.0,) * (3 - len(sim_kwargs["gravity"]))
    for k in ("E", "nu", "radius", "boundary_gap", "theta_c", "theta_s", "hardening"):
        if k in sim_kwargs:
            out[k] = sim_kwargs[k]
    out["boundary_mode"] = {"ref_slip": 0, "sticky": 1}[sim_kwargs.get("boundary_mode", "ref_slip")]
    out["plasticity"] = {None: 0, "none": 0, "snow": 1}[sim_kwargs.get("plasticity")]
    out["colliders"] = tuple(sim_kwargs.get("colliders", ()))
    out["invalid_nodes"] = {"raw": 0, "normalize": 1}[sim_kwargs.get("invalid_nodes", "raw")]
    return out


def make_oracle(scene, f64=False, level_map=None):
    """An oracle holding the scene's initial state (F = I, C = 0)."""
    d, n = scene.dim, scene.n
    o = O.Oracle(d, scene.level, scene.coarsest, n, f64=f64, **oracle_params(scene.sim_kwargs, d))
    o.set_particles(scene.x, scene.v, np.tile(np.eye(d), (n, 1, 1)), np.zeros((n, d, d)), scene.m, scene.g)
    if level_map is not None:
        o.set_level_map(*level_map)
    return o


def step(o, scene, i, threads=0):
    """Substep i of the scene's schedule (refinement first when it is due)."""
    if scene.refine_every and i % scene.refine_every == 0:
        o.refine_levels(scene.refine_band)
    o.substep(scene.dt, 1, threads)


def run(o, scene, first, count, threads=0):
    for i in range(first, first + count):
        step(o, scene, i, threads)


def grid_boxes(x, coarsest, levels, margin=4):
    """(lo, n) per level: a cube of node indices covering every particle."""
    out = []
    lo_x, hi_x = float(np.min(x)), float(np.max(x))
    for l in range(levels):
        size = coarsest << l
        lo = max(int(np.floor(lo_x * size)) - margin, -4)
        hi = min(int(np.ceil(hi_x * size)) + margin, size + 7)
        out.append((lo, hi - lo + 1))
    return out


def _rel(a, b):
    den = np.sqrt((np.asarray(b, np.float64) ** 2).sum())
    return float(np.sqrt(((np.asarray(a, np.float64) - b) ** 2).sum()) / den) if den > 0 else 0.0


def compare(a, b, x0, ga=None, gb=None):
    """Errors of state `a` against state `b` (dicts with x [N, d], v [N, d]),
    both started from positions x0; ga / gb: per-level (m, v) boxes."""
    xa, xb = np.asarray(a["x"], np.float64), np.asarray(b["x"], np.float64)
    disp = float(np.sqrt(((xb - x0) ** 2).sum(1).mean()))
    ex = np.sqrt(((xa - xb) ** 2).sum(1))
    out = {
        "position_rel": float(np.sqrt((ex ** 2).mean()) / disp) if disp > 0 else 0.0,
        "position_max_abs": float(ex.max()) if ex.size else 0.0,
        "velocity_rel": _rel(a["v"], b["v"]),
    }
    if ga is not None and gb is not None:
        out["grid_momentum_rel"] = [
            _rel(np.asarray(ma, np.float64)[..., None] * va, np.asarray(mb, np.float64)[..., None] * vb)
            for (ma, va), (mb, vb) in zip(ga, gb)]
    return out


def oracle_grids(o, boxes):
    return [o.grid(l, lo, n)[:2] for l, (lo, n) in enumerate(boxes)]


def report(gpu, grids_gpu, o32, o64, x0, boxes, substeps):
    """The parity block: the run against the f32 and f64 oracles, and the
    f32-vs-f64 noise floor, with the pass rule (error within 10x the floor
    or 1e-3, whichever is larger, on positions)."""
    p32, p64 = o32.particles(), o64.particles()
    g32, g64 = oracle_grids(o32, boxes), oracle_grids(o64, boxes)
    vs32 = compare(gpu, p32, x0, grids_gpu, g32)
    vs64 = compare(gpu, p64, x0, grids_gpu, g64)
    floor = compare(p32, p64, x0, g32, g64)
    bound = max(10 * floor["position_rel"], 1e-3)
    return {
        "substeps": substeps,
        "vs_f32_oracle": vs32,
        "vs_f64_oracle": vs64,
        "f32_vs_f64_floor": floor,
        "position_bound": bound,
        "pass": bool(vs32["position_rel"] <= bound and vs64["position_rel"] <= bound),
        "levels_equal_f32": bool(np.array_equal(np.asarray(gpu["g"]), p32["g"])) if "g" in gpu else None,
    }


def timed_run(o, scene, first, count, threads, seconds):
    """Run `count` substeps from `first`; the substeps finished within the
    first `seconds` of wall time form the timing sample.  Returns
    (substeps timed, seconds of the sample)."""
    t0 = time.perf_counter()
    timed, el = 0, 0.0
    for i in range(first, first + count):
        step(o, scene, i, threads)
        now = time.perf_counter() - t0
        if el == 0.0 or now <= seconds:
            timed, el = i - first + 1, now
    return timed, el
