"""GPU parity: the CUDA substep (called through the C ABI) against the
reference's golden vectors and the CPU oracle on the same seeded inputs.

Topology and binning (cell_mask, node_mask classes, fl_p) must match
bit-exactly.  Floating point: the GPU sums P2G contributions with atomics in
an unspecified order and evaluates the GIMP stencil in factorised form, so
floats agree to f32 rounding; tolerances below are max|a-b| / max|b| per
array.
"""
import numpy as np
import pytest

import oracle as O
from _golden_util import LO, grid_v_close, load, node_classes, node_norm, scenes, step_input
from _gpu_util import gpu_grid, gpu_sim, gpu_state, have_gpu, oracle_kwargs, scale_rel

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]

RTOL_PART = 2e-5    # particle x, v, F, C after one substep
RTOL_MASS = 2e-5    # nodal mass
RTOL_GRID_V = 2e-4  # nodal momentum / velocity (light nodes amplify summation order)


@pytest.mark.parametrize("name", scenes())
def test_gpu_matches_reference_golden_per_step(name):
    z = load(name)
    dim, L, c = int(z["dim"]), int(z["level"]), int(z["coarsest"])
    n = len(z["x0"])
    sim = gpu_sim(dim, L, c, n, z.get("level_map"), int(z["map_halo"]) if "map_halo" in z else None)
    for s in range(int(z["steps"])):
        st = step_input(z, s)
        sim.set_particles(x=st["x"], v=st["v"], F=st["F"], C=st["C"], m=z["m0"], g=z["g0"])
        sim.substep(float(z["dt"]))
        assert sim.errors() == 0
        pre = "s%d_" % s
        p = gpu_state(sim)
        np.testing.assert_array_equal(p["fl"], z[pre + "fl"])
        np.testing.assert_array_equal(sim.bin_keys(), ref_bin_keys(st["x"], z[pre + "fl"], c))
        nm = sim.node_mask.read_lattice()
        np.testing.assert_array_equal(node_classes(nm), node_classes(z[pre + "node_mask"]))
        np.testing.assert_array_equal(node_norm(nm), node_norm(z[pre + "node_mask"]))
        for l in range(L):
            m, v, cell = gpu_grid(sim, l)
            np.testing.assert_array_equal(cell, z[pre + "cell%d" % l])
            assert scale_rel(m, z[pre + "m%d" % l]) <= RTOL_MASS, (s, l)
            ok, r = grid_v_close(v, z[pre + "v%d" % l], z[pre + "m%d" % l], RTOL_GRID_V)
            assert ok, (s, l, r)
        for k in "xvFC":
            assert scale_rel(p[k], z[pre + k]) <= RTOL_PART, (s, k, scale_rel(p[k], z[pre + k]))
    sim.close()


def ref_bin_keys(x, fl, coarsest):
    """The reference's pid blocks (adaptive_gimp.py:208-216) from a substep's
    input positions and fl_p: level fl, block base // 4 at that level (base =
    int(x / dx + 0.5) - 1 in f32, dx = coarsest_dx / 2**fl), packed like
    agimp_get_bins."""
    x = np.asarray(x, np.float32)
    n, d = x.shape
    keys = np.full(n, np.iinfo(np.uint64).max, np.uint64)
    for p in np.nonzero(fl >= 0)[0]:
        l = int(fl[p])
        dx = np.float32(1.0 / coarsest / 2 ** l)
        base = (x[p] / dx + np.float32(0.5)).astype(np.int64) - 1
        k = l << 60
        for a in range(d):
            k |= int(base[a] // 4 + 1) << (20 * (d - 1 - a))
        keys[p] = k
    return keys


def _run_pair(scene, steps, refine=False, graphs=True):
    """Same scene on the GPU and on the f32 / f64 oracles; returns states."""
    from agimp.simulator import tabulate_level_map
    d, n = scene.dim, scene.n
    sim = scene.build(graphs=graphs)
    kw = oracle_kwargs(scene.sim_kwargs, d)
    orcs = [O.Oracle(d, scene.level, scene.coarsest, n, f64=f, **kw) for f in (False, True)]
    F = np.tile(np.eye(d), (n, 1, 1))
    for o in orcs:
        o.set_particles(scene.x, scene.v, F, np.zeros((n, d, d)), scene.m, scene.g)
        if scene.grid_initializer is not None:
            t, H = tabulate_level_map(scene.grid_initializer, d, scene.level, scene.coarsest)
            o.set_level_map(t, H)
    for i in range(steps):
        if refine and scene.refine_every and i % scene.refine_every == 0:
            sim.refine_levels(scene.refine_band)
            for o in orcs:
                o.refine_levels(scene.refine_band)
        sim.substep(scene.dt)
        for o in orcs:
            o.substep(scene.dt)
    return sim, orcs


# config 1 runs the reference's grid update; configs 2, 3 and 5 normalise the
# momentum of unactivated nodes (invalid_nodes="normalize")
@pytest.mark.parametrize("k,scale,steps", [(1, 0.35, 20), (2, 0.35, 20), (3, 0.3, 10), (5, 0.25, 10)])
def test_gpu_matches_oracle_configs(k, scale, steps):
    """Seeded benchmark scenes (bodies shrunk so the serial oracle is fast):
    after `steps` substeps the GPU positions sit within the f32 noise floor
    (the f32 oracle against the f64 oracle) of the f32 oracle."""
    from agimp import scenes as S
    scene = S.make_config(k, scale=scale)
    sim, (o32, o64) = _run_pair(scene, steps, refine=True)
    assert sim.errors() & ~2 == 0
    g = gpu_state(sim)
    p32, p64 = o32.particles(), o64.particles()
    disp = np.sqrt(((p64["x"] - scene.x) ** 2).sum(1).mean())
    e_gpu = np.sqrt(((g["x"] - p32["x"]) ** 2).sum(1).mean()) / disp
    e_floor = np.sqrt(((p32["x"] - p64["x"]) ** 2).sum(1).mean()) / disp
    # relative position error against the f32 oracle, normalised by the RMS
    # displacement; allowed: 10x the f32-vs-f64 floor or 1e-3, whichever is larger
    assert e_gpu <= max(10 * e_floor, 1e-3), (e_gpu, e_floor)
    np.testing.assert_array_equal(g["g"], p32["g"])
    sim.close()


def test_topology_bit_exact_on_config_scene():
    """One substep of a seeded config scene: cell masks, node classes and
    fl_p equal the oracle's exactly."""
    from agimp import scenes as S
    scene = S.make_config(2, scale=0.3)
    sim, (o32, _) = _run_pair(scene, 1)
    for l in range(scene.level):
        n = (scene.coarsest << l) + 12
        _, _, cg = gpu_grid(sim, l)
        _, _, co = o32.grid(l, LO, n)
        np.testing.assert_array_equal(cg, co)
    np.testing.assert_array_equal(node_norm(sim.node_mask.read_lattice()), node_norm(o32.node_mask()))
    np.testing.assert_array_equal(gpu_state(sim)["fl"], o32.particles()["fl"])
    sim.close()


def test_refine_levels_bit_exact():
    from agimp import scenes as S
    scene = S.make_config(3, scale=0.4)
    sim = scene.build()
    o = O.Oracle(3, scene.level, scene.coarsest, scene.n)
    o.set_particles(scene.x, scene.v, np.tile(np.eye(3), (scene.n, 1, 1)), np.zeros((scene.n, 3, 3)), scene.m,
                    scene.g)
    # band 2: the sphere (r = 15 finest cells) is deep enough for all three levels
    sim.refine_levels(2)
    o.refine_levels(2)
    g = sim.g_p.to_numpy()
    np.testing.assert_array_equal(g, o.particles()["g"])
    assert len(np.unique(g)) == scene.level
    sim.close()


def test_graph_and_direct_launch_agree():
    from agimp import scenes as S
    scene = S.make_config(1, scale=0.3)
    a = scene.build(graphs=True)
    b = scene.build(graphs=False)
    a.substep(scene.dt, 5)
    b.substep(scene.dt, 5)
    xa, xb = a.x_p.to_numpy(), b.x_p.to_numpy()
    assert scale_rel(xa, xb) < 1e-5
    np.testing.assert_array_equal(a.fl_p.to_numpy(), b.fl_p.to_numpy())
    a.close()
    b.close()


def test_empty_scene():
    sim = gpu_sim(3, 3, 16, 0)
    sim.substep(1e-4, 3)
    assert sim.errors() == 0
    assert sim.stats()["n_binned"] == 0
    sim.close()


def test_escaped_particles_are_frozen_and_flagged():
    """Particles outside [0,1)^d (undefined in the reference) are flagged and
    left unchanged; the others evolve exactly as in the oracle, which applies
    the same rule."""
    rng = np.random.default_rng(5)
    n = 600
    x = rng.uniform(0.3, 0.7, (n, 2)).astype(np.float32)
    x[:5] = [[1.5, 0.5], [-0.2, 0.5], [0.5, 1.0], [np.nan, 0.5], [0.5, -1e-3]]
    v = np.zeros((n, 2), np.float32)
    g = np.full(n, 2, np.int32)
    sim = gpu_sim(2, 3, 16, n)
    sim.set_particles(x=x, v=v, F=np.tile(np.eye(2, dtype=np.float32), (n, 1, 1)),
                      C=np.zeros((n, 2, 2), np.float32), m=np.ones(n, np.float32), g=g)
    sim.substep(1e-4, 2)
    assert sim.errors() == 2  # AGIMP_ERR_ESCAPED
    s = gpu_state(sim)
    assert np.all(s["fl"][:5] == -1)
    np.testing.assert_array_equal(s["x"][:5], x[:5])
    o = O.Oracle(2, 3, 16, n)
    o.set_particles(x, v, np.tile(np.eye(2), (n, 1, 1)), np.zeros((n, 2, 2)), np.ones(n), g)
    o.substep(1e-4, 2)
    p = o.particles()
    np.testing.assert_array_equal(s["fl"], p["fl"])
    assert scale_rel(s["x"][5:], p["x"][5:]) < 1e-5
    sim.close()


def test_static_reference_mask_via_scalar_initializer():
    """A reference-style scalar grid_initializer passed to the constructor
    (adaptive_gimp.py:65-66) gives the same substep as the golden run."""
    from agimp import AdaptiveGIMP, scenes
    z = load("static2d_mask4")
    n = len(z["x0"])

    def pinit(sim):
        sim.set_particles(x=z["x0"], v=z["v0"], F=z["F0"], C=z["C0"], m=z["m0"], g=z["g0"])

    sim = AdaptiveGIMP(2, int(z["level"]), int(z["coarsest"]), n, pinit, scenes.initialize_mask4)
    assert sim.static_adaptivity
    sim.substep(float(z["dt"]))
    np.testing.assert_array_equal(sim.fl_p.to_numpy(), z["s0_fl"])
    assert scale_rel(sim.x_p.to_numpy(), z["s0_x"]) <= RTOL_PART
    sim.close()


def test_create_rejects_lattices_beyond_32bit_indices():
    # a 3D level of 2048^3 cells stores 515^3 blocks of 64 cells: more than
    # 2^31 elements, which the kernels' 32-bit element indices cannot address
    import ctypes

    from agimp import _capi
    lib = _capi.load()
    p = _capi.Params()
    lib.agimp_default_params(ctypes.byref(p), 3, 1, 2048, 10)
    h = ctypes.c_void_p()
    assert lib.agimp_create(ctypes.byref(p), 0, ctypes.byref(h)) == 2  # AGIMP_CAPACITY
    assert not h.value


@pytest.mark.parametrize("k,scale,steps", [(3, 0.35, 100)])
def test_gpu_long_horizon_parity(k, scale, steps):
    """The benchmark's dynamic 3D snow scene (refinement every 10 substeps,
    slab collider, invalid-node normalisation) for 100 substeps: the GPU
    against the f32 and the f64 oracle (OpenMP) on positions, velocities and
    per-level grid momentum at the last substep.  Positions must sit within
    10x the f32-vs-f64 floor or 1e-3 (relative, normalised by the RMS
    displacement); velocities and grid momentum within 10x their floor or
    1e-2."""
    import os

    import parity as PY
    from agimp import scenes as S
    scene = S.make_config(k, scale=scale)
    sim = scene.build()
    for i in range(steps):
        if scene.refine_every and i % scene.refine_every == 0:
            sim.refine_levels(scene.refine_band)
        sim.substep(scene.dt)
    assert sim.errors() & ~2 == 0
    gpu = {"x": sim.x_p.to_numpy(), "v": sim.v_p.to_numpy(), "g": sim.g_p.to_numpy()}
    boxes = PY.grid_boxes(gpu["x"], scene.coarsest, scene.level)
    grids = [(sim.ad_grid_m[l].read(lo, n), sim.ad_grid_v[l].read(lo, n)) for l, (lo, n) in enumerate(boxes)]
    sim.close()
    threads = os.cpu_count() or 1
    o32, o64 = PY.make_oracle(scene, False), PY.make_oracle(scene, True)
    PY.run(o32, scene, 0, steps, threads)
    PY.run(o64, scene, 0, steps, threads)
    rep = PY.report(gpu, grids, o32, o64, scene.x, boxes, steps)
    print(rep)
    fl = rep["f32_vs_f64_floor"]
    assert rep["pass"], rep
    for ref in ("vs_f32_oracle", "vs_f64_oracle"):
        e = rep[ref]
        assert e["velocity_rel"] <= max(10 * fl["velocity_rel"], 1e-2), (ref, e)
        for l, (eg, ef) in enumerate(zip(e["grid_momentum_rel"], fl["grid_momentum_rel"])):
            assert eg <= max(10 * ef, 1e-2), (ref, l, eg, ef)
