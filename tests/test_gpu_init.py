"""Scene initialisers on the device (agimp_lattice_fill, agimp_random_fill,
agimp_set_level_map_rule, agimp_set_coarse_level_map) against the numpy
restatement (oracle/init_ref.py) and the host tabulation of the level maps:
bit-exact particle fields and tables."""
import numpy as np
import pytest

import init_ref as R
from _gpu_util import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


def _dev_shapes(shapes):
    from agimp import device_init as di
    out = []
    for s in shapes:
        if s["kind"] == "box":
            out.append(di.box(s["lo"], s["hi"], s["level"], s["velocity"], s["mass"]))
        else:
            out.append(di.sphere(s["centre"], s["radius"], s["level"], s["velocity"], s["mass"]))
    return out


def _check_state(sim, want, dim):
    n = len(want["x"])
    np.testing.assert_array_equal(sim.x_p.to_numpy(), want["x"])
    np.testing.assert_array_equal(sim.v_p.to_numpy(), want["v"])
    np.testing.assert_array_equal(sim.g_p.to_numpy(), want["g"])
    np.testing.assert_array_equal(sim.m_p.to_numpy(), want["m"])
    np.testing.assert_array_equal(sim.F_p.to_numpy(), np.tile(np.eye(dim, dtype=np.float32), (n, 1, 1)))
    np.testing.assert_array_equal(sim.C_p.to_numpy(), np.zeros((n, dim, dim), np.float32))
    np.testing.assert_array_equal(sim.Jp.to_numpy(), np.ones(n, np.float32))


CASES = [
    (2, 3, 32, 2, True, 11, [R.box((0.2, 0.3), (0.41, 0.52), 2, (1.0, -2.0), 1.0),
                              R.sphere((0.6, 0.55), 0.13, 1, (0.0, 3.0), 2.0)]),
    (2, 2, 64, 3, False, 0, [R.box((0.05, 0.1), (0.3, 0.3), 1)]),
    (3, 3, 16, 2, True, 2 ** 40 + 7, [R.sphere((0.5, 0.6, 0.5), 0.15, 2, (0.0, -3.0, 0.0)),
                                      R.box((0.3, 0.2, 0.3), (0.7, 0.3, 0.7), 0)]),
]


@pytest.mark.parametrize("dim,level,coarsest,per_axis,jitter,seed,shapes", CASES)
def test_lattice_fill_matches_restatement(dim, level, coarsest, per_axis, jitter, seed, shapes):
    from agimp import device_init as di
    finest = coarsest << (level - 1)
    want = R.lattice_fill(dim, finest, shapes, seed, per_axis, jitter)
    ds = _dev_shapes(shapes)
    n = di.lattice_count(dim, finest, ds, seed, per_axis, jitter)
    assert n == len(want["x"]) and n > 1000
    sim = di.lattice_simulator(dim, level, coarsest, ds, seed, per_axis, jitter)
    _check_state(sim, want, dim)
    sim.substep(1e-4)
    assert sim.errors() == 0
    sim.close()


def test_lattice_fill_checks_the_count():
    from agimp import AdaptiveGIMP, device_init as di
    from agimp._capi import AgimpError
    shapes = [di.box((0.2, 0.2), (0.4, 0.4), 1)]
    n = di.lattice_count(2, 64, shapes)
    with pytest.raises(AgimpError):
        AdaptiveGIMP(2, 2, 32, n + 1, di.lattice_initializer(shapes), None)


@pytest.mark.parametrize("dim", [2, 3])
def test_random_fill_matches_restatement(dim):
    from agimp import AdaptiveGIMP, device_init as di
    n = 60000
    if dim == 2:
        boxes = di.reference_boxes_2d(n, case=0)
        rboxes = [R.random_box(n // 2, (0.2, 0.1), (0.4, 0.4), 3, (0.0, 20.0), 1.0,
                               ((0.2, 0.8, 0), (0.1, 0.9, 1), (0.03, 0.97, 2))),
                  R.random_box(n - n // 2, (0.4, 0.55), (0.4, 0.4), 3, (0.0, -20.0), 1.0,
                               ((0.2, 0.8, 0), (0.1, 0.9, 1), (0.03, 0.97, 2)))]
        sim = AdaptiveGIMP(2, 4, 64, n, di.random_initializer(boxes, seed=3), None)
    else:
        boxes = di.reference_boxes_3d(n)
        bands = ((0.05, 0.95, 0), (0.01, 0.99, 1))
        rboxes = [R.random_box(25000, (0.2, 0.1, 0.2), (0.3, 0.3, 0.3), 2, (0.0, 20.0, 0.0), 1.0, bands),
                  R.random_box(n - 25000, (0.2, 0.5, 0.2), (0.3, 0.3, 0.3), 2, (0.0, -20.0, 0.0), 1.0, bands)]
        sim = AdaptiveGIMP(3, 3, 16, n, di.random_initializer(boxes, seed=3), None)
    want = R.random_fill(dim, rboxes, seed=3)
    _check_state(sim, want, dim)
    sim.substep(1e-5)
    assert sim.errors() == 0
    sim.close()


@pytest.mark.parametrize("dim,level,coarsest,rule", [
    (2, 4, 16, 1), (2, 4, 16, 2), (2, 3, 16, 3), (2, 4, 16, 4), (2, 4, 16, 5), (3, 4, 4, 5), (3, 3, 8, 3),
])
def test_level_map_rules_match_host_tabulation(dim, level, coarsest, rule):
    from agimp import AdaptiveGIMP, scenes
    from agimp.simulator import tabulate_level_map
    fn = scenes.REFERENCE_MASKS[rule]
    table, H = tabulate_level_map(fn, dim, level, coarsest)
    sim = AdaptiveGIMP(dim, level, coarsest, 0, lambda s: None, fn)  # a rule number: device tabulation
    got, gh = sim.get_level_map()
    assert gh == H
    np.testing.assert_array_equal(got, table)
    sim.close()


def test_coarse_level_map_matches_host_tabulation():
    from agimp import scenes
    from agimp.simulator import tabulate_level_map
    sc = scenes.make_config(1)
    gi = sc.grid_initializer
    table, H = tabulate_level_map(gi, 2, sc.level, sc.coarsest)
    sim = sc.build()  # the band map carries its coarse levels: device expansion
    got, gh = sim.get_level_map()
    assert gh == H
    np.testing.assert_array_equal(got, table)
    sim.close()
    gi3 = scenes.band_level_map([((0.3, 0.2, 0.3), (0.6, 0.5, 0.45))], 3, 3, 16)
    table3, H3 = tabulate_level_map(gi3, 3, 3, 16)
    from agimp import AdaptiveGIMP
    sim3 = AdaptiveGIMP(3, 3, 16, 0, lambda s: None, gi3)
    got3, _ = sim3.get_level_map()
    np.testing.assert_array_equal(got3, table3)
    sim3.close()


def test_device_scene_runs_like_host_scene():
    # the device-generated config 3 at small scale steps without errors and
    # keeps its particles inside the domain
    from agimp import scenes
    sc = scenes.make_device_config(3, seed=1, scale=0.3)
    sim = sc.build()
    assert sim.n_particles == sc.n > 1000
    for i in range(20):
        if i % sc.refine_every == 0:
            sim.refine_levels(sc.refine_band)
        sim.substep(sc.dt)
    x = sim.x_p.to_numpy()
    assert sim.errors() == 0 and np.isfinite(x).all() and (x > 0).all() and (x < 1).all()
    sim.close()


def test_device_generation_is_faster_than_host_generation():
    # config 3 at full size (1.9M particles): numpy generation plus upload
    # against generation on the GPU (both include creating the simulator)
    import time

    import torch

    from agimp import scenes
    t0 = time.perf_counter()
    host = scenes.make_config(3)
    hs = host.build()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    dsc = scenes.make_device_config(3)
    ds = dsc.build()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    print("config 3: host generation + upload %.3f s (%d particles), device generation %.3f s (%d particles)"
          % (t1 - t0, host.n, t2 - t1, dsc.n))
    assert abs(dsc.n - host.n) < 0.01 * host.n
    assert t2 - t1 < t1 - t0
    hs.close()
    ds.close()
