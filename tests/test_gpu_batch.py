"""Batches (config 4 path) and launch tuning.

* A batch of heterogeneous scenes (2-4 levels, 256^2-512^2, static maps, a
  dynamic scene, an empty scene) stepped by shared launches matches the same
  scenes stepped one at a time, and one of its scenes matches the oracle.
* Every P2G work-item size and grid width gives the oracle's result.
* The autotuner leaves the simulation where it was.
"""
import numpy as np
import pytest

import oracle as O
from _gpu_util import gpu_state, have_gpu, oracle_kwargs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


def _batch_scenes():
    from agimp import scenes
    sc = scenes.make_batch_config(seed=5, n_scenes=5, scale=0.2)
    sc.append(scenes.make_config(2, seed=1, scale=0.25))  # dynamic, 4 levels, snow
    empty = scenes.make_batch_config(seed=6, n_scenes=1, scale=0.2)[0]
    empty.x, empty.v, empty.g, empty.m = empty.x[:0], empty.v[:0], empty.g[:0], empty.m[:0]
    sc.append(empty)
    return sc


def _step(sim, sc, i0, n):
    for i in range(i0, i0 + n):
        if sc.refine_every and i % sc.refine_every == 0:
            sim.refine_levels(sc.refine_band)
        sim.substep(sc.dt)


def _oracles(scene):
    from agimp.simulator import tabulate_level_map
    d, n = scene.dim, scene.n
    kw = oracle_kwargs(scene.sim_kwargs, d)
    orcs = [O.Oracle(d, scene.level, scene.coarsest, n, f64=f, **kw) for f in (False, True)]
    for o in orcs:
        o.set_particles(scene.x, scene.v, np.tile(np.eye(d), (n, 1, 1)), np.zeros((n, d, d)), scene.m, scene.g)
        if scene.grid_initializer is not None:
            t, H = tabulate_level_map(scene.grid_initializer, d, scene.level, scene.coarsest)
            o.set_level_map(t, H)
    return orcs


def _against_oracle(sim, scene, orcs):
    g = gpu_state(sim)
    p32, p64 = orcs[0].particles(), orcs[1].particles()
    np.testing.assert_array_equal(g["fl"], p32["fl"])
    disp = np.sqrt(((p64["x"] - scene.x) ** 2).sum(1).mean())
    e_gpu = np.sqrt(((g["x"] - p32["x"]) ** 2).sum(1).mean()) / disp
    e_floor = np.sqrt(((p32["x"] - p64["x"]) ** 2).sum(1).mean()) / disp
    assert e_gpu <= max(10 * e_floor, 1e-3), (e_gpu, e_floor)


def test_batch_matches_scenes_stepped_alone():
    """Refinement rounds of the dynamic scene happen outside the batch step
    (agimp_refine_levels on its simulator), at the same substeps in both runs."""
    from agimp.batch import SceneBatch
    sc = _batch_scenes()
    dt = sc[0].dt
    alone = [s.build() for s in sc]
    together = [s.build() for s in sc]
    batch = SceneBatch(together)
    steps = 20
    for i in range(steps):
        for k, s in enumerate(sc):
            if s.refine_every and i % s.refine_every == 0:
                alone[k].refine_levels(s.refine_band)
                together[k].refine_levels(s.refine_band)
            alone[k].substep(dt)
        batch.substep(dt)
    for k, s in enumerate(sc):
        a, b = gpu_state(alone[k]), gpu_state(together[k])
        assert alone[k].errors() & ~2 == 0 and together[k].errors() & ~2 == 0
        np.testing.assert_array_equal(a["fl"], b["fl"])
        np.testing.assert_array_equal(a["g"], b["g"])
        if s.n:
            # float atomics: both runs differ from each other in the last bits only
            assert np.abs(a["x"] - b["x"]).max() <= 1e-5, (k, np.abs(a["x"] - b["x"]).max())
            assert np.abs(a["v"] - b["v"]).max() <= 1e-3 * max(1.0, np.abs(a["v"]).max())
        assert together[k].stats()["substeps"] == steps
    # 10 topology and binning kernels (k_mark_hier included: one scene is
    # dynamic), P2G, G2P, the return map (one scene has snow plasticity), and
    # a restriction and a prolongation per level above 0 (grid_op runs inside
    # them)
    assert batch.kernels_per_substep() == 10 + 3 + 2 * (max(s.level for s in sc) - 1)
    batch.close()
    for s in alone + together:
        s.close()


def test_batched_scene_matches_oracle():
    from agimp.batch import SceneBatch
    sc = _batch_scenes()
    k = int(np.argmax([s.level for s in sc[:5]]))  # a static scene with the most levels
    sims = [s.build() for s in sc]
    batch = SceneBatch(sims)
    orcs = _oracles(sc[k])
    for i in range(15):
        batch.substep(sc[k].dt)
        for o in orcs:
            o.substep(sc[k].dt)
    _against_oracle(sims[k], sc[k], orcs)
    batch.close()
    for s in sims:
        s.close()


@pytest.mark.parametrize("chunk,cps", [(64, 2), (128, 4), (256, 16), (512, 8), (64, 32)])
@pytest.mark.parametrize("k,scale", [(1, 0.35), (3, 0.3)])
def test_tuning_choices_match_oracle(chunk, cps, k, scale):
    from agimp import scenes
    scene = scenes.make_config(k, scale=scale)
    sim = scene.build()
    sim.set_tuning(chunk, cps)
    assert sim.tuning["chunk"] == chunk and sim.tuning["ctas_per_sm"] == cps
    orcs = _oracles(scene)
    steps = 10
    for i in range(steps):
        if scene.refine_every and i % scene.refine_every == 0:
            sim.refine_levels(scene.refine_band)
            for o in orcs:
                o.refine_levels(scene.refine_band)
        sim.substep(scene.dt)
        for o in orcs:
            o.substep(scene.dt)
    assert sim.errors() & ~2 == 0
    _against_oracle(sim, scene, orcs)
    sim.close()


def test_autotune_restores_state_and_batch_autotune():
    from agimp import scenes
    from agimp.batch import SceneBatch
    scene = scenes.make_config(3, scale=0.3)
    sim = scene.build()
    _step(sim, scene, 0, 5)
    before = gpu_state(sim)
    n0 = sim.stats()["substeps"]
    best = sim.autotune(scene.dt, trials=2)
    assert best["chunk"] in (64, 128, 256, 512) and best["ctas_per_sm"] in (2, 4, 8, 16) and best["ms_per_substep"] > 0
    assert sim.tuning["chunk"] == best["chunk"]
    after = gpu_state(sim)
    for key in before:
        np.testing.assert_array_equal(before[key], after[key])
    assert sim.stats()["substeps"] == n0
    assert sim.errors() & ~2 == 0
    _step(sim, scene, 5, 3)  # keeps stepping normally
    assert sim.stats()["substeps"] == n0 + 3
    sim.close()

    sc = _batch_scenes()
    sims = [s.build() for s in sc]
    batch = SceneBatch(sims)
    batch.substep(sc[0].dt, 3)
    xs = [s.x_p.to_numpy() for s in sims]
    t = batch.autotune(sc[0].dt, trials=2)
    assert t["ms_per_substep"] > 0 and batch.tuning["chunk"] == t["chunk"]
    for s, x in zip(sims, xs):
        np.testing.assert_array_equal(s.x_p.to_numpy(), x)
    batch.substep(sc[0].dt, 2)
    batch.close()
    for s in sims:
        s.close()


def test_batch_rejects_mixed_dims_and_uses_its_own_surrogate_setting():
    """A scene's own surrogate setting applies when it steps alone; in a batch
    of several the batch's setting (agimp_batch_set_surrogate) applies."""
    from agimp import AgimpError, scenes
    from agimp.batch import SceneBatch
    from agimp.surrogate import MLP
    a = scenes.make_config(2, scale=0.2).build()
    b = scenes.make_config(2, seed=3, scale=0.2).build()
    c3 = scenes.make_config(3, scale=0.2).build()
    with pytest.raises(AgimpError):
        SceneBatch([a, c3])
    with pytest.raises(AgimpError):
        SceneBatch([a, a])
    batch = SceneBatch([a, b])
    mlp = MLP()
    a.set_surrogate(mlp, xmax=np.ones(7, np.float32), tol=0.1)
    batch.substep(5e-5)  # the scene's own setting is not the batch's
    assert batch.surrogate_stats()["handed_off"] == 0
    with pytest.raises(AgimpError):
        batch.set_surrogate(mlp, xmax=np.ones(7, np.float32), tol=0.0)
    a.set_surrogate(None)
    batch.substep(5e-5)
    batch.close()
    for s in (a, b, c3):
        s.close()


def test_async_readback_overlaps_next_substep():
    """x_p read asynchronously on a copy stream while the following substeps
    run on another stream equals the state a blocking read returns at the
    same substep (the library orders the overwrite after the copy)."""
    import ctypes

    import torch

    from agimp import scenes
    sc = scenes.make_config(3, scale=0.3)
    a, b = sc.build(), sc.build()
    main_s, copy_s = torch.cuda.Stream(), torch.cuda.Stream()
    sm, scp = ctypes.c_void_p(main_s.cuda_stream), ctypes.c_void_p(copy_s.cuda_stream)
    steps = 12
    outs = [torch.empty((sc.n, 3), dtype=torch.float32, pin_memory=True).numpy() for _ in range(steps)]
    ref = []
    for i in range(steps):
        if i % sc.refine_every == 0:
            a.refine_levels(sc.refine_band, stream=sm)
            b.refine_levels(sc.refine_band)
        a.substep(sc.dt, stream=sm)
        a.x_p.to_numpy(out=outs[i], blocking=False, stream=scp)
        b.substep(sc.dt)
        ref.append(b.x_p.to_numpy())
    copy_s.synchronize()
    main_s.synchronize()
    for i in range(steps):
        assert np.abs(outs[i] - ref[i]).max() <= 1e-5, (i, np.abs(outs[i] - ref[i]).max())
    assert a.stats()["substeps"] == steps
    a.close()
    b.close()


def test_batch_positions_readback():
    """One gathered copy of all scenes' positions equals the per-simulator
    readbacks, also when taken asynchronously while the batch keeps stepping."""
    import ctypes

    import torch

    from agimp.batch import SceneBatch
    sc = _batch_scenes()[:5] + [_batch_scenes()[6]]  # static scenes and the empty one
    sims = [s.build() for s in sc]
    batch = SceneBatch(sims)
    batch.substep(sc[0].dt, 3)
    whole = batch.positions()
    np.testing.assert_array_equal(whole, np.concatenate([s.x_p.to_numpy() for s in sims]))
    main_s, copy_s = torch.cuda.Stream(), torch.cuda.Stream()
    sm, scp = ctypes.c_void_p(main_s.cuda_stream), ctypes.c_void_p(copy_s.cuda_stream)
    outs = [torch.empty(whole.shape, dtype=torch.float32, pin_memory=True).numpy() for _ in range(4)]
    ref = [s.build() for s in sc]
    rbatch = SceneBatch(ref)
    rbatch.substep(sc[0].dt, 3)
    refs = []
    for i in range(4):
        batch.substep(sc[0].dt, stream=sm)
        batch.positions(out=outs[i], blocking=False, stream=scp)
        rbatch.substep(sc[0].dt)
        refs.append(rbatch.positions())
    copy_s.synchronize()
    main_s.synchronize()
    for i in range(4):
        assert np.abs(outs[i] - refs[i]).max() <= 1e-5, i
    batch.close()
    rbatch.close()
    for s in sims + ref:
        s.close()


def test_async_readbacks_follow_uploads_and_refinements():
    """Asynchronous readbacks run their gathers on the library's own stream:
    an upload or a refinement issued between two readbacks (on any stream)
    is seen by the second readback and not by the first."""
    import ctypes

    import torch

    from agimp import scenes
    sc = scenes.make_config(3, scale=0.3)
    sim = sc.build()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    p1, p2 = ctypes.c_void_p(s1.cuda_stream), ctypes.c_void_p(s2.cuda_stream)
    n = sc.n
    sim.refine_levels(sc.refine_band, stream=p1)
    sim.substep(sc.dt, stream=p1)
    before = [torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    after = [torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    g_before = torch.empty((n,), dtype=torch.int32, pin_memory=True).numpy()
    g_after = torch.empty((n,), dtype=torch.int32, pin_memory=True).numpy()
    sim.x_p.to_numpy(out=before[0], blocking=False, stream=p2)
    sim.g_p.to_numpy(out=g_before, blocking=False, stream=p2)
    x_new = (sim.x_p.to_numpy() * np.float32(0.5) + np.float32(0.25)).astype(np.float32)
    sim.x_p.from_numpy(x_new)  # upload on the library's stream
    sim.x_p.to_numpy(out=after[0], blocking=False, stream=p2)
    sim.refine_levels(2, stream=p1)  # another band: other prescribed levels
    sim.g_p.to_numpy(out=g_after, blocking=False, stream=p2)
    s1.synchronize()
    s2.synchronize()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(after[0], x_new)
    assert not np.array_equal(before[0], x_new)
    ref = sc.build()
    ref.x_p.from_numpy(x_new)
    ref.refine_levels(2)
    np.testing.assert_array_equal(g_after, ref.g_p.to_numpy())
    assert not np.array_equal(g_before, g_after)
    ref.close()
    sim.close()


def test_batch_upload_equals_per_scene_uploads():
    """agimp_batch_set_particles with every scene's arrays concatenated in
    batch order leaves each scene exactly as agimp_set_particles on each
    would, also while an asynchronous positions readback is pending, and
    the batch then steps to the same positions (up to the order of float
    additions)."""
    import ctypes

    import torch

    from agimp.batch import SceneBatch
    sc = _batch_scenes()[:5] + [_batch_scenes()[6]]  # static scenes and the empty one
    a_sims = [s.build() for s in sc]
    b_sims = [s.build() for s in sc]
    a, b = SceneBatch(a_sims), SceneBatch(b_sims)
    a.substep(sc[0].dt, 2)
    b.substep(sc[0].dt, 2)
    rng = np.random.default_rng(3)
    ups = []
    for s in sc:
        n, d = s.n, s.dim
        ups.append(dict(x=(rng.uniform(0.3, 0.7, (n, d))).astype(np.float32),
                        v=rng.normal(0, 1, (n, d)).astype(np.float32),
                        F=(np.eye(d) + 0.01 * rng.normal(0, 1, (n, d, d))).astype(np.float32),
                        C=(0.1 * rng.normal(0, 1, (n, d, d))).astype(np.float32),
                        m=rng.uniform(0.5, 1.5, n).astype(np.float32),
                        g=rng.integers(0, s.level, n).astype(np.int32),
                        Jp=rng.uniform(0.9, 1.1, n).astype(np.float32)))
    for sim, u in zip(a_sims, ups):
        sim.set_particles(**u)
    copy_s = torch.cuda.Stream()
    pend = torch.empty((b.n_particles, 2), dtype=torch.float32, pin_memory=True).numpy()
    b.positions(out=pend, blocking=False, stream=ctypes.c_void_p(copy_s.cuda_stream))
    cat = {k: np.concatenate([u[k] for u in ups]) for k in ups[0]}
    b.set_particles(**cat)
    copy_s.synchronize()
    for sa, sb in zip(a_sims, b_sims):
        ga, gb = gpu_state(sa), gpu_state(sb)
        for k in ga:
            np.testing.assert_array_equal(ga[k], gb[k], err_msg=k)
    a.substep(sc[0].dt, 3)
    b.substep(sc[0].dt, 3)
    for sa, sb in zip(a_sims, b_sims):
        # float atomics: the two runs differ in the last bits only
        xa, xb = sa.x_p.to_numpy(), sb.x_p.to_numpy()
        assert xa.size == 0 or np.abs(xa - xb).max() <= 1e-5
    with pytest.raises(ValueError):
        b.set_particles(x=cat["x"][:-1])
    a.close()
    b.close()
    for s in a_sims + b_sims:
        s.close()
