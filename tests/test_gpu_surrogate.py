"""Surrogate return map inside the substep (extension; the reference has no
plasticity): the G2P recorder, the hand-off to the tensor-core MLP and the
finishing kernel with its fallback to the exact (SVD) return map.

* The recorder's pairs equal the exact clamp of the recorded trial state,
  decoded from the stored features and recomputed here in numpy.
* With a network whose every prediction is rejected, the surrogate path must
  reproduce the plain path (every handed-off particle falls back to the same
  SVD clamp, written with explicitly rounded operations) up to the run-to-run
  noise of P2G's float atomics: this pins the slot and metadata plumbing.
* A network trained on the GPU (tensor-core forward/backward) from recorded
  pairs of a small 2D snow scene runs the same scene; its position error
  against the plain run stays within a stated bound, and the test reports the
  share of projections the network handles and the time of both runs (what
  the trained network gains over the method without it).
"""
import time

import numpy as np
import pytest

from _gpu_util import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]

SIG, LJ, HSC = 0.05, 0.5, 5.0  # feature scales of the network's inputs
DSIG, DLJ = 0.02, 0.02  # output scales (changes of sig and log Jp)


def _scene():
    """Two 2D snow boxes (the 4-level, 64^2..512^2 dynamic snow material and
    time step) thrown at each other at +-3: most particles yield within a
    hundred substeps."""
    from agimp import scenes
    base = scenes.make_config(2, seed=3, scale=0.5)
    rng = np.random.default_rng(7)
    fin = base.coarsest << (base.level - 1)
    boxes = (((0.30, 0.40), (0.44, 0.54), 3.0), ((0.46, 0.42), (0.60, 0.56), -3.0))
    xs, vs = [], []
    for lo, hi, u in boxes:
        pts = scenes.fill_lattice(rng, 2, fin, *scenes.box_region(lo, hi))
        xs.append(pts)
        vs.append(np.tile(np.array([u, 0.0], np.float32), (len(pts), 1)))
    x, v = np.concatenate(xs), np.concatenate(vs)
    n = len(x)
    return scenes.Scene("colliding_snow_boxes_2d", 2, base.level, base.coarsest, x, v,
                        np.full(n, base.level - 1, np.int32), np.ones(n, np.float32), base.dt, 400,
                        dict(base.sim_kwargs), refine_every=10, refine_band=3)


def _run(sim, sc, steps):
    for i in range(steps):
        if sc.refine_every and i % sc.refine_every == 0:
            sim.refine_levels(sc.refine_band)
        sim.substep(sc.dt)


def _state(sim):
    # readback is in the caller's particle order (the library tracks ids)
    return sim.x_p.to_numpy(), sim.F_p.to_numpy(), sim.Jp.to_numpy()


def test_recorder_pairs_are_the_exact_clamp():
    import torch
    sc = _scene()
    sim = sc.build()
    cap = 200_000
    X = torch.full((cap, 7), np.nan, dtype=torch.float32, device="cuda")
    T = torch.full((cap, 4), np.nan, dtype=torch.float32, device="cuda")
    sim.set_recorder(X, T, 1)
    _run(sim, sc, 100)
    n = min(sim.recorded(), cap)
    assert n > 10000, n
    assert sim.errors() == 0
    x = X[:n].cpu().numpy().astype(np.float64)
    t = T[:n].cpu().numpy().astype(np.float64)
    assert np.isfinite(x).all() and np.isfinite(t).all()
    p = sim._params
    tc, ts, xi = p.theta_c, p.theta_s, p.hardening
    sig = 1.0 + SIG * x[:, :2]
    jp = np.exp(LJ * x[:, 3])
    assert np.all(np.abs(x[:, 2]) == 0.0)  # 2D: third singular value unused
    np.testing.assert_allclose(x[:, 4], xi * (1.0 - jp) / HSC, atol=2e-5)
    np.testing.assert_allclose(x[:, 5], tc / 0.025 - 1.0, atol=1e-6)
    np.testing.assert_allclose(x[:, 6], ts / 0.0075 - 1.0, atol=1e-6)
    cl = np.clip(sig, 1.0 - tc, 1.0 + ts)
    # features pass through f32 (sig - 1) / 0.05: a few ulp of 1 after decoding
    np.testing.assert_allclose(t[:, :2], (cl - sig) / DSIG, atol=5e-5)
    assert np.all(t[:, 2] == 0.0)
    np.testing.assert_allclose(t[:, 3], np.log(sig.prod(1) / cl.prod(1)) / DLJ, atol=1e-4)
    # elastic directions have no change at all
    inside = (sig > 1.0 - tc + 1e-6) & (sig < 1.0 + ts - 1e-6)
    assert np.all(np.abs(t[:, :2][inside]) < 5e-5)
    # the recorded states are plastic ones: at least one value lies outside
    # the elastic interval for most of them (the skip test is conservative)
    outside = ((sig < 1.0 - tc) | (sig > 1.0 + ts)).any(1)
    assert outside.mean() > 0.5, outside.mean()
    # stride 4 records about a quarter as many
    sim.recorded(reset=True)
    sim.set_recorder(X, T, 4)
    _run(sim, sc, 10)
    assert 0 < sim.recorded() < n
    sim.close()


def _gap(a, b):
    """RMS difference (over particles and components) of positions,
    deformation gradients and log Jp."""
    return tuple(float(np.sqrt(np.mean((np.asarray(u, np.float64) - np.asarray(v, np.float64)) ** 2)))
                 for u, v in zip((a[0], a[1], np.log(a[2])), (b[0], b[1], np.log(b[2]))))


def _within_floor(gap, floors, what):
    # P2G accumulates with float atomics, so two runs of the same path differ
    # in the last bits, and after the collision the difference grows by orders
    # of magnitude within tens of substeps, for a few particles far more than
    # for the rest: compare RMS differences against the larger one between
    # the reference run and two more plain runs (20x, plus one f32 ulp of 1).
    # A wrong return map on the handed-off particles moves the RMS by far more.
    for k, name in enumerate(("x", "F", "log Jp")):
        f = max(fl[k] for fl in floors)
        assert gap[k] <= 20.0 * f + 1.2e-7, (what, name, gap[k], f)


def test_rejected_predictions_reproduce_plain_path():
    from agimp.surrogate import MLP
    sc = _scene()
    a, b, b2, sur = sc.build(), sc.build(), sc.build(), sc.build()
    mlp = MLP(seed=1)  # untrained: its predictions break the residual test
    sur.set_surrogate(mlp, xmax=np.full(7, 1e6, np.float32), tol=1e-12)
    for sim in (a, b, b2, sur):
        _run(sim, sc, 90)  # the boxes touch after about 70 substeps
    st = sur.stats()
    assert st["n_surrogate"] > 0
    assert st["n_fallback"] == st["n_surrogate"], st
    assert a.errors() == 0 and sur.errors() == 0 and mlp.errors() == 0
    ref = _state(a)
    _within_floor(_gap(_state(sur), ref), [_gap(_state(b), ref), _gap(_state(b2), ref)], "all rejected")
    for sim in (a, b, b2, sur):
        sim.close()


def test_out_of_range_features_take_exact_path():
    from agimp.surrogate import MLP
    sc = _scene()
    a, b, b2, sur = sc.build(), sc.build(), sc.build(), sc.build()
    mlp = MLP(seed=2)
    sur.set_surrogate(mlp, xmax=np.full(7, 1e-9, np.float32), tol=0.5)  # nothing is in range
    for sim in (a, b, b2, sur):
        _run(sim, sc, 90)
    assert sur.stats()["n_surrogate"] == 0
    ref = _state(a)
    _within_floor(_gap(_state(sur), ref), [_gap(_state(b), ref), _gap(_state(b2), ref)], "out of range")
    for sim in (a, b, b2, sur):
        sim.close()


def test_trained_surrogate_against_plain():
    import torch

    from agimp.surrogate import MLP, evaluate, record_pairs, train, trained_range
    sc = _scene()
    X, T = record_pairs(sc, 4_000_000, stride=1, max_substeps=sc.steps)
    n = X.shape[0]
    assert n > 500_000, n
    perm = torch.randperm(n, device=X.device, generator=torch.Generator(device=X.device).manual_seed(0))
    nv = n // 20
    Xv, Tv = X[perm[:nv]].contiguous(), T[perm[:nv]].contiguous()
    Xt, Tt = X[perm[nv:]].contiguous(), T[perm[nv:]].contiguous()
    mlp = MLP(seed=0)
    mse0, _ = evaluate(mlp, Xv, Tv)
    train(mlp, Xt, Tt, steps=6000, batch=32768, lr=3e-3, lr_final=2e-4)
    mse, mx = evaluate(mlp, Xv, Tv)
    assert mlp.errors() == 0
    assert mse < 0.05 * mse0, (mse0, mse)
    xmax = trained_range(Xt)

    steps = 300
    plain, sur = sc.build(), sc.build()
    sur.set_surrogate(mlp, xmax=xmax, tol=1e-3)
    times = {}
    for name, sim in (("plain", plain), ("surrogate", sur)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _run(sim, sc, steps)
        torch.cuda.synchronize()
        times[name] = time.perf_counter() - t0
    # counts are per substep: sum them over a few more substeps of both runs
    st = dict(n_surrogate=0, n_fallback=0)
    for i in range(20):
        for sim in (plain, sur):
            if i % sc.refine_every == 0:
                sim.refine_levels(sc.refine_band)
            sim.substep(sc.dt)
        s = sur.stats()
        st["n_surrogate"] += s["n_surrogate"]
        st["n_fallback"] += s["n_fallback"]
    steps += 20
    assert plain.errors() == 0 and sur.errors() == 0 and mlp.errors() == 0
    xp, _, jpp = _state(plain)
    xs, _, jps = _state(sur)
    dx = np.abs(xs - xp).max()
    mdx = np.abs(xs - xp).mean()
    djp = np.abs(np.log(jps) - np.log(jpp)).max()
    share = 1.0 - st["n_fallback"] / max(st["n_surrogate"], 1)
    print("surrogate: val_mse %.3g (untrained %.3g) max %.3g; handled %.3f of %d projections; "
          "max |dx| %.3g mean %.3g, max |dlog Jp| %.3g after %d substeps; plain %.3fs surrogate %.3fs (x%.2f)"
          % (mse, mse0, mx, share, st["n_surrogate"], dx, mdx, djp, steps, times["plain"], times["surrogate"],
             times["plain"] / times["surrogate"]))
    assert st["n_surrogate"] > 0
    assert share > 0.9, st
    # position error over the unit domain after 320 substeps (measured: max
    # about 5e-4, mean about 6e-5; two plain runs differ by about 3e-6, 3e-8)
    assert dx < 5e-3 and mdx < 5e-4, (dx, mdx)
    plain.close()
    sur.close()
    mlp.close()


def test_batched_surrogate_matches_scenes_alone():
    """A batch of several snow scenes with one shared surrogate (one MLP
    launch per substep over every scene's projections) gives each scene what
    it gets stepping alone with the same network, up to the run-to-run noise
    of P2G's float atomics; the batch hands projections to the network."""
    import os

    from agimp.batch import SceneBatch
    from agimp.surrogate import load
    wpath = os.path.join(os.path.dirname(__import__("agimp").__file__), "data", "surrogate_snow.npz")
    mlp, xmax = load(wpath)
    scs = []
    for u in (3.0, 4.0, 2.5):
        sc = _scene()
        sc.v = sc.v * np.float32(u / 3.0)
        scs.append(sc)
    alone = [sc.build() for sc in scs]
    together = [sc.build() for sc in scs]
    for s in alone:
        s.set_surrogate(mlp, xmax, 1e-3)
    batch = SceneBatch(together)
    batch.set_surrogate(mlp, xmax, 1e-3)
    handed = 0
    steps = 60
    for i in range(steps):
        for k, sc in enumerate(scs):
            if sc.refine_every and i % sc.refine_every == 0:
                alone[k].refine_levels(sc.refine_band)
                together[k].refine_levels(sc.refine_band)
            alone[k].substep(sc.dt)
        batch.substep(scs[0].dt)
        handed += batch.surrogate_stats()["handed_off"]
    st = batch.surrogate_stats()
    assert st["errors"] == 0
    assert handed > 0
    for a, b in zip(alone, together):
        assert a.errors() & ~2 == 0 and b.errors() & ~2 == 0
        xa, xb = a.x_p.to_numpy(), b.x_p.to_numpy()
        # float-atomics noise, grown through the collision: well below a
        # finest cell (2e-3); a projection applied to the wrong scene or slot
        # moves particles by cells
        assert np.abs(xa - xb).max() <= 1e-4, np.abs(xa - xb).max()
        assert np.sqrt(np.mean((xa - xb) ** 2)) <= 1e-5
    batch.close()
    for s in alone + together:
        s.close()
