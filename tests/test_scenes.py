"""Host logic: level-map tabulation and the scene generators."""
import numpy as np
import pytest

from _golden_util import load, scenes as golden_scenes


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_reference_masks_match_reference_source(k):
    """The vectorised init.py masks tabulate to exactly the table the golden
    generator obtained by calling the reference's own initialize_maskK."""
    from agimp import scenes
    from agimp.simulator import tabulate_level_map
    z = load("static2d_mask%d" % k)
    table, H = tabulate_level_map(scenes.REFERENCE_MASKS[k], int(z["dim"]), int(z["level"]), int(z["coarsest"]))
    assert H == int(z["map_halo"])
    np.testing.assert_array_equal(table, z["level_map"])


def test_scalar_initializer_tabulation_matches_vectorised():
    from agimp import scenes
    from agimp.simulator import tabulate_level_map

    def mask3_scalar(sim, I):  # init.py:51-64 in the reference's scalar form
        sz = sim.finest_size
        inner = all(8 <= i < sz - 8 for i in I)
        if I[0] < sz / 4 and inner:
            sim.activate_cell(0, I)
            return 0
        if I[0] < sz / 2 and inner:
            sim.activate_cell(1, I)
            return 1
        sim.activate_cell(2, I)
        return 2

    a, Ha = tabulate_level_map(mask3_scalar, 2, 4, 8)
    b, Hb = tabulate_level_map(scenes.initialize_mask3, 2, 4, 8)
    assert Ha == Hb
    np.testing.assert_array_equal(a, b)


def test_bad_initializer_rejected():
    from agimp.simulator import tabulate_level_map

    def bad(sim, I):
        sim.activate_cell(0, I)  # activates a different level than it returns
        return 1

    with pytest.raises(ValueError):
        tabulate_level_map(bad, 2, 2, 4)


@pytest.mark.parametrize("k,lo,hi", [(1, 18000, 24000), (2, 60000, 160000), (3, 1_800_000, 2_000_000)])
def test_config_sizes(k, lo, hi):
    from agimp import scenes
    s = scenes.make_config(k)
    assert lo <= s.n <= hi
    assert s.x.dtype == np.float32 and np.all((s.x > 0) & (s.x < 1))


def test_config_seeded():
    from agimp import scenes
    a = scenes.make_config(2, seed=3)
    b = scenes.make_config(2, seed=3)
    np.testing.assert_array_equal(a.x, b.x)


def test_band_level_map_is_aligned_to_coarse_cells():
    """Every coarsest cell maps to a single level, so no activated cell can
    have an activated ancestor (static mode has no culling,
    adaptive_gimp.py:328-329)."""
    from agimp import scenes
    from agimp.simulator import tabulate_level_map
    s = scenes.make_config(1, scale=0.5)
    table, H = tabulate_level_map(s.grid_initializer, 2, s.level, s.coarsest)
    inner = table[H:-H, H:-H] & 15
    k = 1 << (s.level - 1)
    blocks = inner.reshape(s.coarsest, k, s.coarsest, k)
    assert np.all(blocks.min(axis=(1, 3)) == blocks.max(axis=(1, 3)))


def test_batch_config_shapes():
    """Config 4: 256 scenes, 2-4 levels, finest 256 or 512, 1-3 boxes that do
    not overlap, lognormal particle counts clipped to [2k, 60k]."""
    from agimp import scenes
    sc = scenes.make_batch_config()
    assert len(sc) == 256
    n = np.array([s.n for s in sc])
    assert n.min() >= 1900 and n.max() <= 61000  # the fill rounds the clipped target
    assert 2e6 < n.sum() < 8e6
    assert set(s.level for s in sc) == {2, 3, 4}
    assert set(s.coarsest << (s.level - 1) for s in sc) == {256, 512}
    for s in sc:
        assert s.dim == 2 and s.dt == 1e-4 and s.grid_initializer is not None
        assert np.all((s.x >= 0.1) & (s.x < 0.9))
        # 4 particles per finest cell; boxes do not overlap, so only cells that
        # two neighbouring boxes share at their edges hold more
        fin = s.coarsest << (s.level - 1)
        cells = np.floor(s.x * fin).astype(np.int64)
        _, counts = np.unique(cells[:, 0] * fin + cells[:, 1], return_counts=True)
        assert counts.max() <= 8 and (counts > 4).mean() < 0.02
    # seeded: the same call gives the same scenes
    again = scenes.make_batch_config(n_scenes=3)
    for a, b in zip(sc[:3], again):
        np.testing.assert_array_equal(a.x, b.x)
