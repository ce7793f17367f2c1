"""The numpy restatement of the device scene initialisers (oracle/init_ref.py):
Philox4x32-10 against its published known-answer vectors, the sub-lattice
against the host scene generator, and the level bands of init.py:3-32."""
import numpy as np
import pytest

import init_ref as R
from agimp import scenes

# Known-answer vectors of Philox4x32-10 published with the generator
# (Random123's kat_vectors): (counter, key) -> output.
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_philox_known_answers(ctr, key, out):
    got = R.philox(*[np.array([c]) for c in ctr], *key)
    assert tuple(int(g[0]) for g in got) == out


def test_uniforms_in_unit_interval():
    k = np.arange(100000)
    r = R.philox(k, 0, 0, 0, 7, 0)
    u = R.u53(r[0], r[1])
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01
    f = R.u24(r[2])
    assert f.dtype == np.float32 and f.min() >= 0.0 and f.max() < 1.0


@pytest.mark.parametrize("dim,shape", [
    (2, R.box((0.2, 0.3), (0.41, 0.52), 2)),
    (2, R.sphere((0.5, 0.45), 0.13, 1)),
    (3, R.box((0.1, 0.2, 0.3), (0.3, 0.33, 0.41), 0)),
    (3, R.sphere((0.5, 0.6, 0.5), 0.09, 2)),
])
def test_lattice_without_jitter_is_the_host_lattice(dim, shape):
    finest = 64
    got = R.lattice_fill(dim, finest, [shape], jitter=False)
    if shape["kind"] == "box":
        region = scenes.box_region(shape["lo"], shape["hi"])
    else:
        region = scenes.sphere_region(shape["centre"], shape["radius"])
    want = scenes.fill_lattice(None, dim, finest, *region, per_axis=2, jitter=False)
    assert len(want) > 100
    np.testing.assert_array_equal(got["x"], want)
    assert (got["g"] == shape["level"]).all()


def test_jittered_lattice_stays_near_its_points():
    finest, per = 32, 2
    h = 1.0 / (finest * per)
    shapes = [R.box((0.2, 0.2, 0.2), (0.5, 0.4, 0.45), 1, velocity=(1.0, 2.0, 3.0)),
              R.sphere((0.7, 0.7, 0.7), 0.12, 0, mass=2.0)]
    a = R.lattice_fill(3, finest, shapes, seed=5)
    b = R.lattice_fill(3, finest, shapes, seed=5)
    c = R.lattice_fill(3, finest, shapes, seed=6)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert len(c["x"]) != len(a["x"]) or not np.array_equal(c["x"], a["x"])
    # each point within half a sub-spacing of a sub-lattice centre
    frac = a["x"].astype(np.float64) / h - 0.5
    assert np.abs(frac - np.round(frac)).max() <= 0.5 + 1e-4
    # counts near the volumes times the density
    n_box = (a["g"] == 1).sum()
    assert abs(n_box - 0.3 * 0.2 * 0.25 / h ** 3) < 0.02 * n_box
    n_sph = (a["g"] == 0).sum()
    assert abs(n_sph - 4.0 / 3.0 * np.pi * 0.12 ** 3 / h ** 3) < 0.03 * n_sph
    assert (a["v"][a["g"] == 1] == np.float32([1, 2, 3])).all() and (a["m"][a["g"] == 0] == 2.0).all()


def test_random_fill_reference_bands():
    # init.py:3-32 case 0: two boxes, levels 0..3 by the position in the box
    n = 200000
    bands = ((0.2, 0.8, 0), (0.1, 0.9, 1), (0.03, 0.97, 2))
    boxes = [R.random_box(n // 2, (0.2, 0.1), (0.4, 0.4), 3, (0.0, 20.0), 1.0, bands),
             R.random_box(n - n // 2, (0.4, 0.55), (0.4, 0.4), 3, (0.0, -20.0), 1.0, bands)]
    p = R.random_fill(2, boxes, seed=1)
    x, g = p["x"], p["g"]
    first, second = x[: n // 2], x[n // 2:]
    assert first[:, 0].min() >= 0.2 - 1e-6 and first[:, 1].min() >= 0.1 - 1e-6
    assert first[:, 0].max() <= 0.6 and first[:, 1].max() <= 0.5
    assert second[:, 0].min() >= 0.4 and second[:, 1].min() >= 0.55 - 1e-6
    assert (p["v"][: n // 2, 1] == 20.0).all() and (p["v"][n // 2:, 1] == -20.0).all()
    frac = np.bincount(g, minlength=4) / n
    want = [0.6 ** 2, 0.8 ** 2 - 0.6 ** 2, 0.94 ** 2 - 0.8 ** 2, 1 - 0.94 ** 2]
    np.testing.assert_allclose(frac, want, atol=0.01)
    # the band test on the box-relative coordinate, as in the reference's if chain
    u = (first - np.float32([0.2, 0.1])) / np.float32(0.4)
    inner = np.all((u > 0.2 + 1e-4) & (u < 0.8 - 1e-4), axis=1)
    assert (g[: n // 2][inner] == 0).all()
    outer = np.any((u < 0.03 - 1e-4) | (u > 0.97 + 1e-4), axis=1)
    assert (g[: n // 2][outer] == 3).all()
