"""The CPU oracle against golden vectors produced by the reference's own
adaptive_gimp.py / utils.py / init.py (run under tests/golden/taichi_shim).

Each substep starts from the fixture's state before it, so the grid and
topology of every step are compared from identical inputs.  Topology
(cell_mask, node_mask, fl_p) must match bit-exactly; floats within f32
rounding differences (the shim and the oracle sum in different orders and
use different SVD routines).
"""
import numpy as np
import pytest

import oracle as O
from _golden_util import LO, grid_v_close, load, node_norm, rel_close, scenes, step_input

RTOL = 1e-5
# grid velocities divide momentum by small nodal masses (adaptive_gimp.py:282),
# which amplifies summation-order rounding at light nodes (checked through
# their momentum, _golden_util.grid_v_close)
RTOL_GRID_V = 1e-4


@pytest.mark.parametrize("name", scenes())
def test_oracle_matches_reference_golden(name):
    z = load(name)
    dim, L, c = int(z["dim"]), int(z["level"]), int(z["coarsest"])
    n = len(z["x0"])
    for s in range(int(z["steps"])):
        o = O.Oracle(dim, L, c, n)
        if "level_map" in z:
            o.set_level_map(z["level_map"], int(z["map_halo"]))
        st = step_input(z, s)
        o.set_particles(st["x"], st["v"], st["F"], st["C"], z["m0"], z["g0"])
        o.substep(float(z["dt"]))
        assert o.errors() == 0
        pre = "s%d_" % s
        p = o.particles()
        np.testing.assert_array_equal(p["fl"], z[pre + "fl"])
        np.testing.assert_array_equal(node_norm(o.node_mask()), node_norm(z[pre + "node_mask"]))
        for l in range(L):
            m, v, cell = o.grid(l, LO, (c << l) + 12)
            np.testing.assert_array_equal(cell, z[pre + "cell%d" % l])
            ok, r = rel_close(m, z[pre + "m%d" % l], RTOL)
            assert ok, (s, l, "m", r)
            ok, r = grid_v_close(v, z[pre + "v%d" % l], z[pre + "m%d" % l], RTOL_GRID_V)
            assert ok, (s, l, "v", r)
        for k in "xvFC":
            ok, r = rel_close(p[k], z[pre + k], RTOL)
            assert ok, (s, k, r)


def test_golden_scenes_exercise_topology():
    """The fixtures contain culling, ghost cells, ghost nodes and T-junctions."""
    seen = dict(T=0, G=0, ghost_cell=0, multi_level=0)
    for name in scenes():
        z = load(name)
        nm = z["s0_node_mask"]
        seen["T"] += int(((nm & 4) != 0).sum())
        seen["G"] += int(((nm & 7) == 2).sum())
        L = int(z["level"])
        seen["ghost_cell"] += sum(int(((z["s0_cell%d" % l] & 2) != 0).sum()) for l in range(L))
        seen["multi_level"] += int(len(np.unique(z["s0_fl"])) > 1)
    assert all(v > 0 for v in seen.values()), seen


def test_weight_stencil_partition_of_unity():
    rng = np.random.default_rng(0)
    for dim in (2, 3):
        for _ in range(50):
            tc = rng.uniform(-0.5, 0.5, dim)
            W = O.weight_stencil(tc, 0.5, f64=True)
            assert abs(W[:, 0].sum() - 1.0) < 1e-12
            assert np.abs(W[:, 1:].sum(axis=0)).max() < 1e-12
            # linear reproduction: sum_i w_i x_i = x_p (node offsets 0..2, particle at tc+1)
            nodes = np.array(list(np.ndindex(*(3,) * dim)))[:, ::-1]  # conv (1,3,9): axis 0 fastest
            np.testing.assert_allclose((W[:, :1] * nodes).sum(axis=0), tc + 1, atol=1e-12)


def test_svd_against_numpy():
    rng = np.random.default_rng(1)
    for dim in (2, 3):
        for _ in range(200):
            A = np.eye(dim) + rng.normal(0, 0.4, (dim, dim))
            U, S, V = O.svd(A)
            np.testing.assert_allclose(U @ np.diag(S) @ V.T, A, atol=1e-12)
            np.testing.assert_allclose(U.T @ U, np.eye(dim), atol=1e-12)
            assert np.linalg.det(U) > 0 and np.linalg.det(V) > 0
            np.testing.assert_allclose(np.abs(S), np.linalg.svd(A, compute_uv=False), rtol=1e-12)


def test_stress_against_polar():
    scipy_linalg = pytest.importorskip("scipy.linalg")
    rng = np.random.default_rng(2)
    mu, la = 2083.3, 1388.9
    for dim in (2, 3):
        for _ in range(50):
            F = np.eye(dim) + rng.normal(0, 0.2, (dim, dim))
            if np.linalg.det(F) <= 0:
                continue
            R, _ = scipy_linalg.polar(F)
            J = np.linalg.det(F)
            ref = 2 * mu * (F - R) @ F.T + np.eye(dim) * la * J * (J - 1)
            np.testing.assert_allclose(O.stress(F, mu, la), ref, rtol=1e-10, atol=1e-9)
