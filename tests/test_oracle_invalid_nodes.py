"""The reference's grid update skips nodes that are neither activated, ghost
nor T-junction nodes (adaptive_gimp.py:280), so G2P reads their raw P2G
momentum.  With a dense body whose interior sits on a coarse level that raw
momentum sums many particles and the body blows up; the invalid_nodes =
"normalize" extension divides it by the node mass.  Shown here on the oracle
(3 levels, 16^3..64^3, a sphere of radius 0.3 at 8 particles per finest cell
moving at 3, interior on level 0): the reference form accelerates particles
to many times their speed within 8 substeps, the extension keeps them at 3."""
import numpy as np
import pytest

import oracle as O


def _sphere_run(invalid_nodes):
    from agimp import scenes
    rng = np.random.default_rng(0)
    L, c = 3, 16
    x = scenes.fill_lattice(rng, 3, c << (L - 1), *scenes.sphere_region((0.5, 0.5, 0.5), 0.3))
    n = len(x)
    v = np.tile(np.array([0.0, -3.0, 0.0]), (n, 1))
    o = O.Oracle(3, L, c, n, gravity=(0.0, -9.8, 0.0), E=250.0, nu=0.25, boundary_mode=1, plasticity=1,
                 invalid_nodes=invalid_nodes)
    o.set_particles(x, v, np.tile(np.eye(3), (n, 1, 1)), np.zeros((n, 3, 3)), np.ones(n), np.full(n, L - 1, np.int32))
    o.refine_levels(1)
    levels = np.bincount(o.particles()["g"], minlength=L)
    o.substep(5e-5, 8, 0)
    vv = np.linalg.norm(o.particles()["v"], axis=1)
    return levels, float(vv.max())


@pytest.mark.parametrize("mode", [0, 1])
def test_invalid_node_momentum(mode):
    levels, vmax = _sphere_run(mode)
    assert levels[0] > 50000  # the interior is on the coarsest level
    if mode == 0:
        assert vmax > 20.0, vmax  # reference form: blows up
    else:
        assert vmax < 3.05, vmax  # extension: stays at the initial speed
