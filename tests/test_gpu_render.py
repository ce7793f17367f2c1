"""Headless drawing (gui.py's visualize_mask and particle circles) by the CUDA
kernels against the numpy restatement in oracle/render_ref.py, on read-back
masks of real substeps: the images must be identical bit for bit."""
import numpy as np
import pytest

import render_ref as R
from _gpu_util import LO, have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


def _scene(k, scale, steps):
    from agimp import scenes
    sc = scenes.make_config(k, scale=scale)
    sim = sc.build()
    for i in range(steps):
        if sc.refine_every and i % sc.refine_every == 0:
            sim.refine_levels(sc.refine_band)
        sim.substep(sc.dt)
    return sc, sim


def _expected_mask(sim, res, show_ghost, show_node):
    cells = []
    for l in range(sim.level):
        n = (sim.coarsest_size << l) + 12
        cells.append(sim.cell_mask[l].read(LO, n))
    return R.render_mask(cells, LO, sim.node_mask.read_lattice(), sim.coarsest_size, res, show_ghost, show_node)


@pytest.mark.parametrize("k,scale,steps,res", [(1, 0.35, 3, 768), (1, 0.35, 3, 256), (2, 0.3, 12, 1536)])
@pytest.mark.parametrize("show_ghost,show_node", [(True, True), (False, True), (True, False)])
def test_mask_matches_restatement(k, scale, steps, res, show_ghost, show_node):
    from agimp.render import render_mask
    sc, sim = _scene(k, scale, steps)
    got = render_mask(sim, res, show_ghost, show_node)
    exp = _expected_mask(sim, res, show_ghost, show_node)
    np.testing.assert_array_equal(got, exp)
    # the picture shows something: activated cells (covered by the node
    # markers where the nodes are 3 pixels apart) and, with markers, nodes
    cells_seen = ((got == np.float32(R.ACT_FILL)).all(-1) | (got == np.float32(R.ACT_EDGE)).all(-1)).any()
    if show_node:
        assert (got == np.float32(R.NODE_ACT)).all(-1).any()
    else:
        assert cells_seen
    sim.close()


def test_particles_and_device_output():
    import torch

    from agimp.render import HeadlessGUI, render_mask, render_mask_torch, render_particles
    sc, sim = _scene(1, 0.35, 3)
    rng = np.random.default_rng(0)
    sim.c_p[:] = rng.uniform(0.2, 1.0, sim.c_p.shape).astype(np.float32)
    res = 768
    base = render_mask(sim, res)
    np.testing.assert_array_equal(render_mask_torch(sim, res).cpu().numpy(), base)
    got = render_particles(sim, base.copy(), radius=0.003)
    exp = R.splat_particles(base.copy(), sim.x_p.to_numpy(), sim.c_p, 0.003)
    np.testing.assert_array_equal(got, exp)
    assert (got != base).any(-1).sum() > 1000  # particles were drawn
    gui = HeadlessGUI(res)
    np.testing.assert_array_equal(gui.show(sim), got)
    sim.close()
