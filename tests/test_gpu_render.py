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


def _view_dict(v):
    return dict(eye=tuple(v.eye), right=tuple(v.right), up=tuple(v.up), forward=tuple(v.forward),
                tan_half_fov=v.tan_half_fov, radius=v.radius, color=tuple(v.color), floor=bool(v.floor),
                floor_color=tuple(v.floor_color), ambient=tuple(v.ambient),
                lights=[(tuple(v.light_pos[i]), tuple(v.light_color[i])) for i in range(v.n_lights)],
                background=tuple(v.background))


@pytest.mark.parametrize("res,radius,floor", [(96, 0.02, True), (160, 0.05, False)])
def test_scene3d_matches_restatement(res, radius, floor):
    # a small 3D scene stepped a few substeps (particles in bin order on the
    # device) rendered with GUI3D's camera and lights
    from agimp import scenes
    from agimp.render import render_scene3d, view3d
    sc = scenes.make_config(3, scale=0.25)
    sim = sc.build()
    for i in range(5):
        if i % sc.refine_every == 0:
            sim.refine_levels(sc.refine_band)
        sim.substep(sc.dt)
    v = view3d(radius=radius, floor=floor, ambient=(0.05, 0.05, 0.05))
    got = render_scene3d(sim, res, v)
    exp = R.render_scene3d(sim.x_p.to_numpy(), res, _view_dict(v))
    np.testing.assert_array_equal(got, exp)
    assert (got > 0).any(axis=2).sum() > res  # spheres (and floor) are drawn
    sim.close()


def test_cell_lines_match_restatement():
    from agimp import scenes
    from agimp.render import cell_lines
    sc, sim = _scene(3, 0.25, 12)
    got = cell_lines(sim)
    cells = [sim.cell_mask[l].read(LO, (sim.coarsest_size << l) + 12) for l in range(sim.level)]
    exp = R.cell_lines(cells, LO, sim.coarsest_size)
    assert got.shape == exp.shape and len(got) > 24
    key = lambda v: sorted(map(bytes, v.reshape(-1, 24 * 3)))  # cells in any order
    assert key(got) == key(exp)
    sim.close()
