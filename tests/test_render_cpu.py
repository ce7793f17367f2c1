"""The numpy restatement of the reference GUI's mask view (oracle/render_ref.py)
on hand-made masks: colours, edges and node markers where gui.py:12-43 puts
them."""
import numpy as np

import render_ref as R


def test_restated_mask_view():
    # 2 levels, coarsest 4, finest 8, res 24: scale 6 (level 0), 3 (level 1)
    c0 = np.zeros((4 + 12, 4 + 12), np.int32)
    c1 = np.zeros((8 + 12, 8 + 12), np.int32)
    lo = -4
    c0[0 - lo, 0 - lo] = R.ACT   # level-0 cell (0, 0): pixels [0, 6)^2
    c1[3 - lo, 3 - lo] = R.ACT   # level-1 cell (3, 3): pixels [9, 12)^2
    c1[4 - lo, 3 - lo] = R.GHO   # ghost cell (4, 3): pixels [12, 15) x [9, 12)
    nm = np.zeros((9, 9), np.int32)
    nm[2, 2] = R.ACT
    nm[5, 5] = R.TJ
    nm[6, 6] = R.GHO
    img = R.render_mask([c0, c1], lo, nm, 4, 24, show_ghost=True, show_node=False)
    f = lambda c: np.float32(c)
    assert (img[2, 2] == f(R.ACT_FILL)).all() and (img[0, 3] == f(R.ACT_EDGE)).all()
    assert (img[10, 10] == f(R.ACT_FILL)).all() and (img[9, 10] == f(R.ACT_EDGE)).all()
    assert (img[13, 10] == f(R.GHO_FILL)).all() and (img[12, 10] == f(R.GHO_EDGE)).all()
    assert (img[20, 20] == 0).all()
    no_ghost = R.render_mask([c0, c1], lo, nm, 4, 24, show_ghost=False, show_node=False)
    assert (no_ghost[13, 10] == 0).all()
    with_nodes = R.render_mask([c0, c1], lo, nm, 4, 24, show_ghost=True, show_node=True)
    # node (2, 2) at pixel (6, 6) (fscale 3): a 3x3 red square
    assert (with_nodes[5:8, 5:8] == f(R.NODE_ACT)).all()
    assert (with_nodes[15, 15] == f(R.NODE_TJ)).all() and (with_nodes[18, 18] == f(R.NODE_GHO)).all()


def test_restated_particle_circles():
    img = np.zeros((20, 20, 3), np.float32)
    x = np.array([[0.5, 0.5], [0.52, 0.5]], np.float32)
    cols = np.array([[1, 0, 0], [0, 1, 0]], np.float32)
    R.splat_particles(img, x, cols, radius=0.1)  # 2-pixel radius, centres at (10, 10) and (10.4, 10)
    assert (img[9, 9] == [0, 1, 0]).all()      # covered by both: the later particle wins
    assert (img[11, 8] == [0, 1, 0]).all()     # only the second: (11.5-10)^2 + (8.5-10)^2 > 4
    R.splat_particles(img, x[::-1].copy(), cols[::-1].copy(), radius=0.1)
    assert (img[9, 9] == [1, 0, 0]).all()      # drawn in the other order
    assert (img[11, 8] == [0, 1, 0]).all()
    assert (img[0, 0] == 0).all()


def _view(res_fov=55.0):
    from agimp.render import camera_basis
    r, u, f = camera_basis((0.5, 1.0, 1.95), (0.5, 0.3, 0.5))
    return dict(eye=(0.5, 1.0, 1.95), right=r, up=u, forward=f,
                tan_half_fov=np.float32(np.tan(np.radians(res_fov) / 2)), radius=0.02, color=(0.5, 0.5, 0.5),
                floor=True, floor_color=(0.0, 0.0, 0.9), ambient=(0.0, 0.0, 0.0),
                lights=[((0.5, 1.5, 0.5), (0.5, 0.5, 0.5)), ((0.5, 1.5, 1.5), (0.5, 0.5, 0.5))],
                background=(0.0, 0.0, 0.0))


def test_restated_scene3d_sphere_and_floor():
    v = _view()
    v["radius"] = 0.1
    res = 64
    # a sphere at the look-at point appears at the image centre, lit from above
    img = R.render_scene3d(np.array([[0.5, 0.3, 0.5]], np.float32), res, v)
    c = img[res // 2, res // 2]
    assert c[0] == c[1] == c[2] and c[0] > 0.05
    # the floor (blue) is seen below it (the camera at z = 1.95 sees past its
    # near edge z = 1 at the bottom rows), the background (black) above it
    col = img[:, res // 2]
    floor_rows = np.nonzero((col[:, 2] > 0) & (col[:, 0] == 0))[0]
    assert len(floor_rows) > res // 4 and floor_rows.min() > res // 2 - 8 and floor_rows.max() < res - 4
    assert (img[1, res // 2] == 0).all()
    # no particles: only the floor
    empty = R.render_scene3d(np.zeros((0, 3), np.float32), res, v)
    assert (empty[..., 0] == 0).all() and (empty[..., 2] > 0).sum() > res * res // 10


def test_restated_cell_lines():
    cm0 = np.zeros((2 + 12, 2 + 12, 2 + 12), np.int32)
    cm0[4 + 1, 4 + 0, 4 + 1] = R.ACT  # cell (1, 0, 1) of level 0, coarsest 2
    cm1 = np.zeros((4 + 12,) * 3, np.int32)
    cm1[4 + 3, 4 + 3, 4 + 3] = R.GHO  # not drawn
    v = R.cell_lines([cm0, cm1], -4, 2)
    assert v.shape == (24, 3)
    # first edge: corner 0 -> corner 1 (dI = (0,0,0) -> (1,0,0)), dx = 0.5
    np.testing.assert_array_equal(v[0], [0.5, 0.0, 0.5])
    np.testing.assert_array_equal(v[1], [1.0, 0.0, 0.5])
    np.testing.assert_array_equal(v[-1], [1.0, 0.5, 1.0])  # corner 7
