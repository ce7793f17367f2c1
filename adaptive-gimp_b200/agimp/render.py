"""Headless drawing (libagimp.so agimp_render_*, agimp_cell_lines).

The reference draws into a GGUI window (gui.py: GUI.visualize_mask and
canvas.circles); there is no graphics stack here, so the same picture is
rendered by CUDA kernels into an image buffer and can be written to a file:

    gui = HeadlessGUI(res=768)
    sim.substep(dt)
    gui.show(sim)               # gui.img: [res][res][3] float32, indexed [i][j]
    gui.save("frame.ppm")       # j (the y axis) points up in the picture
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from .simulator import AGIMP_MEM_DEVICE, AGIMP_MEM_HOST, _ptr


def render_mask(sim, res=768, show_ghost=True, show_node=True, out=None):
    """GUI.visualize_mask (gui.py:12-43) into a numpy image [res][res][3]."""
    img = out if out is not None else np.empty((res, res, 3), np.float32)
    _capi.check(sim._L.agimp_render_mask(sim._h, int(res), int(bool(show_ghost)), int(bool(show_node)), _ptr(img),
                                         AGIMP_MEM_HOST, None), sim._h, "render mask")
    return img


def render_particles(sim, img, radius=0.003, colors=None):
    """canvas.circles(x_p, radius, per_vertex_color=c_p) (gui.py:69) drawn over img."""
    res = img.shape[0]
    cols = np.ascontiguousarray(sim.c_p if colors is None else colors, np.float32)
    _capi.check(sim._L.agimp_render_particles(sim._h, int(res), float(radius), _ptr(cols), AGIMP_MEM_HOST, _ptr(img),
                                              AGIMP_MEM_HOST, None), sim._h, "render particles")
    return img


def render_mask_torch(sim, res=768, show_ghost=True, show_node=True):
    """The same into a CUDA tensor (no host copy)."""
    import torch
    img = torch.empty((res, res, 3), dtype=torch.float32, device="cuda:%d" % sim.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(sim._L.agimp_render_mask(sim._h, int(res), int(bool(show_ghost)), int(bool(show_node)),
                                         ctypes.c_void_p(img.data_ptr()), AGIMP_MEM_DEVICE, st), sim._h, "render mask")
    return img


def save_ppm(img, path):
    """Binary PPM with j (y) pointing up: picture row r is j = res - 1 - r."""
    a = np.clip(np.asarray(img, np.float32), 0.0, 1.0)
    pic = (np.transpose(a, (1, 0, 2))[::-1] * 255.0 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (pic.shape[1], pic.shape[0]))
        f.write(pic.tobytes())


class HeadlessGUI:
    """gui.GUI without a window: show() renders into self.img."""

    def __init__(self, res=768):
        self.res = res
        self.img = np.zeros((res, res, 3), np.float32)

    def show(self, simulator, show_particles=True, show_ghost=True, show_node=True, radius=0.003):
        render_mask(simulator, self.res, show_ghost, show_node, out=self.img)
        if show_particles:
            render_particles(simulator, self.img, radius)
        return self.img

    def save(self, path):
        save_ppm(self.img, path)


# ---------------------------------------------------------------------------
# 3D: gui_3d.GUI3D without a window


def camera_basis(position, lookat, up=(0.0, 1.0, 0.0)):
    """Orthonormal (right, up, forward) of a camera at `position` looking at
    `lookat` (computed in float64, returned as float32)."""
    p, q, u = (np.asarray(v, np.float64) for v in (position, lookat, up))
    f = q - p
    f /= np.linalg.norm(f)
    r = np.cross(f, u)
    r /= np.linalg.norm(r)
    uc = np.cross(r, f)
    return r.astype(np.float32), uc.astype(np.float32), f.astype(np.float32)


def view3d(position=(0.5, 1.0, 1.95), lookat=(0.5, 0.3, 0.5), fov=55.0, radius=0.02, color=(0.5, 0.5, 0.5),
           floor=True, floor_color=(0.0, 0.0, 0.9), ambient=(0.0, 0.0, 0.0),
           lights=(((0.5, 1.5, 0.5), (0.5, 0.5, 0.5)), ((0.5, 1.5, 1.5), (0.5, 0.5, 0.5))),
           background=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0)):
    """The view of GUI3D.show (gui_3d.py:14-17, 50-61) as an agimp_view3d:
    camera at (0.5, 1.0, 1.95) looking at (0.5, 0.3, 0.5) with a 55 degree
    field of view, grey spheres of radius 0.02, the blue floor quad, two
    grey point lights above it, no ambient light."""
    v = _capi.View3D()
    r, u, f = camera_basis(position, lookat, up)
    for k in range(3):
        v.eye[k], v.right[k], v.up[k], v.forward[k] = float(position[k]), float(r[k]), float(u[k]), float(f[k])
        v.color[k], v.floor_color[k], v.ambient[k], v.background[k] = color[k], floor_color[k], ambient[k], background[k]
    v.tan_half_fov = float(np.float32(np.tan(np.radians(fov) / 2.0)))
    v.radius = float(radius)
    v.floor = 1 if floor else 0
    if len(lights) > 4:
        raise ValueError("at most 4 lights")
    v.n_lights = len(lights)
    for i, (pos, col) in enumerate(lights):
        for k in range(3):
            v.light_pos[i][k], v.light_color[i][k] = float(pos[k]), float(col[k])
    return v


def render_scene3d(sim, res=768, view=None, out=None):
    """GUI3D.show's picture into a numpy image [res][res][3], row 0 at the top."""
    v = view if view is not None else view3d()
    img = out if out is not None else np.empty((res, res, 3), np.float32)
    _capi.check(sim._L.agimp_render_scene3d(sim._h, int(res), ctypes.byref(v), _ptr(img), AGIMP_MEM_HOST, None),
                sim._h, "render 3D")
    return img


def cell_lines(sim):
    """GUI3D._draw_lines (gui_3d.py:35-47): vertices [24 k][3] of the edges of
    the k exactly-ACTIVATED cells (in no fixed cell order)."""
    n = ctypes.c_int64()
    _capi.check(sim._L.agimp_cell_lines(sim._h, None, 0, ctypes.byref(n), AGIMP_MEM_HOST, None), sim._h, "cell lines")
    vert = np.empty((n.value, 3), np.float32)
    if n.value:
        _capi.check(sim._L.agimp_cell_lines(sim._h, _ptr(vert), n.value, ctypes.byref(n), AGIMP_MEM_HOST, None),
                    sim._h, "cell lines")
    return vert


def save_ppm_rows(img, path):
    """Binary PPM of an image stored row by row (row 0 at the top)."""
    a = np.clip(np.asarray(img, np.float32), 0.0, 1.0)
    pic = (a * 255.0 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (pic.shape[1], pic.shape[0]))
        f.write(pic.tobytes())


class HeadlessGUI3D:
    """gui_3d.GUI3D without a window: show() renders into self.img."""

    def __init__(self, simulator, res=768, **view_kw):
        self.simulator = simulator
        self.res = res
        self.view = view3d(**view_kw)
        self.img = np.zeros((res, res, 3), np.float32)

    def draw_lines(self):
        return cell_lines(self.simulator)

    def show(self):
        render_scene3d(self.simulator, self.res, self.view, out=self.img)
        return self.img

    def save(self, path):
        save_ppm_rows(self.img, path)
