"""Headless drawing of a 2D simulator (libagimp.so agimp_render_*).

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
