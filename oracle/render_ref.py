"""CPU restatement of the reference GUI's drawing (test infrastructure only:
the tests compare the CUDA rendering of libagimp.so against it).

render_mask follows gui.py:12-43 (GUI.visualize_mask) on read-back cell masks
and the finest node mask; the overlapping 3x3 node markers of its second loop
are resolved in serial row-major order.  splat_particles draws
canvas.circles (gui.py:69) with the library's stated rule: a pixel whose
centre lies within radius * res pixels of a particle takes its colour, later
particles on top.
"""
import numpy as np

ACT, GHO, TJ = 1, 2, 4
ACT_FILL, ACT_EDGE = (0.28, 0.68, 0.99), (0.18, 0.58, 0.88)  # gui.py:21-23
GHO_FILL, GHO_EDGE = (0.0, 0.0, 1.0), (0.0, 0.0, 0.77)      # gui.py:25-27
NODE_ACT, NODE_TJ, NODE_GHO = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 0.35)  # gui.py:36, 40, 44


def _is_activated(nm):
    return (nm & (ACT | TJ)) == ACT


def _is_tj(nm):
    return (nm & TJ) == TJ


def _is_ghost(nm):
    return (nm & (ACT | GHO | TJ)) == GHO


def render_mask(cells, lo, nmask, coarsest, res, show_ghost=True, show_node=True):
    """cells[l]: cell_mask of level l read over [lo, lo + n)^2; nmask: node
    mask over [0, finest]^2.  Returns img[res][res][3] float32."""
    L = len(cells)
    img = np.zeros((res, res, 3), np.float32)
    i = np.arange(res)[:, None]
    j = np.arange(res)[None, :]
    for l in range(L):  # gui.py:17-29
        scale = res // (coarsest << l)
        ci, cj = i // scale, j // scale
        arr = cells[l]
        n = arr.shape[0]
        inr = (ci - lo >= 0) & (ci - lo < n) & (cj - lo >= 0) & (cj - lo < n)
        cm = np.where(inr, arr[np.clip(ci - lo, 0, n - 1), np.clip(cj - lo, 0, n - 1)], 0)
        edge = (i % scale == 0) | (i % scale == scale - 1) | (j % scale == 0) | (j % scale == scale - 1)
        for mask, fill, edg in ((cm == ACT, ACT_FILL, ACT_EDGE),
                                ((cm == GHO) & bool(show_ghost), GHO_FILL, GHO_EDGE)):
            col = np.where(edge[..., None], np.float32(edg), np.float32(fill)).astype(np.float32)
            img = np.where(mask[..., None], col, img)
    if show_node:  # gui.py:31-43, serial order
        finest = nmask.shape[0] - 1
        fscale = res // finest
        for a in range(0, res, fscale):
            for b in range(0, res, fscale):
                P = (a // fscale, b // fscale)
                nm = int(nmask[P]) if P[0] <= finest and P[1] <= finest else 0
                col = NODE_ACT if _is_activated(nm) else NODE_TJ if _is_tj(nm) else NODE_GHO if _is_ghost(nm) else None
                if col is None:
                    continue
                img[max(a - 1, 0):min(a + 2, res), max(b - 1, 0):min(b + 2, res)] = np.float32(col)
    return img


def splat_particles(img, x, colors, radius):
    """x [N][2] and colors [N][3] in the caller's order; draws over img in place."""
    res = img.shape[0]
    r = np.float32(np.float32(radius) * np.float32(res))
    r2 = np.float32(r * r)
    for k in range(len(x)):
        px = np.float32(np.float32(x[k, 0]) * np.float32(res))
        py = np.float32(np.float32(x[k, 1]) * np.float32(res))
        if not (np.isfinite(px) and np.isfinite(py)):
            continue
        i0, i1 = max(0, int(np.floor(px - r - 0.5))), min(res - 1, int(np.ceil(px + r - 0.5)))
        j0, j1 = max(0, int(np.floor(py - r - 0.5))), min(res - 1, int(np.ceil(py + r - 0.5)))
        if i1 < i0 or j1 < j0:
            continue
        ii = np.arange(i0, i1 + 1, dtype=np.float32)[:, None]
        jj = np.arange(j0, j1 + 1, dtype=np.float32)[None, :]
        dx = (ii + np.float32(0.5)) - px
        dy = (jj + np.float32(0.5)) - py
        cov = (dx * dx + dy * dy) <= r2
        sub = img[i0:i1 + 1, j0:j1 + 1]
        sub[cov] = np.float32(colors[k])
    return img


# ---------------------------------------------------------------------------
# 3D: the library's stated picture of GUI3D.show (gui_3d.py:50-64): ray-cast
# spheres and floor with Lambert point lights, every operation in float32 in
# the kernel's order (dot products ((a0 b0 + a1 b1) + a2 b2)).

def _dot3(a, b):
    f = np.float32
    return (f(a[0]) * f(b[0]) + f(a[1]) * f(b[1])) + f(a[2]) * f(b[2])


def rays3d(view, res):
    f = np.float32
    col = np.arange(res, dtype=np.float32)[None, :].repeat(res, 0)
    row = np.arange(res, dtype=np.float32)[:, None].repeat(res, 1)
    fr, th = f(res), f(view["tan_half_fov"])
    sx = ((f(2) * (col + f(0.5))) / fr - f(1)) * th
    sy = (f(1) - (f(2) * (row + f(0.5))) / fr) * th
    d = [(f(view["forward"][k]) + sx * f(view["right"][k])) + sy * f(view["up"][k]) for k in range(3)]
    inv = f(1) / np.sqrt(_dot3(d, d))
    return [dk * inv for dk in d]  # three [res][res] arrays


def _shade(view, base, p, n):
    f = np.float32
    out = [f(base[k]) * f(view["ambient"][k]) + np.zeros_like(p[0]) for k in range(3)]
    for lp, lc in view["lights"]:
        L = [f(lp[k]) - p[k] for k in range(3)]
        inv = f(1) / np.sqrt(_dot3(L, L))
        L = [Lk * inv for Lk in L]
        ndl = np.maximum(_dot3(n, L), f(0))
        out = [out[k] + (f(base[k]) * f(lc[k])) * ndl for k in range(3)]
    return out


def render_scene3d(x, res, view):
    """x [N][3] f32 in caller order; view: dict of eye, right, up, forward,
    tan_half_fov, radius, color, floor, floor_color, ambient, lights
    [(pos, colour)], background.  Returns [res][res][3] f32, row 0 on top."""
    f = np.float32
    d = rays3d(view, res)
    R = f(view["radius"])
    eye = [f(v) for v in view["eye"]]
    best_t = np.full((res, res), np.inf, np.float32)
    best_i = np.full((res, res), -1, np.int64)
    for i, c in enumerate(np.asarray(x, np.float32)):
        w = [f(c[k]) - eye[k] for k in range(3)]
        oc = [-wk for wk in w]
        cz = _dot3(w, view["forward"])
        if not cz > R:
            continue
        cc = _dot3(oc, oc) - R * R
        b = _dot3(oc, d)
        disc = b * b - cc
        with np.errstate(invalid="ignore"):
            t = -b - np.sqrt(disc)
        hit = (disc >= 0) & (t > 0) & ((t < best_t) | ((t == best_t) & (i < best_i)))
        best_t = np.where(hit, t, best_t)
        best_i = np.where(hit, i, best_i)
    img = np.zeros((res, res, 3), np.float32)
    for k in range(3):
        img[..., k] = f(view["background"][k])
    tf = np.full((res, res), np.inf, np.float32)
    if view["floor"]:
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (-eye[1]) / d[1]
        hf = [eye[k] + t * d[k] for k in range(3)]
        ok = (d[1] != 0) & (t > 0) & (hf[0] >= 0) & (hf[0] <= 1) & (hf[2] >= 0) & (hf[2] <= 1)
        tf = np.where(ok, t, tf)
        use = tf < best_t
        if use.any():
            p = [hf[0][use], np.zeros(use.sum(), np.float32), hf[2][use]]
            ny = f(1) if eye[1] >= 0 else f(-1)
            n = [np.zeros_like(p[0]), np.full_like(p[0], ny), np.zeros_like(p[0])]
            out = _shade(view, view["floor_color"], p, n)
            for k in range(3):
                img[..., k][use] = out[k]
    sph = ~(tf < best_t) & np.isfinite(best_t)
    if sph.any():
        t = best_t[sph]
        cen = np.asarray(x, np.float32)[best_i[sph]]
        p = [eye[k] + t * d[k][sph] for k in range(3)]
        n = [(p[k] - cen[:, k]) / R for k in range(3)]
        out = _shade(view, view["color"], p, n)
        for k in range(3):
            img[..., k][sph] = out[k]
    return img


STENCIL = (0, 1, 2, 3, 4, 5, 6, 7, 0, 2, 1, 3, 4, 6, 5, 7, 0, 4, 1, 5, 2, 6, 3, 7)  # gui_3d.py:30-32


def cell_lines(cell_masks, lo, coarsest):
    """GUI3D._draw_lines over read-back 3D cell masks (level l array indexed
    from `lo`): 24 vertices per exactly-ACTIVATED cell, cells in index order."""
    out = []
    for l, cm in enumerate(cell_masks):
        dx = np.float32(np.float32(1.0 / coarsest) / np.float32(2 ** l))
        for I in np.argwhere(cm == ACT):
            I = I + lo
            corners = [np.float32(I + np.array([(k >> a) & 1 for a in range(3)])) * dx for k in range(8)]
            out.extend(corners[k] for k in STENCIL)
    return np.asarray(out, np.float32).reshape(-1, 3)
