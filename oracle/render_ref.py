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
