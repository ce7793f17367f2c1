"""Helpers shared by the golden-vector tests."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LO = -4  # fixtures store level arrays over indices [-4, size + 8)


def scenes():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def step_input(z, s):
    """Particle state that substep s starts from."""
    if s == 0:
        return dict(x=z["x0"], v=z["v0"], F=z["F0"], C=z["C0"])
    return {k: z["s%d_%s" % (s - 1, k)] for k in "xvFC"}


def node_norm(m):
    """Node mask with the GHOST bit dropped where T_JUNCTION is set: the
    reference sets GHOST only on nodes whose mask is 0 at the time of the check
    (adaptive_gimp.py:182-183), so T|G versus T depends on thread order, while
    both classify as a T-junction (adaptive_gimp.py:130-140)."""
    m = np.asarray(m)
    return np.where(m & 4, m & ~2, m)


def node_classes(nm):
    """0 invalid, 1 activated, 2 T-junction, 3 ghost (adaptive_gimp.py:130-140)."""
    nm = np.asarray(nm)
    cls = np.zeros(nm.shape, np.int8)
    cls[(nm & 5) == 1] = 1
    cls[(nm & 4) == 4] = 2
    cls[(nm & 7) == 2] = 3
    return cls


def rel_close(a, b, rtol):
    """max |a-b| <= rtol * max(|b|, tiny)"""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= rtol * scale, np.abs(a - b).max() / scale


# Nodes lighter than this fraction of a level's heaviest node carry velocities
# v = p / m whose rounding error grows like 1 / m (a node touched only by the
# far edge of one particle's stencil can weigh 1e-10 of a typical node); their
# velocity is checked through the momentum m v instead.
LIGHT_NODE = 1e-5


def grid_v_close(v, v_ref, m_ref, rtol):
    """Nodal velocities: momentum m_ref v within rtol of the largest momentum,
    and velocity within rtol of the largest velocity at nodes heavier than
    LIGHT_NODE of the heaviest.  Returns (ok, worst ratio)."""
    v = np.asarray(v, np.float64)
    v_ref = np.asarray(v_ref, np.float64)
    m = np.asarray(m_ref, np.float64)[..., None]
    ok_p, r_p = rel_close(m * v, m * v_ref, rtol)
    heavy = np.broadcast_to(m > LIGHT_NODE * max(m.max(), 1e-30), v.shape)
    if not heavy.any():
        return ok_p, r_p
    ok_v, r_v = rel_close(v[heavy], v_ref[heavy], rtol)
    return ok_p and ok_v, max(r_p, r_v)
