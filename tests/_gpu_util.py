"""Helpers for the GPU parity tests: run the CUDA path (through the C ABI, via
the AdaptiveGIMP facade) and the oracle on identical inputs."""
import numpy as np

import oracle as O

LO = -4


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def gpu_sim(dim, level, coarsest, n, table=None, halo=None, **kw):
    from agimp import AdaptiveGIMP
    sim = AdaptiveGIMP(dim, level, coarsest, n, lambda s: None, None, **kw)
    if table is not None:
        sim.set_level_map(table, halo)
    return sim


def oracle_kwargs(kw, dim):
    """AdaptiveGIMP keyword overrides -> oracle parameters."""
    out = {}
    if "gravity" in kw:
        out["gravity"] = tuple(kw["gravity"]) + (0.0,) * (3 - len(kw["gravity"]))
    for k in ("E", "nu", "radius", "boundary_gap", "theta_c", "theta_s", "hardening"):
        if k in kw:
            out[k] = kw[k]
    if "boundary_mode" in kw:
        out["boundary_mode"] = {"ref_slip": 0, "sticky": 1}[kw["boundary_mode"]]
    if "plasticity" in kw:
        out["plasticity"] = {None: 0, "none": 0, "snow": 1}[kw["plasticity"]]
    if "colliders" in kw:
        out["colliders"] = tuple(kw["colliders"])
    if "invalid_nodes" in kw:
        out["invalid_nodes"] = {"raw": 0, "normalize": 1}[kw["invalid_nodes"]]
    return out


def gpu_state(sim):
    return dict(x=sim.x_p.to_numpy(), v=sim.v_p.to_numpy(), F=sim.F_p.to_numpy(), C=sim.C_p.to_numpy(),
                fl=sim.fl_p.to_numpy(), g=sim.g_p.to_numpy(), Jp=sim.Jp.to_numpy())


def gpu_grid(sim, l):
    n = (sim.coarsest_size << l) + 12
    return sim.ad_grid_m[l].read(LO, n), sim.ad_grid_v[l].read(LO, n), sim.cell_mask[l].read(LO, n)


def scale_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)) if a.size else 0.0
