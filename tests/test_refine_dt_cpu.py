"""The refinement rule's depth as the kernels compute it (csrc/refine.cu: a
separable Chebyshev distance transform, one pass per axis, capped at
K = 1 + band (2^(L-1) - 1)), restated in numpy and checked against the oracle,
which erodes the occupancy iteratively (oracle/oracle.cpp refine_levels): the
prescribed levels must agree particle for particle."""
import numpy as np
import pytest

import oracle as O


def _depth_by_passes(occ, K):
    """f_0 = 0 on empty, K on occupied cells; pass along each axis (innermost
    first): f_a(c) = min over x' of max(f_{a-1}(c|x'), |x - x'|), positions
    outside the box empty; the scan stops once the offset reaches the best."""
    f = np.where(occ, K, 0).astype(np.int64)
    for a in range(occ.ndim - 1, -1, -1):
        fm = np.moveaxis(f, a, -1)
        n = fm.shape[-1]
        out = fm.copy()
        for o in range(1, K):
            left = np.concatenate([np.zeros(fm.shape[:-1] + (o,), np.int64), fm[..., :-o]], -1) if o < n else \
                np.zeros_like(fm)
            right = np.concatenate([fm[..., o:], np.zeros(fm.shape[:-1] + (o,), np.int64)], -1) if o < n else \
                np.zeros_like(fm)
            out = np.minimum(out, np.maximum(np.minimum(left, right), o))
        f = np.moveaxis(out, -1, a)
    return f


def _levels(x, level, coarsest, band):
    """g_p from the depth of each particle's finest cell (the kernels' rule)."""
    sz = coarsest << (level - 1)
    cell = np.floor(x * np.float32(sz)).astype(np.int64)
    lo, hi = cell.min(0), cell.max(0)
    occ = np.zeros(tuple(hi - lo + 1), bool)
    occ[tuple((cell - lo).T)] = True
    K = min(band * ((1 << (level - 1)) - 1) + 1, 250)
    depth = _depth_by_passes(occ, K)[tuple((cell - lo).T)]
    g = np.zeros(len(x), np.int32)
    for i, dd in enumerate(depth):
        for k in range(level - 1):
            if dd <= band * ((1 << (k + 1)) - 1):
                g[i] = level - 1 - k
                break
    return g


@pytest.mark.parametrize("dim,level,coarsest,band,seed", [(3, 3, 16, 2, 0), (3, 4, 8, 1, 1), (2, 4, 32, 3, 2),
                                                         (2, 3, 64, 2, 3)])
def test_distance_transform_matches_oracle_erosion(dim, level, coarsest, band, seed):
    rng = np.random.default_rng(seed)
    sz = coarsest << (level - 1)
    # one particle per finest cell of a ball, a few cells left out (holes)
    # and a few stray particles: surfaces inside and out
    axes = np.meshgrid(*[(np.arange(sz) + 0.5) / sz] * dim, indexing="ij")
    pts = np.stack(axes, -1).reshape(-1, dim)
    keep = (np.linalg.norm(pts - 0.5, axis=1) < 0.35) & (rng.random(len(pts)) > 0.02)
    x = pts[keep].astype(np.float32)
    x = np.concatenate([x, rng.uniform(0.05, 0.95, (20, dim)).astype(np.float32)])
    x = np.clip(x, 0.0, np.float32(1.0 - 1.0 / sz))
    n = len(x)
    o = O.Oracle(dim, level, coarsest, n)
    o.set_particles(x, np.zeros((n, dim)), np.tile(np.eye(dim), (n, 1, 1)), np.zeros((n, dim, dim)),
                    np.ones(n), np.full(n, level - 1, np.int32))
    o.refine_levels(band)
    want = o.particles()["g"]
    got = _levels(x, level, coarsest, band)
    np.testing.assert_array_equal(got, want)
    assert len(np.unique(want)) >= 2
