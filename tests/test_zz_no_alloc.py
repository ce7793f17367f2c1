"""The allocation-free refinement entry point against the handle-based one.

agimp_refine_levels_noalloc serves callers that cannot let a library allocate
device memory (their own pool owns it); it keeps its scratch in a static
device array inside libagimp.so.  This file is collected last, so a run that
stops at the first failure has run every other test before it.  It must pass
alone in a fresh process and after the other tests; each call is checked
against agimp_refine_levels (integer levels: exact), twice in a row, in 3D
and in 2D, with the default band and with a wide one whose deepest threshold
is close to the byte limit of the stored depths.
"""
import ctypes

import numpy as np
import pytest

from _gpu_util import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


def _noalloc(lib, x, n, dim, L, c, band, stream):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    gd = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    st = lib.agimp_refine_levels_noalloc(ctypes.c_void_p(xd.data_ptr()), n, dim, L, c, band,
                                         ctypes.c_void_p(gd.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    return gd.cpu().numpy(), xd, gd


def _check_twice(scene, band, shift):
    import torch

    from agimp import _capi
    lib = _capi.load()
    n, L, c, d = scene.n, scene.level, scene.coarsest, scene.dim
    sim = scene.build()
    stream = torch.cuda.current_stream()
    xs = [scene.x, (scene.x + np.float32(shift)).astype(np.float32)]  # second call: shifted bodies
    for x in xs:
        assert x.min() >= 0 and x.max() < 1  # every particle gets a level from both paths
        sim.x_p.from_numpy(x)
        sim.refine_levels(band)
        expect = sim.g_p.to_numpy()
        got, xd, gd = _noalloc(lib, x, n, d, L, c, band, stream)
        np.testing.assert_array_equal(got, expect)
        assert len(np.unique(got)) >= 2
    sim.close()
    return lib, xd, gd, n


def test_refine_levels_noalloc_matches_handle_path_twice():
    from agimp import scenes
    scene = scenes.make_config(3, scale=0.4)
    lib, xd, gd, n = _check_twice(scene, 2, 0.013)
    # a grid beyond the static scratch (512^3 cells) is rejected with AGIMP_CAPACITY
    assert lib.agimp_refine_levels_noalloc(ctypes.c_void_p(xd.data_ptr()), n, 3, 4, 64, 2,
                                           ctypes.c_void_p(gd.data_ptr()), None) == 2
    # a band whose deepest threshold, band (2^(L-1) - 1), reaches 250 is rejected
    # (depths are kept in bytes): band 32 with 5 levels of 16..256
    assert lib.agimp_refine_levels_noalloc(ctypes.c_void_p(xd.data_ptr()), n, 3, 5, 16, 32,
                                           ctypes.c_void_p(gd.data_ptr()), None) == 1


def test_refine_levels_noalloc_2d_wide_band_twice():
    from agimp import scenes
    # 2D dynamic scene of 4 levels (64^2 .. 512^2); band 8: deepest threshold 56
    scene = scenes.make_config(2)
    _check_twice(scene, 8, 0.02)
    # band 30 with 4 levels: deepest threshold 210, close to the byte limit
    _check_twice(scene, 30, -0.011)
