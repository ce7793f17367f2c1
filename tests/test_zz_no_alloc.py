"""The allocation-free refinement entry point against the handle-based one.

agimp_refine_levels_noalloc serves callers that cannot let a library allocate
device memory (their own pool owns it); it keeps its scratch in a static
device array inside libagimp.so.  This file is collected last, so a run that
stops at the first failure has run every other test before it.  It must pass
alone in a fresh process and after the other tests; each call is checked
against agimp_refine_levels (integer levels: exact), twice in a row.
"""
import ctypes

import numpy as np
import pytest

from _gpu_util import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


def test_refine_levels_noalloc_matches_handle_path_twice():
    import torch

    from agimp import _capi, scenes
    lib = _capi.load()
    scene = scenes.make_config(3, scale=0.4)
    n, L, c = scene.n, scene.level, scene.coarsest
    sim = scene.build()
    stream = torch.cuda.current_stream()
    xs = [scene.x, (scene.x + np.float32(0.013)).astype(np.float32)]  # second call: shifted sphere
    for x in xs:
        sim.x_p.from_numpy(x)
        sim.refine_levels(2)
        expect = sim.g_p.to_numpy()
        xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        gd = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        st = lib.agimp_refine_levels_noalloc(ctypes.c_void_p(xd.data_ptr()), n, 3, L, c, 2,
                                             ctypes.c_void_p(gd.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert st == 0
        torch.cuda.synchronize()
        got = gd.cpu().numpy()
        np.testing.assert_array_equal(got, expect)
        assert len(np.unique(got)) == L
    sim.close()
    # a grid beyond the static scratch (512^3 cells) is rejected with AGIMP_CAPACITY
    assert lib.agimp_refine_levels_noalloc(ctypes.c_void_p(xd.data_ptr()), n, 3, 4, 64, 2,
                                           ctypes.c_void_p(gd.data_ptr()), None) == 2
