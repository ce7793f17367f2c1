"""Failure detection on the device without a fault: the bounded completion
wait of the tensor-core kernels (an mbarrier that nothing arrives on) gives
up after its poll limit, the kernel reports the timeout through the error
word, and the CUDA context stays usable for the next substep."""
import ctypes

import numpy as np
import pytest

from _gpu_util import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA device")]


def test_bounded_wait_times_out_and_context_survives():
    from agimp import _capi, scenes
    lib = _capi.load()
    bits = ctypes.c_uint32(99)
    # the barrier completes: no timeout
    assert lib.agimp_wait_selftest(0, 1, 1000, ctypes.byref(bits)) == 0
    assert bits.value == 0
    # nothing arrives: the wait gives up after 1000 polls and says so
    assert lib.agimp_wait_selftest(0, 0, 1000, ctypes.byref(bits)) == 4  # AGIMP_DEVICE_TIMEOUT
    assert bits.value == _capi.ERR_WAIT
    # the context still runs a substep correctly
    scene = scenes.make_config(1, scale=0.3)
    sim = scene.build()
    sim.substep(scene.dt, 3)
    assert sim.errors() == 0
    assert np.isfinite(sim.x_p.to_numpy()).all()
    sim.close()
