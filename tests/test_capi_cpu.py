"""C ABI checks that need no GPU: the library loads, exports every function
include/agimp.h declares, and rejects invalid parameters before touching a
device."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "agimp.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(agimp_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from agimp import _capi
    lib = _capi.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_capi.EXPORTS)


def test_abi_version_and_status_strings():
    from agimp import _capi
    lib = _capi.load()
    assert lib.agimp_abi_version() == 2
    assert lib.agimp_status_string(0) == b"ok"
    assert lib.agimp_status_string(1) == b"invalid argument"


def test_default_params_are_reference_constants():
    from agimp import _capi
    lib = _capi.load()
    p = _capi.Params()
    lib.agimp_default_params(ctypes.byref(p), 3, 3, 16, 50000)
    # adaptive_gimp.py:18, 48-53
    assert p.radius == 0.5 and p.boundary_gap == 4 and p.boundary_mode == 0 and p.plasticity == 0
    assert tuple(p.gravity) == (0.0, -100.0, 0.0)
    assert p.E == 5e3 and p.nu == 0.2
    assert p.invalid_nodes == 0  # the reference's grid update (adaptive_gimp.py:280)


@pytest.mark.parametrize("field,value", [("dim", 4), ("level", 0), ("level", 9), ("coarsest_size", 12),
                                         ("coarsest_size", 2), ("n_particles", -1), ("radius", 0.75),
                                         ("n_colliders", 5), ("plasticity", 7),
                                         ("invalid_nodes", 2), ("n_particles", 2 ** 30 + 1),
                                         ("coarsest_size", 8192)])  # finest 16384 > 8192
def test_create_rejects_invalid_params(field, value):
    from agimp import _capi
    lib = _capi.load()
    p = _capi.Params()
    lib.agimp_default_params(ctypes.byref(p), 2, 3, 16, 100)
    setattr(p, field, value)
    h = ctypes.c_void_p()
    assert lib.agimp_create(ctypes.byref(p), 0, ctypes.byref(h)) == 1  # AGIMP_INVALID_ARG
    assert not h.value


def test_null_handle_calls_fail_cleanly():
    from agimp import _capi
    lib = _capi.load()
    assert lib.agimp_substep(None, 1e-4, 1, None) == 1
    assert lib.agimp_destroy(None) == 1
    assert lib.agimp_last_error(None) == b"null handle"
