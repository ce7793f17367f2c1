"""ctypes binding of libagimp.so (the C ABI declared in include/agimp.h).

This is the product path: it loads the in-tree CUDA library and raises if it
cannot; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libagimp.so")

AGIMP_MEM_DEVICE = 0
AGIMP_MEM_HOST = 1

ERR_OOB = 1
ERR_ESCAPED = 2
ERR_MAP_OOB = 4
ERR_NOBIN = 8
ERR_WAIT = 16

# every symbol include/agimp.h declares
EXPORTS = (
    "agimp_abi_version", "agimp_status_string", "agimp_default_params", "agimp_create", "agimp_destroy",
    "agimp_last_error", "agimp_set_particles", "agimp_get_particles", "agimp_set_level_map",
    "agimp_clear_level_map", "agimp_get_bins", "agimp_substep", "agimp_set_graphs", "agimp_refine_levels", "agimp_get_grid",
    "agimp_get_node_mask", "agimp_errors", "agimp_get_stats", "agimp_kernels_per_substep",
    "agimp_profile_substep", "agimp_refine_levels_noalloc",
    "agimp_mlp_num_params", "agimp_mlp_create", "agimp_mlp_destroy", "agimp_mlp_set_params", "agimp_mlp_get_params",
    "agimp_mlp_forward", "agimp_mlp_errors", "agimp_wait_selftest", "agimp_mlp_grad", "agimp_mlp_train_step", "agimp_mlp_reset_optimizer",
    "agimp_set_surrogate", "agimp_set_recorder", "agimp_recorded",
    "agimp_set_tuning", "agimp_get_tuning", "agimp_autotune",
    "agimp_batch_create", "agimp_batch_destroy", "agimp_batch_last_error", "agimp_batch_substep",
    "agimp_batch_set_graphs", "agimp_batch_set_tuning", "agimp_batch_get_tuning", "agimp_batch_autotune",
    "agimp_batch_kernels_per_substep", "agimp_batch_profile_substep", "agimp_batch_set_surrogate",
    "agimp_batch_surrogate_stats",
    "agimp_render_mask", "agimp_render_particles", "agimp_get_particles_async", "agimp_batch_positions_async",
    "agimp_batch_set_particles",
    "agimp_get_level_map", "agimp_lattice_count", "agimp_lattice_fill", "agimp_random_fill",
    "agimp_set_level_map_rule", "agimp_set_coarse_level_map", "agimp_render_scene3d", "agimp_cell_lines",
)
PHASES = ("blocks", "topology", "binning", "p2g", "restrict", "gridop", "prolong", "g2p")


class Params(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("level", ctypes.c_int32), ("coarsest_size", ctypes.c_int32),
        ("boundary_gap", ctypes.c_int32), ("boundary_mode", ctypes.c_int32), ("plasticity", ctypes.c_int32),
        ("n_particles", ctypes.c_int64), ("radius", ctypes.c_double), ("gravity", ctypes.c_double * 3),
        ("E", ctypes.c_double), ("nu", ctypes.c_double), ("theta_c", ctypes.c_double),
        ("theta_s", ctypes.c_double), ("hardening", ctypes.c_double), ("n_colliders", ctypes.c_int32),
        ("colliders", (ctypes.c_double * 6) * 4), ("invalid_nodes", ctypes.c_int32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [("active_blocks", ctypes.c_int32 * 8), ("n_binned", ctypes.c_int32), ("n_chunks", ctypes.c_int32),
                ("substeps", ctypes.c_int64), ("n_surrogate", ctypes.c_int32), ("n_fallback", ctypes.c_int32)]


class Tuning(ctypes.Structure):
    _fields_ = [("chunk", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32), ("ms_per_substep", ctypes.c_float)]

    def as_dict(self):
        return dict(chunk=self.chunk, ctas_per_sm=self.ctas_per_sm, ms_per_substep=self.ms_per_substep)


SHAPE_BOX = 0
SHAPE_SPHERE = 1


class Shape(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("level", ctypes.c_int32), ("lo", ctypes.c_double * 3),
                ("hi", ctypes.c_double * 3), ("centre", ctypes.c_double * 3), ("radius", ctypes.c_double),
                ("velocity", ctypes.c_float * 3), ("mass", ctypes.c_float)]


class RandomBox(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int64), ("lo", ctypes.c_float * 3), ("size", ctypes.c_float * 3),
                ("velocity", ctypes.c_float * 3), ("mass", ctypes.c_float), ("n_bands", ctypes.c_int32),
                ("band_lo", ctypes.c_float * 4), ("band_hi", ctypes.c_float * 4), ("band_level", ctypes.c_int32 * 4),
                ("level", ctypes.c_int32)]


class View3D(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("right", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("forward", ctypes.c_float * 3), ("tan_half_fov", ctypes.c_float), ("radius", ctypes.c_float),
                ("color", ctypes.c_float * 3), ("floor", ctypes.c_int32), ("floor_color", ctypes.c_float * 3),
                ("ambient", ctypes.c_float * 3), ("n_lights", ctypes.c_int32),
                ("light_pos", (ctypes.c_float * 3) * 4), ("light_color", (ctypes.c_float * 3) * 4),
                ("background", ctypes.c_float * 3)]


class AgimpError(RuntimeError):
    pass


_lib = None


def load(path: str | None = None):
    """Load libagimp.so; build it first when it is missing and nvcc exists."""
    global _lib
    if _lib is not None:
        return _lib
    # AGIMP_LIBRARY: another build of the library (comparing builds)
    path = path or os.environ.get("AGIMP_LIBRARY") or LIB_PATH
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(path)
    vp, fp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int32)
    L.agimp_abi_version.restype = ctypes.c_int
    L.agimp_status_string.restype = ctypes.c_char_p
    L.agimp_status_string.argtypes = [ctypes.c_int]
    L.agimp_default_params.argtypes = [ctypes.POINTER(Params), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int64]
    L.agimp_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int32, ctypes.POINTER(vp)]
    L.agimp_destroy.argtypes = [vp]
    L.agimp_last_error.restype = ctypes.c_char_p
    L.agimp_last_error.argtypes = [vp]
    L.agimp_set_particles.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int32, vp]
    L.agimp_get_particles.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int32, vp]
    L.agimp_set_level_map.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, vp]
    L.agimp_clear_level_map.argtypes = [vp]
    L.agimp_substep.argtypes = [vp, ctypes.c_float, ctypes.c_int32, vp]
    L.agimp_set_graphs.argtypes = [vp, ctypes.c_int32]
    L.agimp_refine_levels.argtypes = [vp, ctypes.c_int32, vp]
    L.agimp_get_grid.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_int32, vp]
    L.agimp_get_node_mask.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.agimp_errors.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int32]
    L.agimp_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.agimp_get_bins.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.agimp_kernels_per_substep.argtypes = [vp]
    L.agimp_kernels_per_substep.restype = ctypes.c_int32
    L.agimp_profile_substep.argtypes = [vp, ctypes.c_float, fp, ctypes.c_int32, vp]
    L.agimp_refine_levels_noalloc.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_int32, vp, vp]
    L.agimp_mlp_num_params.restype = ctypes.c_int32
    L.agimp_mlp_create.argtypes = [ctypes.c_int32, ctypes.POINTER(vp)]
    L.agimp_mlp_destroy.argtypes = [vp]
    L.agimp_mlp_set_params.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.agimp_mlp_get_params.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.agimp_mlp_forward.argtypes = [vp, vp, vp, ctypes.c_int64, vp]
    L.agimp_mlp_errors.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int32]
    L.agimp_wait_selftest.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
    L.agimp_mlp_grad.argtypes = [vp, vp, vp, ctypes.c_int64, vp, vp, vp]
    L.agimp_mlp_train_step.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_float, vp, vp]
    L.agimp_mlp_reset_optimizer.argtypes = [vp]
    L.agimp_set_surrogate.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_float), ctypes.c_float]
    L.agimp_batch_set_surrogate.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_float), ctypes.c_float]
    L.agimp_batch_surrogate_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                              ctypes.POINTER(ctypes.c_uint32)]
    L.agimp_set_recorder.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_int32]
    L.agimp_recorded.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]
    tp = ctypes.POINTER(Tuning)
    L.agimp_set_tuning.argtypes = [vp, tp]
    L.agimp_get_tuning.argtypes = [vp, tp]
    L.agimp_autotune.argtypes = [vp, ctypes.c_float, ctypes.c_int32, tp, vp]
    L.agimp_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ctypes.POINTER(vp)]
    L.agimp_batch_destroy.argtypes = [vp]
    L.agimp_batch_last_error.restype = ctypes.c_char_p
    L.agimp_batch_last_error.argtypes = [vp]
    L.agimp_batch_substep.argtypes = [vp, ctypes.c_float, ctypes.c_int32, vp]
    L.agimp_batch_set_graphs.argtypes = [vp, ctypes.c_int32]
    L.agimp_batch_set_tuning.argtypes = [vp, tp]
    L.agimp_batch_get_tuning.argtypes = [vp, tp]
    L.agimp_batch_autotune.argtypes = [vp, ctypes.c_float, ctypes.c_int32, tp, vp]
    L.agimp_batch_kernels_per_substep.argtypes = [vp]
    L.agimp_batch_kernels_per_substep.restype = ctypes.c_int32
    L.agimp_batch_profile_substep.argtypes = [vp, ctypes.c_float, fp, ctypes.c_int32, vp]
    L.agimp_get_particles_async.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.agimp_batch_positions_async.argtypes = [vp, vp, vp]
    L.agimp_batch_set_particles.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int32, vp]
    L.agimp_render_mask.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int32, vp]
    L.agimp_render_particles.argtypes = [vp, ctypes.c_int32, ctypes.c_float, vp, ctypes.c_int32, vp, ctypes.c_int32, vp]
    L.agimp_get_level_map.argtypes = [vp, vp, ip, ctypes.c_int32, vp]
    L.agimp_lattice_count.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64,
                                      ctypes.POINTER(Shape), ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.c_int32]
    L.agimp_lattice_fill.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(Shape),
                                     ctypes.c_int32, vp]
    L.agimp_random_fill.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(RandomBox), ctypes.c_int32, vp]
    L.agimp_set_level_map_rule.argtypes = [vp, ctypes.c_int32, vp]
    L.agimp_set_coarse_level_map.argtypes = [vp, vp, ctypes.c_int32, vp]
    L.agimp_render_scene3d.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(View3D), vp, ctypes.c_int32, vp]
    L.agimp_cell_lines.argtypes = [vp, vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32, vp]
    _lib = L
    return L


def check(status: int, handle=None, what: str = "", batch=False):
    if status != 0:
        L = load()
        msg = L.agimp_status_string(status).decode()
        if handle:
            detail = (L.agimp_batch_last_error if batch else L.agimp_last_error)(handle).decode()
            if detail:
                msg += ": " + detail
        raise AgimpError("%s failed (%d): %s" % (what or "agimp call", status, msg))
