"""B200 adaptive GIMP substep: the reference's AdaptiveGIMP simulator over
hand-written sm_100a CUDA kernels (libagimp.so, C ABI in include/agimp.h)."""
from ._capi import AgimpError, load  # noqa: F401
from .simulator import ACTIVATED, CULLING, GHOST, T_JUNCTION, UNACTIVATED, AdaptiveGIMP, align_size  # noqa: F401
from . import scenes  # noqa: F401
