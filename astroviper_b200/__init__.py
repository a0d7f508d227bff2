"""astroviper_b200: the standard-gridder imaging path of astroviper on B200.

Module paths mirror the reference package (``astroviper.core.imaging...``):
``astroviper_b200.core.imaging.imaging_utils.standard_grid`` etc. keep the
reference's function names, arguments, in-place behaviour and errors, and run
on hand-written sm_100a kernels (``libav200.so``, C ABI in include/av200.h).

``config.precision`` selects the arithmetic of the gridding kernels:
"fp32" (default; tiled FP32 kernels, FP64 index math) or "fp64" (plain FP64
kernels, the reference's per-sample arithmetic).  Every gridding function also
takes ``precision=`` as a keyword.
"""
from .config import config  # noqa: F401

__version__ = "0.1.0"
