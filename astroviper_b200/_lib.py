"""ctypes binding of libav200.so (the C ABI declared in include/av200.h).

The library is built in-tree by ``astroviper_b200.build``.  There is no
fallback: if the library or a CUDA device is missing, every compute call
raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libav200.so")

AV_OK, AV_ERR_ARG, AV_ERR_CUDA, AV_ERR_TIMEOUT, AV_ERR_NAN, AV_ERR_UNSUPPORTED, AV_ERR_WORKSPACE = \
    range(7)
AV_F32, AV_F64, AV_C64, AV_C128 = range(4)
AV_TUNE_GRID_CHUNKS_PER_SM, AV_TUNE_DEGRID_CHUNKS_PER_SM, AV_TUNE_GRID_LANES, \
    AV_TUNE_DEGRID_LANES, AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US = range(5)
AV_HOGBOM_BARRIER_TIMEOUT_US_DEFAULT = 2000000
AV_GRID_LANES_MMA, AV_GRID_LANES_ROWS, AV_GRID_LANES_AUTO = 1, 2, 3
AV_DEGRID_LANES_TF32, AV_DEGRID_LANES_FP32, AV_DEGRID_LANES_AUTO, AV_DEGRID_LANES_TC05 = 1, 2, 3, 4

_vp = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_sz = ctypes.c_size_t

# the common arguments of av_mosaic_grid and av_aperture_grid
_MOSAIC = [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64,
           _i64, _i64, _vp, _i, _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64, _i64, _i64, _i64]

# name: (restype, [argtypes])
SIGNATURES = {
    "av_version": (_i, []),
    "av_last_error": (ctypes.c_char_p, []),
    "av_device_sm_count": (_i, []),
    "av_probe_fp64_mma": (_i, [_vp, _vp]),
    "av_launch_count": (ctypes.c_ulonglong, []),
    "av_tune_set": (_i, [_i, _i64]),
    "av_tune_get": (_i64, [_i]),
    "av_pswf": (_i, [_vp, _i64, _vp, _vp, _vp]),
    "av_pswf_table": (_i, [_vp, _i, _i, _vp]),
    "av_corr_term": (_i, [_vp, _i64, _i64, _vp]),
    "av_pswf_kernel4d": (_i, [_vp, _i, _i, _vp]),
    "av_grid_plain": (_i, [_vp, _i, _vp, _i, _i, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp,
                           _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64, _i64, _i64, _i64, _vp]),
    "av_grid_tiled_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64, _i]),
    "av_grid_tiled_plan": (_i, [_vp, _vp, _vp, _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64,
                                _i64, _vp, _sz, _vp]),
    "av_grid_tiled_plan_weighted": (_i, [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _d, _d, _i, _i,
                                         _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "av_grid_tiled_clear": (_i, [_vp, _i, _i64, _i64, _i64, _i, _i64, _i64, _i64, _i64, _vp,
                                 _sz, _vp]),
    "av_tiled_plan_shared": (_i, [_vp, _vp, _vp, _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64,
                                  _i64, _vp, _sz, _vp]),
    "av_tiled_plan_counts": (_i, [_i64, _i64, _i64, _i64, _i64, _i64, _i, _vp, _sz, _vp, _vp]),
    "av_degrid_fault_read": (_i, [_vp, _i, _vp]),
    "av_grid_tiled_execute": (_i, [_vp, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp, _i64, _i64, _i,
                                   _i, _i64, _i64, _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "av_grid_tiled_execute_det": (_i, [_vp, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp, _i64, _i64,
                                       _i, _i, _i64, _i64, _i64, _i64, _i64, _i64, _vp, _sz, _vp,
                                       _sz, _vp]),
    "av_grid_tiled_det_workspace_size": (_sz, [_i64, _i64, _i64, _i64]),
    "av_tiled_plan_order_rows": (_i, [_i64, _i64, _i64, _i64, _i64, _i64, _i, _vp, _sz, _vp]),
    "av_grid_tiled": (_i, [_vp, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _i64,
                           _i64, _d, _d, _i, _i, _i64, _i64, _i64, _i64, _i64, _i64, _vp, _sz,
                           _vp]),
    "av_degrid_plain": (_i, [_vp, _vp, _vp, _i, _vp, _d, _d, _d, _d, _vp, _i, _i64, _i64, _i64,
                             _i64, _vp, _d, _i, _i, _vp, _vp, _vp, _i64, _i64, _i64, _i64,
                             _vp]),
    "av_degrid_plain_adjoint": (_i, [_vp, _vp, _vp, _i, _vp, _d, _d, _d, _d, _vp, _i, _i64, _i64,
                                     _i64, _i64, _vp, _d, _i, _i, _vp, _vp, _vp, _i64, _i64,
                                     _i64, _i64, _vp]),
    "av_degrid_tiled_adjoint": (_i, [_vp, _i, _vp, _i, _vp, _i64, _i64, _i64, _i64, _i, _i, _vp,
                                     _vp, _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "av_degrid_tiled_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64, _i]),
    "av_degrid_tiled_plan": (_i, [_vp, _vp, _vp, _d, _d, _d, _d, _i64, _i64, _i64, _i, _i, _i64,
                                  _i64, _i64, _vp, _sz, _vp]),
    "av_degrid_tiled_execute": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _i64, _i64, _i64, _i64, _vp,
                                     _i, _i, _vp, _vp, _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "av_degrid_tiled": (_i, [_vp, _vp, _vp, _i, _i, _vp, _d, _d, _d, _d, _vp, _i, _i64, _i64,
                             _i64, _i64, _vp, _d, _i, _i, _vp, _vp, _vp, _i64, _i64, _i64, _i64,
                             _vp, _sz, _vp]),
    "av_fft_workspace_size": (_sz, [_i64, _i64, _i64, _i]),
    "av_grid_to_image_workspace_size": (_sz, [_i64, _i64, _i64]),
    "av_grid_to_image": (_i, [_vp, _i, _vp, _vp, _i, _i64, _i64, _i64, _i, _vp, _sz, _vp]),
    "av_image_to_grid": (_i, [_vp, _i, _vp, _i, _i64, _i64, _i64, _i, _vp, _sz, _vp]),
    "av_fft_shifted": (_i, [_vp, _vp, _i, _i64, _i64, _i64, _i, _vp, _sz, _vp]),
    "av_weight_density": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp, _i64, _i64, _d, _d, _i64, _i64,
                               _i64, _i64, _vp]),
    "av_briggs_factors_workspace_size": (_sz, [_i64]),
    "av_briggs_factors": (_i, [_vp, _vp, _vp, _i64, _i64, _i64, _d, _vp, _sz, _vp]),
    "av_briggs_factors_noalloc": (_i, [_vp, _vp, _vp, _i64, _i64, _i64, _d, _vp]),
    "av_imaging_weight_degrid": (_i, [_vp, _vp, _i, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp,
                                      _i, _i64, _i64, _d, _d, _i64, _i64, _i64, _i64, _vp]),
    "av_briggs_apply": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _i, _vp, _i64, _i64, _d, _d,
                             _i64, _i64, _i64, _i64, _vp, _vp]),
    "av_maximg": (_i, [_vp, _vp, _i, _i64, _i64, _vp, _vp]),
    "av_hogbom_state_size": (_sz, []),
    "av_hogbom_workspace_size": (_sz, [_i64, _i64, _i]),
    "av_hogbom_run": (_i, [_vp, _vp, _vp, _vp, _i, _i64, _i64, _i64, _i64, _i, _i, _i, _i, _i,
                           _i, _i, _i, _d, _d, _d, _vp, _i, _vp, _sz, _vp]),
    "av_hogbom_state_read": (_i, [_vp, _vp, _vp, _vp]),
    "av_abs_sum_workspace_size": (_sz, [_i64, _i]),
    "av_abs_sum_ordered": (_i, [_vp, _i, _i64, _vp, _vp, _sz, _vp]),
    "av_pol_transform": (_i, [_vp, _i, _vp, _i, _vp, _i, _i, _i64, _i64, _vp]),
    "av_argmax_workspace_size": (_sz, [_i64]),
    "av_argmax": (_i, [_vp, _i, _i64, _i, _vp, _vp, _vp, _sz, _vp]),
    "av_psf_sidelobe_workspace_size": (_sz, [_i64, _i64, _i, _i]),
    "av_psf_sidelobe": (_i, [_vp, _i, _i64, _i64, _i, _i, _d, _vp, _vp, _sz, _vp]),
    "av_plane_sum_workspace_size": (_sz, [_i64, _i64]),
    "av_plane_rescale": (_i, [_vp, _i, _i64, _i64, _i, _d, _vp, _vp, _vp]),
    "av_apply_pb": (_i, [_vp, _i, _i64, _i64, _i64, _vp, _i, _i64, _i64, _i64, _i64, _i, _vp]),
    "av_plane_sum": (_i, [_vp, _i, _i64, _i64, _vp, _vp, _sz, _vp]),
    "av_vis_residual": (_i, [_vp, _vp, _vp, _i, _i64, _vp]),
    "av_cf_phase_product": (_i, [_vp, _i, _vp, _vp, _i64, _i64, _i64, _vp]),
    "av_airy_pattern": (_i, [_vp, _vp, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _d,
                             _d, _i, _i, _i, _vp]),
    "av_mosaic_grid": (_i, _MOSAIC + [_vp]),
    "av_aperture_grid_workspace_size": (_sz, [_i64, _i64, _i64]),
    "av_mosaic_tiled_workspace_size": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64, _i]),
    "av_mosaic_tiled_plan": (_i, [_vp, _vp, _vp, _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64,
                                  _i64, _vp, _sz, _vp]),
    "av_mosaic_tiled_execute": (_i, _MOSAIC + [_vp, _sz, _vp]),
    "av_aperture_grid": (_i, _MOSAIC + [_vp, _sz, _vp]),
}

_LIB = None


class AVError(RuntimeError):
    """A libav200 call failed (status code in .code)."""

    def __init__(self, msg, code):
        super().__init__(msg)
        self.code = code


def lib():
    """The loaded library; raises ImportError when it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libav200.so is not built ({LIB_PATH}); run "
                          "`python -m astroviper_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def last_error():
    return lib().av_last_error().decode(errors="replace")


def check(rc, what):
    if rc == AV_OK:
        return
    msg = last_error() or f"{what} failed"
    if rc == AV_ERR_NAN:
        raise ValueError(msg)
    if rc == AV_ERR_ARG:
        raise ValueError(f"{what}: {msg}")
    raise AVError(f"{what}: {msg}", rc)
