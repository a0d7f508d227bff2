"""Host-side behaviour of the drop-in API that needs no GPU: parameter
validation and error messages (deconvolution.py:74-120, bindings.cpp:24-42,
81-106 of the reference), dtype helpers, overload selection, module layout."""
import numpy as np
import pytest

from astroviper_b200.core.imaging import deconvolution as D
from astroviper_b200.core.imaging.deconvolvers import hogbom


def test_validate_defaults_and_partial():
    assert D._validate_deconv_params({}) == {"gain": 0.1, "niter": 1000, "threshold": 0.0,
                                             "clean_box": (-1, -1, -1, -1)}
    got = D._validate_deconv_params({"gain": 0.25})
    assert got["gain"] == 0.25 and got["niter"] == 1000
    p = {"gain": 0.05, "niter": 7, "threshold": 2e-6, "clean_box": (1, 2, 3, 4)}
    assert D._validate_deconv_params(dict(p)) == p


@pytest.mark.parametrize("gain", [0.0, -0.5, 1.0001, 3.0])
def test_validate_gain_rejected(gain):
    with pytest.raises(ValueError, match="CLEAN gain must be between 0 and 1"):
        D._validate_deconv_params({"gain": gain})


@pytest.mark.parametrize("niter", [0, -3, 2.5, "10", None])
def test_validate_niter_rejected(niter):
    with pytest.raises(ValueError, match="Maximum number of iterations must be a positive integer"):
        D._validate_deconv_params({"niter": niter})


def test_validate_threshold():
    for t in (None, 0.0, 0.5):
        assert D._validate_deconv_params({"threshold": t})["threshold"] == t
    with pytest.raises(ValueError, match="Threshold must be non-negative or None"):
        D._validate_deconv_params({"threshold": -1e-9})


def test_validate_edge_values_and_order_as_reference():
    # deconvolution.py:100-118: a NaN gain fails "0 < g <= 1"; a NaN threshold
    # passes "not < 0"; the parameters are checked in the order gain, niter,
    # threshold, clean_box, defaults filled in on the way
    with pytest.raises(ValueError, match="CLEAN gain"):
        D._validate_deconv_params({"gain": float("nan")})
    got = D._validate_deconv_params({"threshold": float("nan")})
    assert np.isnan(got["threshold"]) and got["gain"] == 0.1
    p = {"niter": 0, "clean_box": "x"}
    with pytest.raises(ValueError, match="Maximum number of iterations"):
        D._validate_deconv_params(p)
    assert p["gain"] == 0.1 and "threshold" not in p
    assert D._validate_deconv_params({"clean_box": None})["clean_box"] is None


@pytest.mark.parametrize("box", [(1, 2), (1, 2, 3), (1, 2, 3, 4, 5), "box", []])
def test_validate_clean_box_rejected(box):
    with pytest.raises(ValueError, match="Clean box must be a 4-tuple.*or None"):
        D._validate_deconv_params({"clean_box": box})


def test_hogbom_clean_shape_errors():
    a = np.zeros((8, 8), np.float32)
    with pytest.raises(ValueError, match="dirty_image must be a 2D numpy array"):
        D.hogbom_clean(np.zeros(8), a, {})
    with pytest.raises(ValueError, match="psf must be a 2D numpy array"):
        D.hogbom_clean(a, np.zeros((2, 8, 8)), {})
    with pytest.raises(ValueError, match="dirty_image and psf must have same shape"):
        D.hogbom_clean(a, np.zeros((8, 9), np.float32), {})


def test_clean_and_maximg_errors():
    a = np.zeros((8, 8), np.float32)
    with pytest.raises(RuntimeError, match="Dirty image must be 2D"):
        hogbom.clean(np.zeros(8, np.float32), a)
    with pytest.raises(RuntimeError, match="PSF must be 2D"):
        hogbom.clean(a, np.zeros(8, np.float32))
    with pytest.raises(RuntimeError, match="PSF dimensions must match image spatial dimensions"):
        hogbom.clean(a, np.zeros((8, 4), np.float32))
    with pytest.raises(RuntimeError, match="Mask must be 2D with same spatial dimensions"):
        hogbom.clean(a, a, mask=np.ones((4, 4), np.float32))
    with pytest.raises(RuntimeError, match="Image must be 2D array"):
        hogbom.maximg(np.zeros(5, np.float32))
    with pytest.raises(RuntimeError, match="Image must be 2D array"):
        hogbom.maximg(np.zeros((2, 5, 5), np.float32))
    with pytest.raises(RuntimeError, match="Mask dimensions must match image spatial dimensions"):
        hogbom.maximg(a, np.ones((4, 4), np.float32))


def test_dtype_helpers():
    assert hogbom.get_dtype_name(np.zeros(2, np.float32)) == "float32"
    assert hogbom.get_dtype_name(np.zeros(2, np.float64)) == "float64"
    assert hogbom.get_dtype_name(np.zeros(2, np.int32)) == "int32"
    assert hogbom.is_float32(np.zeros(2, np.float32)) is True
    assert hogbom.is_float32(np.zeros(2, np.float64)) is False
    assert hogbom.is_float64(np.zeros(2, np.float64)) is True
    assert hogbom.is_float64(np.zeros(2, np.int32)) is False


def test_overload_selection_follows_the_reference():
    """FP64 only when every array argument is float64 (an explicit empty
    float32 mask selects FP32, as pybind11 does with the reference)."""
    f64 = np.zeros((4, 4))
    f32 = np.zeros((4, 4), np.float32)
    assert hogbom._pick_dtype(f64, f64, None) == np.float64
    assert hogbom._pick_dtype(f64, f64, np.array([], np.float32)) == np.float32
    assert hogbom._pick_dtype(f32, f32, None) == np.float32
    assert hogbom._pick_dtype(f64, f32, None) == np.float32
    assert hogbom._pick_dtype(np.zeros((4, 4), np.int32), f64, None) == np.float32


def test_clean_box_parsing():
    assert hogbom._box((-1, -1, -1, -1), 10, 8) == (0, 10, 0, 8)
    assert hogbom._box((3, 99, -5, 2), 10, 8) == (3, 10, 0, 2)
    assert hogbom._box((12, 5, 7, 3), 10, 8) == (9, 10, 7, 8)


def test_module_layout_mirrors_reference():
    import importlib
    for mod, names in {
        "astroviper_b200.core.imaging.imaging_utils.standard_grid": [
            "standard_grid_numpy_wrap_input_checked", "standard_grid_numpy_wrap",
            "standard_grid_psf_numpy_wrap", "standard_grid_jit", "grid2image_spheroid_ms4",
            "standard_imaging_weight_degrid_numpy_wrap", "standard_imaging_weight_degrid_jit"],
        "astroviper_b200.core.imaging.imaging_utils.standard_degrid": [
            "sgrid", "sgrid_numba", "dgrid", "dgrid_optimized", "dgrid2", "dgrid_numba",
            "degrid_spheroid_ms4"],
        "astroviper_b200.core.imaging.imaging_utils.gcf_prolate_spheroidal": [
            "create_prolate_spheroidal_kernel", "create_prolate_spheroidal_kernel_1D",
            "prolate_spheroidal_function", "coordinates", "coordinates2"],
        "astroviper_b200.core.imaging.imaging_utils.make_point_spread_function": ["make_psf"],
        "astroviper_b200.core.imaging.imaging_weighting.grid_imaging_weights": [
            "grid_imaging_weights", "grid_imaging_weights_jit", "degrid_imaging_weights",
            "degrid_imaging_weights_jit"],
        "astroviper_b200.core.imaging.imaging_weighting.briggs_weighting": [
            "calculate_briggs_params"],
        "astroviper_b200.core.imaging.calculate_imaging_weights": ["calculate_imaging_weights"],
        "astroviper_b200.core.imaging.deconvolution": ["hogbom_clean", "progress_callback"],
        "astroviper_b200.core.imaging.fft": ["fft_lm_to_uv"],
        "astroviper_b200.core.imaging.ifft": ["ifft_uv_to_lm"],
        "astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation": [
            "make_image_xds", "remove_padding", "make_empty_padded_uv_image", "apply_pb",
            "_mult_div", "fft_to_uv", "ifft_to_lm", "correct_fft_to_uv", "correct_ifft_to_lm",
            "grid2xradio_spheroid_ms4"],
        "astroviper_b200.core.imaging.imaging_utils.make_primary_beam": [
            "cube_single_field_primary_beam"],
    }.items():
        m = importlib.import_module(mod)
        for n in names:
            assert callable(getattr(m, n)), f"{mod}.{n}"


def test_sgrid_numba_matches_python_round():
    """sgrid math against Python round() (test_standard_degrid.py:89-120 of the
    reference, restated)."""
    from astroviper_b200.core.imaging.imaging_utils.standard_degrid import sgrid_numba
    uvw = np.array([1.0, 2.0, 3.0])
    c = 299792458.0
    scale = np.array([1.0e-4, 1.0e-4, 0.0])
    offset = np.array([500.0, 500.0, 0.0])
    phasor, loc, off = sgrid_numba(uvw, 0.0, 1.0e9, c, scale, offset, 1)
    ex = scale[0] * uvw[0] * 1.0e9 / c + offset[0]
    ey = scale[1] * uvw[1] * 1.0e9 / c + offset[1]
    assert loc[0] == int(round(ex)) and loc[1] == int(round(ey))
    assert off[0] == int(round((round(ex) - ex) * 1)) and off[1] == int(round((round(ey) - ey)))
    assert phasor == 1.0 + 0j


def test_product_path_refuses_to_run_without_gpu():
    """No CPU fallback: compute entry points raise when no CUDA device is
    visible."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from astroviper_b200.core.imaging.imaging_utils.gcf_prolate_spheroidal import \
        create_prolate_spheroidal_kernel_1D
    with pytest.raises(RuntimeError, match="needs a CUDA device"):
        create_prolate_spheroidal_kernel_1D(100, 7)
    from astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation import (
        correct_ifft_to_lm, make_image_xds)
    img = make_image_xds([8, 8], [1e-5, 1e-5], 1e9, None, [0.0, 0.0])
    with pytest.raises(RuntimeError, match="needs a CUDA device"):
        correct_ifft_to_lm(img)


def test_stream_time_chunks_cover_every_step_once():
    """The time chunks of the streamed host-input paths tile range(nt)."""
    from astroviper_b200 import _kernels as K
    for nt, per_t, cb in ((1, 10, 4096), (7, 4096, 4096), (100, 1000, 4096), (5, 1, None),
                          (1000, 3 << 20, None)):
        ch = K.time_chunks(nt, per_t, cb)
        assert ch[0][0] == 0 and ch[-1][1] == nt
        assert all(a[1] == b[0] for a, b in zip(ch, ch[1:]))
        assert all(t1 > t0 for t0, t1 in ch)
        if cb is not None:
            assert len(ch) == min(nt, -(-nt * per_t // cb))


def test_streamable_needs_numpy_arrays_of_two_chunks():
    from astroviper_b200 import _host as H
    a = np.zeros((8, 100))
    assert H.streamable(a, None, min_bytes=a.nbytes)
    assert not H.streamable(a, min_bytes=a.nbytes + 1)
    assert not H.streamable(a, np.zeros((7, 100)), min_bytes=1)
    assert not H.streamable(None, min_bytes=1)
    assert not H.streamable(a, [[1.0]], min_bytes=1)
