"""The SkyImage dataset surface the drop-ins use in place of xarray's:
variables over (time, frequency, polarization, l, m), per-plane and uv
variables given as (dims, array), sizes over variables and dimension
coordinates, isel with slices (views), coordinate attributes, and the
shape-keeping data setter."""
import numpy as np
import pytest

from astroviper_b200.core.imaging.sky_image import SkyImage, make_sky_image, make_uv_coords


def _img():
    img = make_sky_image((0.1, -0.2), (12, 10), (1e-5, 2e-5), [1e9, 1.1e9], ["XX", "YY"],
                         [0.0])
    img["SKY"] = np.arange(1 * 2 * 2 * 12 * 10, dtype=np.float64).reshape(1, 2, 2, 12, 10)
    return img


def test_variables_and_sizes():
    img = _img()
    img["SKY_NORM"] = np.ones((1, 2, 2))
    img["VIS"] = (("time", "frequency", "polarization", "u", "v"),
                  np.zeros((1, 2, 2, 16, 14), complex))
    assert img["SKY_NORM"].dims == ("time", "frequency", "polarization")
    assert img.sizes == {"time": 1, "frequency": 2, "polarization": 2, "l": 12, "m": 10,
                         "u": 16, "v": 14}
    with pytest.raises(ValueError):
        img["BAD"] = np.zeros((2, 2))
    with pytest.raises(ValueError):
        img["BAD"] = (("time", "l"), np.zeros((1, 2, 3)))
    uv = SkyImage(coords={"u": np.arange(8), "v": np.arange(6), "l": np.arange(4)})
    uv["G"] = (("u", "v"), np.zeros((8, 6)))
    assert uv.sizes == {"u": 8, "v": 6, "l": 4}


def test_isel_gives_views_of_variables_and_coordinates():
    img = _img()
    img.coords["frequency"].attrs["channel_width"] = {"data": 1e6, "units": "Hz"}
    sub = img.isel(l=slice(2, 8), m=slice(1, 9))
    assert sub["SKY"].shape == (1, 2, 2, 6, 8)
    assert np.array_equal(sub.coords["l"].values, img.coords["l"].values[2:8])
    assert sub.sizes["l"] == 6 and sub.sizes["m"] == 8
    sub["SKY"].data[0, 0, 0, 0, 0] = -1.0
    assert img["SKY"].data[0, 0, 0, 2, 1] == -1.0
    assert sub.coords["frequency"].attrs["channel_width"]["data"] == 1e6
    with pytest.raises(TypeError):
        img.isel(l=3)


def test_data_setter_keeps_the_shape_and_copy_keeps_attrs():
    img = _img()
    new = np.zeros_like(img["SKY"].data)
    img["SKY"].data = new
    assert img["SKY"].data is new
    with pytest.raises(ValueError):
        img["SKY"].data = np.zeros((1, 2, 2, 6, 5))
    img.coords["time"].attrs["scale"] = "utc"
    deep = img.copy(deep=True)
    assert deep.coords["time"].attrs == {"scale": "utc"}
    assert deep["SKY"].data is not img["SKY"].data


def test_uv_coordinates_pair_with_the_image_cell():
    uv = make_uv_coords((8, 5), (1e-5, -2e-5))
    assert uv["u"][4] == 0.0 and uv["v"][2] == 0.0
    assert np.allclose(np.diff(uv["u"]), 1.0 / (8 * 1e-5))
    assert np.allclose(np.diff(uv["v"]), 1.0 / (5 * 2e-5))
