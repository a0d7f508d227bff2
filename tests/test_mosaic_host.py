"""Host logic of the mosaic / A-projection gridder on CPU: the
convolution-function maps, the support search and the resize /
normalisation against the reference's outputs (tests/golden/mosaic.npz,
made by tests/golden/make_golden_mosaic.py), the phase gradient's geometry,
and the wrappers' argument checks (which raise before any device work)."""
import numpy as np
import pytest

from conftest import golden


def test_cf_baseline_map_matches_reference():
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    g = golden("mosaic.npz")
    m, pairs = G.create_cf_baseline_map(g["cbm_unique_ant_indx"], g["cbm_baseline_ant"], 2)
    assert np.array_equal(m, g["cbm_map"]) and np.array_equal(pairs, g["cbm_pairs"])


def test_cf_chan_map_matches_reference():
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    g = golden("mosaic.npz")
    for i in range(int(g["n_ccm"])):
        m, pf = G.create_cf_chan_map(g[f"ccm{i}_freq"], float(g[f"ccm{i}_tol"]))
        assert np.array_equal(m, g[f"ccm{i}_map"]) and np.array_equal(pf, g[f"ccm{i}_pbfreq"]), i
    assert G.find_nearest([1.0, 2.0, 4.0], 3.1) == (2, 4.0)


def test_support_and_resize_match_reference():
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    g = golden("mosaic.npz")
    os_, ms = g["gcf_oversampling"], g["gcf_max_support"]
    assert G.calc_conv_size(g["ckc"][1, 0, 0], g["grid_image_size_padded"], float(g["gcf_cut"]),
                            os_, ms) == list(g["conv_size_one"])
    gcf = {"oversampling": os_, "max_support": ms, "support_cut_level": float(g["gcf_cut"]),
           "resize_conv_size": (ms + 1) * os_}
    rk, rkc, sup = G.resize_and_calc_support(g["ck"], g["ckc"], gcf,
                                             {"image_size_padded": g["grid_image_size_padded"]})
    assert np.array_equal(sup, g["support"])
    assert np.array_equal(rk, g["rk"]) and np.array_equal(rkc, g["rkc"])
    with pytest.raises(AssertionError, match="support_cut_level too small"):
        G.calc_conv_size(np.ones((8, 8)), np.array([8, 8]), 0.5, os_, ms)


def test_phase_gradient_geometry():
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    gcf = {"phase_direction": np.array([0.3, -0.5]), "oversampling": np.array([4, 4]),
           "resize_conv_size": np.array([48, 48])}
    gp = {"image_size_padded": np.array([96, 96]), "cell_size": np.array([-1e-4, 1e-4])}
    pg = G.make_phase_gradient(np.array([[0.3, -0.5]]), gcf, gp)
    assert pg.shape == (1, 48, 48) and np.allclose(pg, 1.0)
    # a field 3 cells north: a ramp along v only, -2 pi 3 / (96 x 4) per function cell
    dec = -0.5 + 3e-4
    pg = G.make_phase_gradient(np.array([[0.3, dec]]), gcf, gp)
    m = np.sin(dec) * np.cos(-0.5) - np.cos(dec) * np.sin(-0.5)
    step = -(m / 1e-4) * 2 * np.pi / (96 * 4)
    assert np.allclose(np.angle(pg[0, 24, 25] / pg[0, 24, 24]), step, rtol=1e-9)
    assert np.allclose(np.angle(pg[0, 25, 24] / pg[0, 24, 24]), 0.0, atol=1e-12)


def test_mosaic_wrapper_helpers_and_errors():
    from astroviper_b200.core.imaging.imaging_utils import mosaic_grid as M
    assert M.ndim_list((2, 3)) == [[None] * 3, [None] * 3]
    assert M.tree_sum_list([1, 2, 3, 4, 5]) == [15]
    w = np.ones((1, 1, 1, 1))
    with pytest.raises(TypeError, match="complex_grid"):
        M.mosaic_grid_numpy_wrap(None, None, w, None, None, None, None, None, None, None, None,
                                 {"chan_mode": "cube", "image_size_padded": [8, 8],
                                  "complex_grid": False})


def test_oracle_mosaic_grid_matches_reference():
    """The oracle's C restatement of mosaic_grid_jit against the Numba
    kernel's own grids (the CPU baseline of the benchmark)."""
    import oracle as O
    g = golden("mosaic.npz")
    cf = g["rk"] * g["mg_pg"][0]
    n_uv = g["grid_image_size_padded"]
    for tag, cm, nic in (("cube", np.arange(2), 2), ("cont", np.zeros(2, dtype=int), 1)):
        for do_psf in (False, True):
            grid = np.zeros((nic, 2, n_uv[0], n_uv[1]), dtype=np.complex128)
            sw = np.zeros((nic, 2))
            O.mosaic_grid(grid, sw, do_psf, g["mg_vis"], g["mg_uvw"], g["mg_freq"], cm,
                          np.arange(2), g["mg_cfb"], g["mg_cfc"], g["mg_cfp"], g["mg_wt"], cf,
                          g["support"], n_uv, g["grid_cell"], g["gcf_oversampling"])
            want = g[f"mg_{tag}_{int(do_psf)}_grid"]
            assert np.array_equal(grid, want), (tag, do_psf)
            assert np.array_equal(sw, g[f"mg_{tag}_{int(do_psf)}_sw"]), (tag, do_psf)


def test_check_params_semantics(capsys):
    """utils/check_params.py:4-189: defaults written, lists by length and
    element type, scalars by type / value / range, dict entries filled."""
    from astroviper_b200.utils.check_params import check_params
    d = {}
    assert check_params(d, "x", [int], default=3) and d["x"] == 3
    assert not check_params(d, "y", [int])
    assert "must be specified" in capsys.readouterr().out
    d = {"a": [1, 2], "b": [1, 2.5], "c": [1, 2, 3], "s": "cube", "r": 11.0}
    assert check_params(d, "a", [list], list_acceptable_data_types=[int], list_len=2)
    assert not check_params(d, "b", [list], list_acceptable_data_types=[int], list_len=2)
    assert "Wrong type of" in capsys.readouterr().out
    assert not check_params(d, "c", [list], list_acceptable_data_types=[int], list_len=2)
    assert "Wrong length" in capsys.readouterr().out
    assert check_params(d, "c", [list, np.array], list_acceptable_data_types=[int], list_len=-1)
    assert not check_params(d, "s", [str], acceptable_data=["continuum"])
    assert not check_params(d, "r", [float], acceptable_range=[1, 10])
    assert "within the range" in capsys.readouterr().out
    assert not check_params(d, "r", [int])
    # a dict parameter: missing entries from the default; it passes whatever
    # its entries' checks find, as in the reference
    d = {"p": {"k1": "wrong type"}}
    assert check_params(d, "p", [dict], default={"k1": 1, "k2": 2.0})
    assert d["p"] == {"k1": "wrong type", "k2": 2.0}


def test_grid_and_gcf_param_checks():
    from astroviper_b200.core.imaging.check_imaging_parameters import (check_gcf_params,
                                                                       check_grid_params)
    g = {"image_size": [100, 80], "cell_size": [1e-5, 1e-5], "fft_padding": 1.5}
    assert check_grid_params(g)
    assert np.array_equal(g["image_size_padded"], [150, 120])
    assert np.array_equal(g["image_center"], [50, 40]) and g["chan_mode"] == "cube"
    assert not check_grid_params({"image_size": [100, 80], "cell_size": [1e-5, 1e-5],
                                  "fft_padding": 20.0})
    gcf = {"freq_chan": [1e9], "list_dish_diameters": [12.0, 25.0],
           "list_blockage_diameters": [0.75], "unique_ant_indx": [0, 1], "pol": ["XX"]}
    assert not check_gcf_params(gcf)  # diameters of different lengths
    gcf["list_blockage_diameters"] = [0.75, 0.0]
    assert check_gcf_params(gcf)
    assert gcf["function"] == "casa_airy" and np.array_equal(gcf["oversampling"], [10, 10])
    assert gcf["max_support"].dtype.kind == "i" and gcf["a_chan_num_chunk"] == 3


def test_check_sel_params_data_groups():
    import types
    from astroviper_b200.utils.check_params import check_sel_params
    xds = types.SimpleNamespace(data_vars=["VISIBILITY", "WEIGHT"],
                                attrs={"data_groups": {"base": {"correlated_data": "VISIBILITY",
                                                                "weight": "WEIGHT"}}})
    gin, gout = check_sel_params(xds, {}, default_data_group_in_name="base",
                                 default_data_group_out_name="imaging",
                                 default_data_group_out_modified={"weight_imaging":
                                                                  "WEIGHT_IMAGING"})
    assert gin["data_group_in_name"] == "base" and gout["data_group_out_name"] == "imaging"
    assert gout["weight_imaging"] == "WEIGHT_IMAGING" and gout["weight"] == "WEIGHT"
    with pytest.raises(AssertionError, match="not found in xds data_groups"):
        check_sel_params(xds, {"data_group_in_name": "other"})
    with pytest.raises(AssertionError, match="already exists in xds"):
        check_sel_params(xds, {"data_group_out": {"weight": "WEIGHT"}},
                         default_data_group_in_name="base")


def test_minimal_dataset():
    from astroviper_b200.core.imaging.dataset import Dataset
    ds = Dataset()
    assert len(ds) == 0
    ds["A"] = (("baseline", "u"), np.zeros((5, 3)))
    ds["B"] = (("baseline",), np.arange(5))
    assert len(ds) == 2 and ds.baseline.size == 5 and ds.sizes == {"baseline": 5, "u": 3}
    assert ds["B"].dims == ("baseline",) and "A" in ds
    with pytest.raises(ValueError):
        ds["C"] = (("baseline",), np.arange(4))
    ds2 = ds.assign_coords({"u": np.arange(3)})
    assert "u" in ds2.coords and "u" not in ds.coords
