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
