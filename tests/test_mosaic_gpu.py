"""The mosaic / A-projection gridder on the GPU against the reference's own
outputs (tests/golden/mosaic.npz): the Airy-disk beams of
make_pb_symmetric.py, the baseline patterns and their transforms, the
support and resize steps on functions built here, and mosaic_grid_jit /
aperture_grid_jit (Numba) on the reference's functions - grids within 1e-12
relative (FP64, atomics change only the summation order)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (nb if nb else 1.0)


def test_airy_beams_match_reference():
    from astroviper_b200.core.imaging.imaging_utils import make_pb_symmetric as PB
    g = golden("mosaic.npz")
    gp = {"cell_size": g["pb_cell"], "image_size": g["pb_size"], "image_center": g["pb_center"]}
    for name in ("airy_disk", "casa_airy_disk", "airy_disk_rorder", "casa_airy_disk_rorder"):
        for ip in (1, 2):
            pbp = {"list_dish_diameters": g["pb_dish"], "list_blockage_diameters": g["pb_block"],
                   "ipower": ip}
            got = getattr(PB, name)(g["pb_freq"], np.array([0, 1]), pbp, gp)
            want = g[f"pb_{name}_{ip}"]
            assert got.shape == want.shape, name
            # J1 from CUDA against scipy's: a few ulp
            assert np.allclose(got, want, rtol=1e-13, atol=1e-15), (name, ip)


def test_baseline_patterns_kernels_and_supports():
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    from astroviper_b200.core.imaging.imaging_utils import make_pb_symmetric as PB
    g = golden("mosaic.npz")
    os_, ms = g["gcf_oversampling"], g["gcf_max_support"]
    gcf = {"list_dish_diameters": np.array([12.0, 25.0]),
           "list_blockage_diameters": np.array([0.75, 0.0]), "oversampling": os_,
           "max_support": ms, "support_cut_level": float(g["gcf_cut"]),
           "resize_conv_size": (ms + 1) * os_}
    grid = {"image_size": np.array([64, 64]), "image_size_padded": g["grid_image_size_padded"],
            "cell_size": g["grid_cell"]}
    pairs = np.array([[0, 0], [0, 1], [1, 1]])
    for ip, key in ((1, "bp1"), (2, "bp2")):
        gcf["ipower"] = ip
        bp = G.make_baseline_patterns(np.array([1.1e9, 1.4e9]), np.array([0]), pairs,
                                      PB.airy_disk_rorder, dict(gcf), grid)
        assert np.allclose(bp, g[key], rtol=1e-13, atol=1e-15), key
    ck = G.conv_kernels(g["bp1"])
    ckc = G.conv_kernels(g["bp2"])
    for got, want in ((ck, g["ck"]), (ckc, g["ckc"])):
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    rk, rkc, sup = G.resize_and_calc_support(ck, ckc, gcf, grid)
    assert np.array_equal(sup, g["support"])
    assert rel(rk, g["rk"]) <= 1e-12 and rel(rkc, g["rkc"]) <= 1e-12


@pytest.mark.parametrize("tag", ["cube", "cont"])
def test_mosaic_and_aperture_grids_match_reference(tag):
    from astroviper_b200.core.imaging.imaging_utils import mosaic_grid as M
    g = golden("mosaic.npz")
    nchan, npol = 2, 2
    chan_map = np.arange(nchan) if tag == "cube" else np.zeros(nchan, dtype=int)
    nic = nchan if tag == "cube" else 1
    n_uv = g["grid_image_size_padded"]
    common = (g["mg_uvw"], g["mg_freq"], chan_map, np.arange(npol), g["mg_cfb"], g["mg_cfc"],
              g["mg_cfp"], g["mg_wt"])
    for do_psf in (False, True):
        grid = np.zeros((nic, npol, n_uv[0], n_uv[1]), dtype=np.complex128)
        sw = np.zeros((nic, npol))
        M.mosaic_grid_jit(grid, sw, do_psf, g["mg_vis"], *common, g["rk"], n_uv, g["grid_cell"],
                          g["support"], g["gcf_oversampling"], g["mg_pg"])
        want = g[f"mg_{tag}_{int(do_psf)}_grid"]
        assert rel(grid, want) <= 1e-12, (tag, do_psf)
        assert np.allclose(sw, g[f"mg_{tag}_{int(do_psf)}_sw"], rtol=1e-12), (tag, do_psf)
    grid = np.zeros((nic, npol, n_uv[0], n_uv[1]), dtype=np.complex128)
    sw = np.zeros((nic, npol))
    M.aperture_grid_jit(grid, sw, *common, g["rkc"], n_uv, g["grid_cell"], g["support"],
                        g["gcf_oversampling"], g["mg_pg"])
    assert rel(grid, g[f"ag_{tag}_grid"]) <= 1e-12
    assert np.allclose(sw, g[f"ag_{tag}_sw"], rtol=1e-12)


def test_mosaic_wrappers_grid_through_the_kernel():
    from astroviper_b200.core.imaging.imaging_utils import mosaic_grid as M
    g = golden("mosaic.npz")
    params = {"chan_mode": "cube", "image_size_padded": g["grid_image_size_padded"],
              "cell_size": g["grid_cell"], "oversampling": g["gcf_oversampling"],
              "complex_grid": True, "do_psf": False, "field_id": 0}
    gr, sw = M.mosaic_grid_numpy_wrap(g["mg_vis"], g["mg_uvw"], g["mg_wt"], None, g["mg_cfb"],
                                      g["mg_cfc"], g["mg_cfp"], g["rk"], g["support"], g["mg_pg"],
                                      g["mg_freq"], params)
    assert rel(gr, g["mg_cube_0_grid"]) <= 1e-12
    params["do_psf"] = True
    gr, sw = M.mosaic_psf_grid_numpy_wrap(g["mg_uvw"], g["mg_wt"], None, g["mg_cfb"],
                                          g["mg_cfc"], g["mg_cfp"], g["rk"], g["support"],
                                          g["mg_pg"], g["mg_freq"], params)
    assert rel(gr, g["mg_cube_1_grid"]) <= 1e-12
    assert np.allclose(sw, g["mg_cube_1_sw"], rtol=1e-12)


@pytest.mark.parametrize("chan_mode", ["cube", "continuum"])
def test_tiled_mosaic_matches_per_sample_kernel(chan_mode):
    """The binned kernel against the one-warp-per-sample kernel on 16 time
    steps x 2016 baselines x 4 channels x 2 pols with the reference's
    functions (supports 5 and 7) and flagged / NaN / zero-weight samples."""
    import torch

    from astroviper_b200 import _kernels as K
    from astroviper_b200 import synthetic as S
    g = golden("mosaic.npz")
    uvw, rng = S.array_uvw(64, 16, radius_m=200.0, seed=7)
    uvw[3, 5, 1] = np.nan
    nb = uvw.shape[1]
    nchan, npol = 4, 2
    freq = np.linspace(1.0e9, 1.4e9, nchan)
    shape = (16, nb, nchan, npol)
    vis = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    wt = rng.uniform(0.5, 2.0, size=shape)
    wt[2, 7, :, 0] = 0.0
    wt[4, 9, 1, 1] = np.nan
    cfb = np.arange(nb) % 3
    cfc = np.array([0, 0, 1, 1])
    cm = np.arange(nchan) if chan_mode == "cube" else np.zeros(nchan, dtype=int)
    nic = nchan if chan_mode == "cube" else 1
    cf = K.cf_phase_product(torch.as_tensor(g["rk"], device="cuda"),
                            torch.as_tensor(g["mg_pg"][0], device="cuda"))
    n = 256
    out = []
    for tiled in (False, True):
        for do_psf in (False, True):
            grid = torch.zeros((nic, npol, n, n), dtype=torch.complex128, device="cuda")
            sw = torch.zeros((nic, npol), dtype=torch.float64, device="cuda")
            K.mosaic_grid(grid, sw, do_psf, torch.as_tensor(vis, device="cuda"),
                          torch.as_tensor(wt, device="cuda"), uvw, freq, cm, np.arange(npol),
                          cfb, cfc, np.zeros(npol, dtype=int), cf, g["support"], (n, n),
                          g["grid_cell"] * 0.3, g["gcf_oversampling"], tiled=tiled)
            out.append((grid.cpu().numpy(), sw.cpu().numpy()))
    for i in range(2):
        (ga, sa), (gb, sb) = out[i], out[i + 2]
        assert np.abs(ga).max() > 0
        assert rel(gb, ga) <= 1e-12, i
        assert np.allclose(sb, sa, rtol=1e-12), i


def _duck_ms(g, names_2d=False):
    """An MSv4-like dataset with the attributes the driver reads."""
    import types
    names = [str(x) for x in g["names"]]
    pairs = g["pairs"]

    class _Field:
        def isel(self, **kw):
            return types.SimpleNamespace(data=g["ra_dec"])

    return types.SimpleNamespace(
        data_vars=["VISIBILITY", "UVW", "WEIGHT", "FLAG"],
        attrs={"data_groups": {"base": {"correlated_data": "VISIBILITY", "uvw": "UVW",
                                        "weight": "WEIGHT", "flag": "FLAG"}}},
        xr_ms=types.SimpleNamespace(get_field_and_source_xds=lambda name: types.SimpleNamespace(
            FIELD_PHASE_CENTER_DIRECTION=_Field())),
        antenna_xds=types.SimpleNamespace(antenna_name=np.array(names)),
        baseline_antenna1_name=np.array([names[i] for i, _ in pairs]),
        baseline_antenna2_name=np.array([names[j] for _, j in pairs]),
        frequency=types.SimpleNamespace(values=g["freq"]),
        polarization=types.SimpleNamespace(values=g["pols"]))


def test_make_gridding_convolution_function_driver():
    """The driver (make_gridding_convolution_function.py:24-193) against the
    variables the reference's own driver built (tests/golden/gcf_driver.npz):
    maps and supports equal, kernels within cuFFT's rounding of numpy's FFT;
    PHASE_GRADIENT (the reference's needs astropy.wcs, absent) equal to
    make_phase_gradient's for the field centre.  A second call on the result
    keeps its kernels and remakes the phase gradient only."""
    import types
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    from astroviper_b200.core.imaging.dataset import Dataset
    g = golden("gcf_driver.npz")
    gcf_params = {"function": "casa_airy", "list_dish_diameters": [12.0, 25.0],
                  "list_blockage_diameters": [0.75, 0.0], "unique_ant_indx": [0, 1, 0, 1, 1, 0],
                  "oversampling": [4, 4], "max_support": [11, 11], "support_cut_level": 0.025,
                  "chan_tolerance_factor": 0.05,
                  "phase_direction": types.SimpleNamespace(values=np.array([0.3, -0.5]))}
    grid_params = {"image_size": [64, 64], "cell_size": [-1e-4, 1e-4], "fft_padding": 1.5,
                   "chan_mode": "cube"}
    before = repr(gcf_params), repr(grid_params)
    ds = G.make_gridding_convolution_function(Dataset(), _duck_ms(g), gcf_params, grid_params,
                                              {})
    assert (repr(gcf_params), repr(grid_params)) == before  # the caller's dicts untouched
    for name in ("SUPPORT", "CF_BASELINE_MAP", "CF_CHAN_MAP", "CF_POL_MAP", "PS_CORR_IMAGE"):
        assert np.array_equal(ds[name].values, g[f"var_{name}"]), name
        assert tuple(ds[name].dims) == tuple(str(x) for x in g[f"dims_{name}"]), name
    for name in ("CONV_KERNEL", "CONV_KERNEL_CONVOLVED"):
        assert tuple(ds[name].dims) == tuple(str(x) for x in g[f"dims_{name}"])
        a, b = ds[name].values, g[f"var_{name}"]
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b), name
    assert np.array_equal(ds.attrs["cell_uv"], g["attr_cell_uv"])
    assert np.array_equal(ds.attrs["oversampling"], g["attr_oversampling"])
    pg_params = {"phase_direction": gcf_params["phase_direction"],
                 "oversampling": np.array([4, 4]), "resize_conv_size": np.array([48, 48])}
    pg = G.make_phase_gradient(g["ra_dec"][None, :], pg_params,
                               {"image_size_padded": np.array([96, 96]),
                                "cell_size": np.array([-1e-4, 1e-4])})
    assert ds["PHASE_GRADIENT"].dims == ("field_id", "u", "v")
    assert np.array_equal(ds["PHASE_GRADIENT"].values, pg)
    # reuse: same number of baselines, kernels kept
    kept = ds["CONV_KERNEL"].values
    ds2 = G.make_gridding_convolution_function(ds, _duck_ms(g), gcf_params, grid_params, {})
    assert ds2 is ds and ds2["CONV_KERNEL"].values is kept
    with pytest.raises(AssertionError, match="gcf_params checking failed"):
        G.make_gridding_convolution_function(Dataset(), _duck_ms(g), dict(gcf_params,
                                             function="gauss"), grid_params, {})
