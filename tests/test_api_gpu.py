"""The numpy/xarray drop-in API (astroviper_b200.core...) on the GPU, against
the reference's golden outputs, its own known-answer tests and, for CLEAN
callbacks, the reference's compiled Hogbom module (oracle/_ref)."""
import glob
import importlib.util
import os

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (nb if nb else 1.0)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
@pytest.mark.parametrize("case", ["a", "b", "c"])
def test_standard_grid_wrappers(precision, tol, case):
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG
    g = golden(f"grid_{case}.npz")
    sup, os_ = int(g["support"]), int(g["oversampling"])
    for do_psf in (False, True):
        for mode in ("continuum", "cube"):
            key = f"{'psf' if do_psf else 'vis'}_{mode}"
            gr, sw = SG.standard_grid_numpy_wrap_input_checked(
                g["vis"], np.array([]), np.array([]), g["uvw"], g["weight"], g["freq"], g["cgk"],
                g["image_size"], g["cell"], os_, sup, True, do_psf, mode, precision=precision)
            assert gr.dtype == np.complex128 and gr.shape == g["grid_" + key].shape
            assert rel(gr, g["grid_" + key]) <= tol, key
            assert np.allclose(sw, g["sumwt_" + key], rtol=1e-7)
    # accumulate into given arrays, in place
    gr = g["acc_grid0"].copy()
    sw = g["acc_sumwt0"].copy()
    out = SG.standard_grid_numpy_wrap_input_checked(
        g["vis"], gr, sw, g["uvw"], g["weight"], g["freq"], g["cgk"], g["image_size"], g["cell"],
        os_, sup, True, False, "continuum", precision=precision)
    assert out[0] is gr and out[1] is sw
    assert rel(gr, g["acc_grid"]) <= tol and np.allclose(sw, g["acc_sumwt"], rtol=1e-7)


class _Coord:
    def __init__(self, v):
        self.values = v
        self.data = v
        self.dims = ("time", "baseline_id", "frequency", "polarization")
        self.coords = {}


class MS4:
    """Duck-typed MSv4 node (UVW, WEIGHT, FLAG, VISIBILITY, frequency)."""

    def __init__(self, vis, uvw, weight, flag, freq):
        self._d = {}
        for k, v in (("VISIBILITY", vis), ("UVW", uvw), ("WEIGHT", weight), ("FLAG", flag)):
            self[k] = _Coord(v)
        self.frequency = _Coord(freq)
        self.coords = {"frequency": _Coord(freq)}
        nt, nb, nc, npol = vis.shape
        self.dims = {"time": nt, "baseline_id": nb, "frequency": nc, "polarization": npol}

    def __getitem__(self, k):
        return self._d[k]

    def __setitem__(self, k, v):
        self._d[k] = v
        setattr(self, k, v)

    def __contains__(self, k):
        return k in self._d


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_grid2image_spheroid_ms4(precision, tol):
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG
    g = golden("image.npz")
    for dopsf in (False, True):
        for mode, nci in (("continuum", 1), ("cube", 2)):
            tag = f"{'psf' if dopsf else 'vis'}_{mode}"
            w = g["weight"].copy()
            ms = MS4(g["vis"].copy(), g["uvw"].copy(), w, g["flag"].copy(), g["freq"])
            img = np.zeros((nci, 2, 64, 64))
            SG.grid2image_spheroid_ms4(ms, img, g["cell"], 7, 100, dopsf, "VISIBILITY", mode,
                                       precision=precision)
            assert rel(img, g["img_" + tag]) <= tol, tag
            # the caller's WEIGHT is zeroed where flagged / NaN uvw, as the reference does
            assert np.array_equal(w, g["weight_after_" + tag])
    with pytest.raises(TypeError):
        SG.grid2image_spheroid_ms4([object()], np.zeros((1, 2, 64, 64)), g["cell"])
    ms = MS4(g["vis"].copy(), g["uvw"].copy(), g["weight"].copy(), g["flag"].copy(), g["freq"])
    with pytest.raises(RuntimeError, match="Shapes of gridded vis and image do no match"):
        SG.grid2image_spheroid_ms4(ms, np.zeros((3, 2, 64, 64)), g["cell"])


@pytest.mark.parametrize("mode", ["cube", "continuum"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), (None, 1e-6)])
def test_make_psf_dropin(mode, precision, tol):
    """make_psf (make_point_spread_function.py:1-79): the planes the reference
    computes (grid2image_spheroid_ms4 with dopsf and pixelincr [-cell0, cell1]
    into an (n_freq, n_pol, image_size[1], image_size[0]) array; non-square
    sizes show the transpose), as the POINT_SPREAD_FUNCTION of a sky image
    over the visibilities' frequencies, polarisations and first time."""
    from astroviper_b200 import synthetic as S
    from astroviper_b200.core.imaging.imaging_utils.make_point_spread_function import make_psf
    g = golden("psf_dropin.npz")
    nch = 2 if mode == "cube" else 1
    node = S.Ms4Node(g["vis"][:, :, :nch].copy(), g["uvw"].copy(),
                     g["weight"][:, :, :nch].copy(), g["flag"][:, :, :nch].copy(),
                     g["freq"][:nch], ["XX", "YY"])
    size = tuple(int(n) for n in g[f"image_size_{mode}"])
    img = make_psf(node, {"image_size": size, "cell_size": g["cell"], "phase_center": (0.3, -0.5),
                          "chan_mode": mode}, {"sampling": 100, "support": 7},
                   precision=precision)
    psf = img["POINT_SPREAD_FUNCTION"]
    ref = g[f"psf_{mode}"]
    assert psf.dims == ("time", "frequency", "polarization", "l", "m")
    assert psf.values.shape == (1, nch, 2, size[1], size[0]) == (1,) + ref.shape
    assert rel(psf.values[0], ref) <= tol
    assert np.array_equal(node["WEIGHT"].data, g[f"weight_after_{mode}"])
    assert np.array_equal(img.coords["frequency"].values, g["freq"][:nch])
    assert list(img.coords["polarization"].values) == ["XX", "YY"]
    assert img.coords["time"].values[0] == node.coords["time"].values[0]
    assert img.attrs["phase_center"] == (0.3, -0.5)


def test_reference_lattice_known_answer_on_gpu():
    """test_standard_grid.py:14-111 of the reference through the drop-in API."""
    from astroviper_b200.core.imaging.fft import fft_lm_to_uv
    from astroviper_b200.core.imaging.ifft import ifft_uv_to_lm
    from astroviper_b200.core.imaging.imaging_utils import gcf_prolate_spheroidal as GCF
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG
    n = 200
    c = 299792458.0
    freq = np.array([1.4e9])
    maxuv = 2e3
    cell = 0.5 * c / freq[0] / maxuv
    mod = np.zeros((n, n))
    mod[np.array([110, 87]), np.array([115, 92])] = np.array([1.0, 2.0])
    ft = np.conj(fft_lm_to_uv(mod, axes=[0, 1]))
    ax = np.linspace(-maxuv, maxuv, n)
    uu, vv = np.meshgrid(ax, ax, indexing="ij")
    uvw = np.stack([uu.ravel(), vv.ravel(), np.zeros(n * n)], -1)[None]
    vis = ft.reshape(1, n * n, 1, 1).astype(np.complex128)
    w = np.ones(vis.shape)
    cgk = GCF.create_prolate_spheroidal_kernel_1D(100, 7)
    _, ct = GCF.create_prolate_spheroidal_kernel(100, 7, np.array([n, n]))
    for do_psf in (False, True):
        gr, sw = SG.standard_grid_numpy_wrap_input_checked(
            vis, np.array([]), np.array([]), uvw, w, freq, cgk, np.array([n, n]),
            np.array([cell, cell]), 100, 7, True, do_psf, "continuum")
        img = ifft_uv_to_lm(gr, axes=[2, 3]) / ct * n * n / sw[..., None, None]
        if do_psf:
            assert abs(img[0, 0, 100, 100] - 1.0) < 0.01
        else:
            assert img[0, 0, 87, 92] > 1.8 and img[0, 0, 110, 115] > 0.9


def test_fft_helpers_round_trip_known_answer():
    """test_fft_ifft.py:12-26 of the reference (round trip < 1e-10)."""
    from astroviper_b200.core.imaging.fft import fft_lm_to_uv
    from astroviper_b200.core.imaging.ifft import ifft_uv_to_lm
    sky = np.zeros((128, 128))
    sky[64, 64] = 1
    sky[50, 40] = 1
    rt = ifft_uv_to_lm(fft_lm_to_uv(sky, (0, 1)), (0, 1))
    assert np.max(np.abs(sky - rt)) < 1e-10
    g = golden("image.npz")
    assert rel(fft_lm_to_uv(g["fft_in"], axes=[2, 3]), g["fft_out"]) < 1e-13
    assert rel(ifft_uv_to_lm(g["fft_out"], axes=[2, 3]), g["ifft_out"]) < 1e-13
    # other axes than the last two
    a = np.moveaxis(g["fft_in"], [2, 3], [0, 1]).copy()
    assert rel(fft_lm_to_uv(a, axes=[0, 1]), np.moveaxis(g["fft_out"], [2, 3], [0, 1])) < 1e-13


@pytest.mark.parametrize("precision,tol", [("fp64", 0.0), ("fp32", 1e-6)])
def test_dgrid_numba_dropin(precision, tol):
    from astroviper_b200.core.imaging.imaging_utils import standard_degrid as SD
    g = golden("degrid.npz")
    nt, nb = g["uvw"].shape[:2]
    for sup, os_ in ((7, 100), (9, 64), (8, 100)):
        cf = O.create_prolate_spheroidal_kernel_1D(os_, sup)
        v = g[f"v0_{sup}_{os_}_zero"].copy()
        SD.dgrid_numba(g["uvw"], np.zeros((nt, nb)), v, g["flag"], g["scale"], g["offset"],
                       g["grid"], g["freq"], 299792458.0, sup, os_, cf, g["chanmap"], g["polmap"],
                       precision=precision)
        ref = g[f"v_{sup}_{os_}_zero"]
        if tol == 0.0:
            assert np.array_equal(v, ref)
        else:
            assert rel(v - g[f"v0_{sup}_{os_}_zero"], ref - g[f"v0_{sup}_{os_}_zero"]) <= tol


def test_degrid_spheroid_ms4_store_mode():
    """A fresh VISIBILITY_MODEL: flagged and off-grid samples are 0, the rest
    the model; NaN-uvw rows get flagged and uvw 1e9 in the caller's arrays."""
    from astroviper_b200.core.imaging.imaging_utils import standard_degrid as SD
    from astroviper_b200 import synthetic as S
    uvw, rng = S.array_uvw(10, 6, radius_m=800.0, seed=5)
    uvw[:, -1, :2] *= 30.0
    uvw[2, 3, 0] = np.nan
    nt, nb = uvw.shape[:2]
    freq = np.array([1.1e9, 1.3e9])
    grid = rng.normal(size=(1, 2, 64, 64)) + 1j * rng.normal(size=(1, 2, 64, 64))
    cell = np.array([-20.0, 20.0]) * np.pi / (180 * 3600)
    flag = rng.uniform(size=(nt, nb, 2, 2)) < 0.2
    vis = np.zeros((nt, nb, 2, 2), complex)
    ms = MS4(vis, uvw.copy(), np.ones(vis.shape), flag.copy(), freq)
    SD.degrid_spheroid_ms4(ms, grid, cell)
    got = ms.VISIBILITY_MODEL.data
    flag2 = flag.copy()
    flag2[2, 3] = True
    uvw2 = uvw.copy()
    uvw2[2, 3] = 1e9
    ref = O.degrid(grid, uvw2, freq, cell, flag=flag2)
    assert np.all(got[flag2] == 0)
    assert rel(got, ref) <= 1e-6
    assert ms.FLAG.data[2, 3].all() and np.all(ms.UVW.data[2, 3] == 1e9)
    # incremental: adds to the existing model
    SD.degrid_spheroid_ms4(ms, grid, cell, incremental=True)
    assert rel(ms.VISIBILITY_MODEL.data, 2 * ref) <= 1e-6


def test_gridder_store_and_accumulate_agree():
    import torch
    from astroviper_b200.gridder import Gridder
    from astroviper_b200 import synthetic as S
    W = S.workload_small(n_time=6)
    G = Gridder(W["uvw"], W["freq"], (256, 256), W["pixelincr"], 2)
    gr, sw = G.grid(W["vis"], W["weight"])
    a = G.degrid(gr)
    b = torch.full_like(a, 3 + 4j)
    G.degrid(gr, values=b, accumulate=True)
    assert torch.allclose(b - (3 + 4j), a, rtol=1e-6, atol=1e-6)


def test_weights_dropin_against_golden():
    from astroviper_b200.core.imaging.imaging_weighting import briggs_weighting as BW
    from astroviper_b200.core.imaging.imaging_weighting import grid_imaging_weights as GIW
    g = golden("weights.npz")
    for npol in (1, 2, 4):
        q = lambda k: g[f"p{npol}_{k}"]
        G = np.zeros((2, 1) + tuple(int(x) for x in q("n")))
        sw = np.zeros((2, 1))
        GIW.grid_imaging_weights(G, sw, q("uvw"), q("wd"), q("freq"),
                                 {"image_size": q("n"), "cell_size": q("cell")})
        assert rel(G, q("G")) <= 1e-13 and np.allclose(sw, q("sw"), rtol=1e-13)
        for robust in (-1.0, 0.5, 2.0):
            bf = BW.calculate_briggs_params(G, sw, {"weighting": "briggs", "robust": robust})
            assert np.allclose(bf, q(f"bf_{robust}"), rtol=1e-12)
            iw = GIW.degrid_imaging_weights(G, q("uvw"), q("wd"), bf, q("freq"),
                                            {"image_size": q("n"), "cell_size": q("cell")})
            assert np.allclose(np.tile(iw, (1, 1, 1, npol)), q(f"iw_{robust}"), rtol=1e-12,
                               equal_nan=True)
        assert np.array_equal(BW.calculate_briggs_params(
            G, sw, {"weighting": "briggs_abs", "robust": 0.7, "briggs_abs_noise": 0.3}),
            q("bf_abs"))


def test_imaging_weight_degrid_dropin_against_golden():
    """standard_imaging_weight_degrid_numpy_wrap / _jit (standard_grid.py:441-604)
    on the GPU: bit-exact to the reference's outputs for numpy and torch
    inputs, float64 and float32 grids, permuted maps into a prefilled array
    (entries of samples off the grid untouched); maps outside the grid raise."""
    import torch
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG
    g = golden("iw_degrid.npz")
    for npol in (1, 2, 4):
        q = lambda k: g[f"p{npol}_{k}"]
        params = {"image_size_padded": q("n"), "cell_size": q("cell")}
        iw = SG.standard_imaging_weight_degrid_numpy_wrap(q("G"), q("uvw"), q("nat"), q("bf"),
                                                          q("freq"), params)
        assert isinstance(iw, np.ndarray) and iw.dtype == np.float64
        assert np.array_equal(iw, q("iw"), equal_nan=True)
        iw32 = SG.standard_imaging_weight_degrid_numpy_wrap(q("G").astype(np.float32), q("uvw"),
                                                            q("nat"), q("bf"), q("freq"), params)
        assert np.array_equal(iw32, q("iw32"), equal_nan=True)
        t = SG.standard_imaging_weight_degrid_numpy_wrap(
            torch.as_tensor(q("G"), device="cuda"), q("uvw"),
            torch.as_tensor(q("nat").astype(np.float32), device="cuda"), q("bf"), q("freq"),
            params)
        nat32 = q("nat").astype(np.float32).astype(np.float64)
        ref32 = O.standard_imaging_weight_degrid_numpy_wrap(q("G"), q("uvw"), nat32, q("bf"),
                                                            q("freq"), params)
        assert t.is_cuda and np.array_equal(t.cpu().numpy(), ref32, equal_nan=True)
        jit = np.full(q("nat").shape, -7.0)
        SG.standard_imaging_weight_degrid_jit(jit, q("G"), q("bf"), q("uvw"), q("freq"), q("cm"),
                                              q("pm"), q("nat"), q("n"), q("cell"))
        assert np.array_equal(jit, q("jit"), equal_nan=True)
        with pytest.raises(ValueError):
            SG.standard_imaging_weight_degrid_jit(jit, q("G"), q("bf"), q("uvw"), q("freq"),
                                                  q("cm") + 1, q("pm"), q("nat"), q("n"),
                                                  q("cell"))


def test_calculate_imaging_weights_processing_set():
    from astroviper_b200.core.imaging.calculate_imaging_weights import calculate_imaging_weights
    g = golden("weights.npz")
    for npol in (2, 4):
        q = lambda k: g[f"p{npol}_{k}"]
        w = q("w").copy()
        node = MS4(np.zeros(w.shape, complex), q("uvw"), w, q("flag").copy(), q("freq"))
        node.data_groups = {}
        ps = {"ms0": node}
        out, grp, dens = calculate_imaging_weights(
            ps, {"image_size": q("n"), "cell_size": q("cell")},
            {"weighting": "briggs", "robust": 0.5}, {}, return_weight_density_grid=True)
        assert rel(dens, q("G")) <= 1e-13
        got = node["WEIGHT_IMAGING"]
        got = getattr(got, "values", got)
        assert np.allclose(got, q("iw_0.5"), rtol=1e-12, equal_nan=True)
        assert np.all(np.isnan(w[q("flag")]))  # flagged weights NaN'd in place
        assert grp["data_group_out_name"] == "imaging"


def _ref_hogbom():
    so = glob.glob(os.path.join(ROOT, "oracle", "_ref", "_hogbom_ext*.so"))
    if not so:
        pytest.skip("reference Hogbom module not built")
    spec = importlib.util.spec_from_file_location("_hogbom_ext", so[0])
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_hogbom_clean_dropin_with_callbacks(dt):
    """Callback sequence (iteration, px, py, peak) and stop semantics equal the
    reference module's; results bit-exact."""
    from astroviper_b200.core.imaging.deconvolvers import hogbom
    H = _ref_hogbom()
    g = golden("hogbom.npz")
    d = g["dirty"].astype(dt)
    p = g["psf"].astype(dt)
    for kw in (dict(max_iter=137, gain=0.1), dict(max_iter=60, start_iter=7, gain=0.3),
               dict(max_iter=500, gain=0.2, threshold=0.05)):
        seq_ref, seq = [], []
        r = H.clean(d, p, progress_callback=lambda *a: seq_ref.append(a), **kw)
        o = hogbom.clean(d, p, progress_callback=lambda *a: seq.append(a), **kw)
        assert seq == seq_ref
        assert o["iterations_performed"] == r["iterations_performed"]
        assert np.array_equal(o["model_image"], r["model_image"])
        assert np.array_equal(o["residual_image"], r["residual_image"])
        assert o["final_peak"] == r["final_peak"]
        assert o["total_flux_cleaned"] == r["total_flux_cleaned"]
        assert o["converged"] == r["converged"]
    # stop_callback ends the run at the first callback point that returns True
    calls = {"n": 0}

    def stop():
        calls["n"] += 1
        return calls["n"] >= 3
    r = H.clean(d, p, max_iter=300, stop_callback=stop)
    calls["n"] = 0
    o = hogbom.clean(d, p, max_iter=300, stop_callback=stop)
    assert o["iterations_performed"] == r["iterations_performed"]
    assert np.array_equal(o["model_image"], r["model_image"])


def test_hogbom_clean_stats_and_maximg():
    from astroviper_b200.core.imaging import deconvolution as D
    from astroviper_b200.core.imaging.deconvolvers import hogbom
    g = golden("hogbom.npz")
    for tag, dt in (("f32", np.float32), ("f64", np.float64)):
        assert np.array_equal(np.array(hogbom.maximg(g["dirty"].astype(dt))), g[f"{tag}_maximg"])
        assert np.array_equal(np.array(hogbom.maximg(g["dirty"].astype(dt), g["mask"].astype(dt))),
                              g[f"{tag}_maximg_mask"])
        r = hogbom.clean(g["dirty"].astype(dt), g["psf"].astype(dt), max_iter=1000, gain=0.05)
        assert r["model_image"].dtype == dt
        assert r["total_flux_cleaned"] == float(g[f"{tag}_long_total_flux_cleaned"])
        assert r["final_peak"] == float(g[f"{tag}_long_final_peak"])
        assert r["converged"] == bool(g[f"{tag}_long_converged"])
    # hogbom_clean passes an empty float32 mask: the FP32 overload, as the reference
    stats, model, resid = D.hogbom_clean(g["dirty"].astype(np.float64),
                                         g["psf"].astype(np.float64), {"niter": 100})
    assert model.dtype == np.float32
    assert stats["iterations_performed"] == 100
    assert np.array_equal(model, g["f32_default_model_image"])
    assert np.array_equal(resid, g["f32_default_residual_image"])


def test_hogbom_large_psf_matches_restatement():
    """A PSF twice the image size (centre at its middle): the restated loop
    (reference hclean.cpp:124-200 with the PSF's own size) is matched exactly."""
    from astroviper_b200.core.imaging.deconvolvers import hogbom
    g = golden("hogbom.npz")
    d = g["dirty"]
    p2 = g["psf2"]
    o = hogbom.clean(d, p2, max_iter=400, gain=0.1, large_psf=True)
    r = O.hogbom_clean(d, p2, max_iter=400, gain=0.1)
    assert o["iterations_performed"] == r["iterations_performed"]
    assert np.array_equal(o["model_image"], r["model_image"])
    assert np.array_equal(o["residual_image"], r["residual_image"])
