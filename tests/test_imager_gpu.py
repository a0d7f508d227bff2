"""The major/minor-cycle imager on the GPU: the polarisation products, the
argmax, the PSF sidelobe, the plane sums and the residual visibilities
against the reference's outputs (tests/golden/imager.npz) and numpy;
deconvolve against the oracle's Hogbom per plane; run_imaging_loop against
the oracle's restatement of the loop, bit-for-bit in its integer decisions
(iterations per cycle, stop codes) and within 1e-9 (FP64 mode) / 1e-4 (FP32
mode) in its images, with the reference's side effects on the measurement
set."""
import json
import os
import sys

import numpy as np
import pytest
import torch

import oracle as O
import oracle.imager as OI
from conftest import GOLDEN, golden

sys.path.insert(0, GOLDEN)
import imager_ops  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (nb if nb else 1.0)


def test_polarisation_products_match_reference_bitwise():
    from astroviper_b200.core.imaging.imaging_utils import corr_to_stokes as CS
    g = golden("imager.npz")
    kw = {"c1": dict(corr_type="linear", pol_axis=2),
          "c2": dict(corr_type="linear", pol_axis=2, stokes_out=["V", "I"]),
          "c3": dict(corr_type="circular", pol_axis=1),
          "c4": dict(corr_type="linear", pol_axis=1),
          "c5": dict(corr_type="circular", pol_axis=-3, stokes_out=["V"]),
          "c6": dict(corr_type="linear", pol_axis=1, stokes_out=["I"]),
          "c7": dict(corr_type="circular", pol_axis=2, stokes_out=["U", "Q", "V", "I"])}
    for k, a in kw.items():
        out = CS.image_corr_to_stokes(g[k + "_in"], **a)
        assert out.dtype == g[k + "_out"].dtype and np.array_equal(out, g[k + "_out"]), k
        dev = CS.image_corr_to_stokes(torch.as_tensor(g[k + "_in"], device="cuda"), **a)
        assert dev.is_cuda and np.array_equal(dev.cpu().numpy(), g[k + "_out"]), k
    kw = {"s1": dict(corr_type="linear", pol_axis=1), "s2": dict(corr_type="linear", pol_axis=1),
          "s3": dict(corr_type="linear", pol_axis=1), "s4": dict(corr_type="circular", pol_axis=1),
          "s5": dict(corr_type="linear", pol_axis=1, stokes_in=["I", "U"]),
          "s6": dict(corr_type="circular", pol_axis=1)}
    for k, a in kw.items():
        out = CS.image_stokes_to_corr(g[k + "_in"], **a)
        assert out.dtype == g[k + "_out"].dtype and np.array_equal(out, g[k + "_out"]), k
    assert np.array_equal(CS.corr_to_stokes(g["b_in"], "linear"), g["b1_out"])
    assert np.array_equal(CS.stokes_to_corr(g["b_in"], "circular"), g["b2_out"])
    # an arbitrary matrix: numpy's matmul may fuse or reorder; agree to rounding
    got = CS.corr_to_stokes(g["b_in"], "custom", transformation_matrix=g["b_custom"])
    assert np.allclose(got, g["b3_out"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_argmax_first_occurrence_and_nan(dtype):
    from astroviper_b200 import _kernels as K
    rng = np.random.default_rng(3)
    for n in (1, 7, 1000, 300001):
        x = rng.normal(size=n).astype(dtype)
        if n > 10:
            x[n // 3] = x[n // 2] = -50.0  # tie in |x|: first index wins
            x[n // 4] = 49.0
        for mode, ref in ((0, np.abs(x).argmax()), (1, x.argmax())):
            i, v = K.argmax(torch.as_tensor(x, device="cuda"), mode)
            assert i == ref and v == float(x[ref]), (n, mode)
    x = rng.normal(size=5000).astype(dtype)
    x[4000] = np.nan
    x[4500] = np.nan
    for mode in (0, 1):
        i, v = K.argmax(torch.as_tensor(x, device="cuda"), mode)
        assert i == 4000 and np.isnan(v)


def test_psf_sidelobe_matches_reference():
    from astroviper_b200 import _kernels as K
    g = golden("imager.npz")
    for i in range(int(g["n_psf"])):
        for dt in (np.float64, np.float32):
            p = g[f"psf{i}"].astype(dt)
            got = K.psf_sidelobe(torch.as_tensor(p, device="cuda"))
            want = OI.psf_max_sidelobe(p) if dt == np.float32 else float(g[f"psf{i}_sidelobe"])
            assert got == want, (i, dt)


def test_plane_sums_and_residual_visibilities():
    from astroviper_b200 import _kernels as K
    rng = np.random.default_rng(4)
    x = rng.normal(size=(3, 2, 129, 67))
    s = K.plane_sum(torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert s.shape == (3, 2) and np.allclose(s, x.sum(axis=(-2, -1)), rtol=1e-12, atol=1e-12)
    for dt in (np.complex64, np.complex128):
        a = (rng.normal(size=(5, 7, 3, 2)) + 1j * rng.normal(size=(5, 7, 3, 2))).astype(dt)
        b = (rng.normal(size=(5, 7, 3, 2)) + 1j * rng.normal(size=(5, 7, 3, 2))).astype(dt)
        r = K.vis_residual(torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda"))
        assert np.array_equal(r.cpu().numpy(), a - b)


def _small_sky(rng, ny=96, nx=96, npol=2):
    y, x = np.mgrid[0:ny, 0:nx]
    psf = np.exp(-0.5 * (((y - ny // 2) / 2.0) ** 2 + ((x - nx // 2) / 2.5) ** 2))
    psf += 0.15 * np.cos(np.hypot(y - ny // 2, x - nx // 2) / 2.0) * np.exp(
        -np.hypot(y - ny // 2, x - nx // 2) / 20.0)
    psf /= psf.max()
    dirty = np.zeros((1, 2, npol, ny, nx))
    for c in range(2):
        for p in range(npol):
            for _ in range(6):
                sy, sx = rng.integers(20, ny - 20), rng.integers(20, nx - 20)
                dirty[0, c, p] += rng.uniform(0.1, 1.0) * np.roll(
                    np.roll(psf, sy - ny // 2, 0), sx - nx // 2, 1)
            dirty[0, c, p] += rng.normal(0, 0.002, size=(ny, nx))
    return dirty, psf


def test_deconvolve_planes_match_oracle():
    from astroviper_b200.core.imaging.deconvolution import deconvolve
    from astroviper_b200.core.imaging.sky_image import make_sky_image
    rng = np.random.default_rng(5)
    dirty, psf = _small_sky(rng)
    d = make_sky_image((0.1, -0.5), (96, 96), (1e-5, 1e-5), [1.0e9, 1.1e9], ["I", "Q"], [5.0])
    d["RESIDUAL"] = dirty
    p = make_sky_image((0.1, -0.5), (96, 96), (1e-5, 1e-5), [1.0e9, 1.1e9], ["I"], [5.0])
    p["POINT_SPREAD_FUNCTION"] = np.broadcast_to(psf, (1, 2, 1, 96, 96)).copy()
    start = np.zeros_like(dirty)
    start[0, 1, 0, 40, 40] = 0.25
    m = make_sky_image((0.1, -0.5), (96, 96), (1e-5, 1e-5), [1.0e9, 1.1e9], ["I", "Q"], [5.0])
    m["MODEL"] = start
    params = {"gain": 0.1, "niter": 150, "threshold": 0.01}
    rd, model, resid = deconvolve(d, p, m, "hogbom", params)
    recs, omodel, oresid = OI.deconvolve_planes(dirty, p["POINT_SPREAD_FUNCTION"].values, 0.1, 150,
                                                0.01, start)
    assert np.array_equal(model["MODEL"].values, omodel)
    assert np.array_equal(resid["RESIDUAL"].values, oresid)
    assert "RESIDUAL" not in model and "MODEL" in model
    for r in recs:
        tt, pp, nn = r["key"]
        e = rd.sel(time=tt, pol=pp, chan=nn)
        assert e["iter_done"] == [r["iter_done"]]
        assert e["max_psf_sidelobe"] == r["max_psf_sidelobe"]
        assert e["start_peakres"] == [r["start_peakres"]] and e["peakres"] == [r["peakres"]]
        assert e["start_model_flux"] == [r["start_model_flux"]]
        assert abs(e["model_flux"][0] - r["model_flux"]) <= 1e-6 * abs(r["model_flux"])
        assert e["masksum"] == [96 * 96] and e["phase_center"] == "0.1,-0.5"
        assert e["niter"] == 150 and e["loop_gain"] == 0.1 and e["threshold"] == 0.01


class _Col:
    def __init__(self, v, dims=("time", "baseline_id", "frequency", "polarization")):
        self.values = v
        self.data = v
        self.dims = dims
        self.coords = {}

    def __len__(self):
        return len(self.values)


class ImagingMS4:
    """Duck-typed MSv4 node with the coordinates the imager reads."""

    def __init__(self, vis, uvw, weight, flag, freq, pols, phase_center=(0.0, 0.0)):
        self._d = {}
        for k, v in (("VISIBILITY", vis), ("UVW", uvw), ("WEIGHT", weight), ("FLAG", flag)):
            self[k] = _Col(v)
        self.frequency = _Col(freq, ("frequency",))
        self.coords = {"frequency": _Col(freq, ("frequency",)),
                       "polarization": _Col(np.asarray(pols), ("polarization",)),
                       "time": _Col(np.arange(vis.shape[0]) * 10.0, ("time",))}
        nt, nb, nc, npol = vis.shape
        self.dims = {"time": nt, "baseline_id": nb, "frequency": nc, "polarization": npol}
        self.attrs = {"phase_center": phase_center}

    def __getitem__(self, k):
        return self._d[k]

    def __setitem__(self, k, v):
        self._d[k] = v
        setattr(self, k, v)

    def __contains__(self, k):
        return k in self._d


_loop_inputs = imager_ops.loop_inputs
_params = imager_ops.loop_params


def _run_oracle(vis, uvw, weight, flag, freq, params, initial_model=None):
    from astroviper_b200.core.imaging.imaging_utils import iteration_control as IC
    from astroviper_b200.core.imaging.imaging_utils.return_dict import ReturnDict
    ctl = IC.IterationController(niter=params["niter"], nmajor=params["nmajor"],
                                 threshold=params["threshold"], gain=params["gain"],
                                 cyclefactor=params["cyclefactor"])
    return OI.run_imaging_loop(vis, uvw, weight, flag, freq, params, ctl, IC.merge_return_dicts,
                               ReturnDict, initial_model)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_imaging_loop_matches_oracle(precision):
    from astroviper_b200.core.imaging.imager import run_imaging_loop
    vis, uvw, weight, flag, freq, cell = _loop_inputs()
    params = _params(cell)
    ref = _run_oracle(vis.copy(), uvw.copy(), weight.copy(), flag.copy(), freq, params)
    ms = ImagingMS4(vis.copy(), uvw.copy(), weight.copy(), flag.copy(), freq, ["XX", "YY"])
    model, resid, combined, ctl = run_imaging_loop(ms, params, precision=precision)
    rctl = ref["controller"]
    assert model.shape == (2, 2, 128, 128) and model.dtype == np.float64
    assert ctl.major_done == rctl.major_done and ctl.stopcode == rctl.stopcode
    assert ctl.get_state() == rctl.get_state()
    assert ctl.major_done >= 2
    keys = list(combined.data.keys())
    assert keys == list(ref["combined"].data.keys())
    for k in keys:
        a, b = combined.data[k], ref["combined"].data[k]
        assert a["iter_done"] == b["iter_done"], k
        assert a["max_psf_sidelobe"] == pytest.approx(b["max_psf_sidelobe"], rel=1e-9)
    tol = 1e-9 if precision == "fp64" else 1e-4
    assert rel(model, ref["model"]) <= tol
    assert rel(resid, ref["residual"]) <= tol
    # side effects on the measurement set, as the reference leaves them
    assert np.array_equal(ms.FLAG.data, ref_flag := flag | _nan_rows(uvw))
    assert np.all(ms.UVW.data[5, 7] == 1e9)
    assert np.array_equal(ms.WEIGHT.data == 0, ref_flag | _nan_rows(uvw, uv_only=True))
    vm = ms["VISIBILITY_MODEL"].data
    assert vm.dtype == np.complex128 and rel(vm, ref["vis_model"]) <= (1e-9 if precision ==
                                                                        "fp64" else 1e-5)
    assert np.array_equal(ms["RESIDUAL"].data, vis - vm)


def _nan_rows(uvw, uv_only=False, nchan=2, npol=2):
    bad = np.isnan(uvw[:, :, :2] if uv_only else uvw).any(axis=-1)
    return np.broadcast_to(bad[:, :, None, None], bad.shape + (nchan, npol))


@pytest.mark.parametrize("case", ["linear4", "circular2", "initial_model_threshold"])
def test_imaging_loop_variants_match_oracle(case):
    """Four correlations (IQUV, complex model correlations in the predict),
    circular feeds (I, V), and a loop started from an initial model with a
    global threshold (the stop code, like everything else the controller
    decides, must be the oracle's); FP64 mode against the oracle's loop."""
    from astroviper_b200.core.imaging.imager import run_imaging_loop
    scale = {"linear4": (1.0, 0.1, 0.05, 0.8), "circular2": (1.0, 0.7),
             "initial_model_threshold": (1.0, 0.8)}[case]
    pols = {"linear4": ["XX", "XY", "YX", "YY"], "circular2": ["RR", "LL"],
            "initial_model_threshold": ["XX", "YY"]}[case]
    vis, uvw, weight, flag, freq, cell = _loop_inputs(n_time=12, pol_scale=scale)
    params = _params(cell)
    params.update(niter=120, nmajor=3)
    init = None
    if case == "circular2":
        params["corr_type"] = "circular"
    if case == "initial_model_threshold":
        params.update(threshold=0.05, nmajor=6, niter=2000)
        init = np.zeros((2, 2, 128, 128))
        init[0, 0, 60, 64] = 0.3
    ref = _run_oracle(vis.copy(), uvw.copy(), weight.copy(), flag.copy(), freq, params,
                      init)
    ms = ImagingMS4(vis.copy(), uvw.copy(), weight.copy(), flag.copy(), freq, pols)
    model, resid, combined, ctl = run_imaging_loop(ms, params, initial_model=init,
                                                   precision="fp64")
    rctl = ref["controller"]
    assert ctl.get_state() == rctl.get_state()
    assert model.shape == ref["model"].shape
    assert rel(model, ref["model"]) <= 1e-9 and rel(resid, ref["residual"]) <= 1e-9
    for k in combined.data:
        a, b = combined.data[k], ref["combined"].data[k]
        assert a["iter_done"] == b["iter_done"], k
        assert a["start_model_flux"] == pytest.approx(b["start_model_flux"], rel=1e-12,
                                                      abs=1e-12)
    if ref["vis_model"] is not None:
        assert rel(ms["VISIBILITY_MODEL"].data, ref["vis_model"]) <= 1e-9


def _close(a, b, tol):
    if isinstance(b, list):
        return isinstance(a, list) and len(a) == len(b) and all(
            _close(x, y, tol) for x, y in zip(a, b))
    if isinstance(b, float):
        return a == pytest.approx(b, rel=tol, abs=tol)
    return a == b


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", imager_ops.LOOP_CASES)
def test_imaging_loop_decisions_match_reference_controller(case, precision):
    """imager_loop.json holds what the reference's own IterationController,
    merge_return_dicts and ReturnDict decided when they drove the oracle's
    loop on the same inputs: this package's loop (its controller, on the
    GPU's peaks and sidelobes) ends in the same controller state, with the
    same iterations per plane and cycle, and the peaks, fluxes and sidelobes
    the controller read agree to the precision mode's tolerance."""
    from astroviper_b200.core.imaging.imager import run_imaging_loop
    with open(os.path.join(GOLDEN, "imager_loop.json")) as f:
        fix = json.load(f)[case]
    vis, uvw, weight, flag, freq, pols, params, init = imager_ops.loop_case(case)
    ms = ImagingMS4(vis, uvw, weight, flag, freq, pols)
    _model, _resid, combined, ctl = run_imaging_loop(ms, params, initial_model=init,
                                                     precision=precision)
    assert imager_ops._py(ctl.get_state()) == fix["state"]
    got = imager_ops._dump(combined)
    assert [k for k, _ in got] == [k for k, _ in fix["combined"]]
    # CLEAN runs in FP32 in both loops (as the reference's deconvolve selects
    # it), so peaks and fluxes carry FP32 rounding even in the FP64 mode
    tol = 1e-6 if precision == "fp64" else 2e-5
    for (key, a), (_, b) in zip(got, fix["combined"]):
        assert a["iter_done"] == b["iter_done"], key
        assert a["niter"] == b["niter"] == fix["cycles"][-1]["niter"], key
        # the fields the oracle loop records (the package's loop records the
        # reference deconvolve's others besides)
        assert set(b) <= set(a), key
        for field in b:
            assert _close(a[field], b[field], tol), (key, field, a[field], b[field])


def test_imaging_loop_drop_in_steps():
    """grid_visibilities, predict_model_visibilities and
    compute_residual_visibilities against the oracle."""
    from astroviper_b200.core.imaging import imager
    vis, uvw, weight, flag, freq, cell = _loop_inputs(n_time=8)
    ms = ImagingMS4(vis.copy(), uvw.copy(), weight.copy(), flag.copy(), freq, ["XX", "YY"])
    cs = (abs(cell[0]), abs(cell[1]))
    d = imager.grid_visibilities(ms, (128, 128), cs, precision="fp64")
    w = weight.copy()
    w[flag] = 0
    w[np.isnan(uvw[:, :, 0]) | np.isnan(uvw[:, :, 1])] = 0
    cgk = O.create_prolate_spheroidal_kernel_1D(100, 7)
    g, sw = O.standard_grid(vis, uvw, w, freq, cgk, (128, 128), cs, chan_mode="cube")
    assert rel(d, O.grid_to_image(g, sw)) <= 1e-12
    model = np.zeros((2, 2, 128, 128))
    model[:, :, 60, 70] = 0.5
    imager.predict_model_visibilities(ms, model, cs, precision="fp64")
    fl = flag | _nan_rows(uvw)
    u2 = uvw.copy()
    u2[np.isnan(u2).any(axis=-1)] = 1e9
    want = O.degrid(O.fft_lm_to_uv(model, axes=[2, 3]), u2, freq, cs, flag=fl)
    assert rel(ms["VISIBILITY_MODEL"].data, want) <= 1e-12
    imager.compute_residual_visibilities(ms)
    assert np.array_equal(ms["RESIDUAL"].data, ms["VISIBILITY"].data - ms["VISIBILITY_MODEL"].data)
