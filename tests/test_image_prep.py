"""remove_padding / apply_pb / fft_to_uv / ifft_to_lm / correct_fft_to_uv /
correct_ifft_to_lm (standard_image_grid_preparation.py:99-492).

CPU: the oracle's restatement of the two normalisations and of apply_pb's
_mult_div against the reference's outputs in tests/golden/image_prep.npz
(bit-exact, NaN positions compared as positions); remove_padding on a
SkyImage against the reference's crops.  GPU: the drop-in functions on SkyImage datasets
against the same outputs: the normalisations and apply_pb bit-exact where the reference's
inputs are used as they are (with the spheroid correction, to 1e-13
relative, since the device's grid-correction term is within 1e-14 of the
reference's; the rescale itself bit-exact against the oracle given the same
term); the transforms to 1e-12 of each plane's peak (cuFFT against numpy's
pocketfft); grid2xradio_spheroid_ms4's grids to 1e-12 of the peak with the
FP64 kernels and 1e-6 with the FP32 tiled ones.
"""
import numpy as np
import pytest

import oracle as O
import oracle.imager as OI
from conftest import golden

UV_DIMS = ("time", "frequency", "polarization", "u", "v")


def same_bits(a, b):
    """Equal values bit for bit (signs of zeros included); NaNs compared by
    position, since NaN payloads are not specified by either side."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if np.iscomplexobj(a):
        return same_bits(a.real.copy(), b.real.copy()) and same_bits(a.imag.copy(), b.imag.copy())
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    return np.array_equal(a[~na].view(u), b[~nb].view(u))


def _cases(g, prefix):
    names = sorted({k.split("/")[0] for k in g.files if k.split("/")[0].startswith(prefix)})
    return names


def _vars(g, case, which):
    return {k.split("/")[1]: g[k] for k in g.files
            if k.startswith(case + "/") and k.endswith("/" + which)}


# ----------------------------------------------------------------- CPU ---
def test_oracle_correct_fft_to_uv_matches_reference():
    g = golden("image_prep.npz")
    cases = _cases(g, "cfu_")
    assert len(cases) == 4
    for case in cases:
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        named = "named" in case
        for n, x in ins.items():
            y = x.copy()
            if named or n in ("VISIBILITY", "VISIBILITY_RESIDUAL", "VISIBILITY_MODEL"):
                with np.errstate(all="ignore"):
                    OI.correct_fft_to_uv_planes(y, x.shape[3], x.shape[4])
            assert same_bits(y, outs[n]), (case, n)


def test_oracle_correct_ifft_to_lm_matches_reference():
    g = golden("image_prep.npz")
    for case in ("cil_f64", "cil_f32", "cil_c64"):
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        for n, x in ins.items():
            y = x.copy()
            if n in ("SKY", "RESIDUAL"):
                with np.errstate(all="ignore"):
                    OI.correct_ifft_to_lm_planes(y, x.shape[3], x.shape[4])
            assert same_bits(y, outs[n]), (case, n)
    ins, outs = _vars(g, "cil_sph", "in"), _vars(g, "cil_sph", "out")
    nx, ny = ins["SKY"].shape[3:]
    corr = O.corr_term((nx, ny))
    for n, norm in (("SKY", "VISIBILITY_NORMALIZATION"),
                    ("RESIDUAL", "VISIBILITY_RESIDUAL_NORMALIZATION")):
        y = ins[n].copy()
        OI.correct_ifft_to_lm_planes(y, nx, ny, corr, ins[norm])
        assert same_bits(y, outs[n]), n
    ins, outs = _vars(g, "cil_sph_named", "in"), _vars(g, "cil_sph_named", "out")
    y = ins["RESIDUAL"].copy()
    OI.correct_ifft_to_lm_planes(y, 20, 20, g["cil_sph_named/corr"],
                                 ins["VISIBILITY_RESIDUAL_NORMALIZATION"])
    assert same_bits(y, outs["RESIDUAL"])


def test_oracle_transforms_match_reference():
    g = golden("image_prep.npz")
    for n in ("SKY", "MODEL"):
        ref = g[f"fft/VISIBILITY_{n}/out"]
        assert np.array_equal(O.fft_lm_to_uv(g[f"fft/{n}/in"], axes=[3, 4]), ref)
    for n, dst in (("VISIBILITY", "SKY"), ("VISIBILITY_RESIDUAL", "RESIDUAL")):
        assert np.array_equal(O.ifft_uv_to_lm(g[f"ifft/{n}/in"], axes=[3, 4]),
                              g[f"ifft/{dst}/out"])


def _pb_cases(g):
    return sorted({k.split("/")[0] for k in g.files
                   if k.startswith("pb_") and k.endswith("/PRIMARY_BEAM/in")})


def test_oracle_apply_pb_matches_reference():
    g = golden("image_prep.npz")
    cases = _pb_cases(g)
    assert len(cases) == 17
    for case in cases:
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        multiply = case.endswith("_mul")
        for n, x in ins.items():
            if n == "PRIMARY_BEAM":
                continue
            y = x.copy()
            with np.errstate(all="ignore"):
                OI.mult_div_planes(y, ins["PRIMARY_BEAM"], multiply)
            assert same_bits(y, outs[n]), (case, n)


def test_remove_padding_matches_reference():
    from astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation import (
        remove_padding)
    from astroviper_b200.core.imaging.sky_image import SkyImage
    g = golden("image_prep.npz")
    for tag in ("even", "odd"):
        x = g[f"pad_{tag}/SKY/in"]
        img = SkyImage({"SKY": x.copy()}, coords={"l": np.arange(x.shape[3]),
                                                  "m": np.arange(x.shape[4])})
        out = remove_padding(img, g[f"pad_{tag}/size"])
        assert np.array_equal(out["SKY"].data, g[f"pad_{tag}/SKY/out"])
        assert out.sizes["l"] == out.coords["l"].values.size


def _ms4_nodes(g, tag):
    return [tuple(g[f"ms4_{tag}/node{k}/{n}"].copy() for n in ("vis", "uvw", "weight", "flag"))
            + (g[f"ms4_{tag}/freq"],) for k in range(2)]


# the cell of the grid2xradio_spheroid_ms4 fixtures: the spacing of their l / m coordinates
MS4_CELL = np.array([2.0e-5, 2.4e-5])


def test_oracle_grid2xradio_spheroid_ms4_matches_reference():
    g = golden("image_prep.npz")
    for tag, psf, mode in (("vis", False, "continuum"), ("psf", True, "cube")):
        ref = g[f"ms4_{tag}/grid"]
        grid = np.zeros(ref.shape, complex)
        sumwt = np.zeros(ref.shape[:3])
        nodes = _ms4_nodes(g, tag)
        OI.grid_ms4_into_image(nodes, grid, sumwt, MS4_CELL, do_psf=psf,
                               chan_mode=mode)
        assert np.max(np.abs(grid - ref)) <= 1e-12 * np.max(np.abs(ref)), tag
        assert np.allclose(sumwt, g[f"ms4_{tag}/sumwt"], rtol=1e-13, atol=0), tag
        for k, node in enumerate(nodes):
            assert np.array_equal(node[2], g[f"ms4_{tag}/node{k}/weight_after"])


def _ref_test_image(npol=1, nchan=1, which="SKY", fill=1.0):
    """The image of the reference's own tests of this module
    (test_standard_image_grid_preparation.py:17-65): 200 x 200 pixels of
    4.8e-6 rad, frequencies 1e9 + k 1e8, pols from RR LL LR RL, one epoch,
    the variable `which` float32 ones."""
    from astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation import (
        make_image_xds)
    freq = np.arange(1, nchan + 1) * 1e8 + 1e9
    pol = np.array(["RR", "LL", "LR", "RL"])[:npol]
    a = make_image_xds([200, 200], [4.8e-6, 4.8e-6], freq, None, [1.0, 0.0], which=which,
                       pol=pol, time=[5.7e4])
    a[which].data[...] = fill
    return a


def test_make_image_xds_layout():
    from astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation import (
        make_image_xds)
    a = make_image_xds([30, 20], [1e-5, 2e-5], 1.4e9, 1e6, [0.5, -0.3], which="MODEL")
    assert a.sizes == {"time": 1, "frequency": 1, "polarization": 1, "l": 30, "m": 20}
    assert a["MODEL"].data.dtype == np.float32 and not a["MODEL"].data.any()
    assert list(a.coords["polarization"].values) == ["I"]
    assert list(a.coords["time"].values) == [0.0]
    assert a.coords["frequency"].attrs["channel_width"] == {"data": 1e6, "units": "Hz"}
    assert np.isclose(abs(a.coords["l"].values[1] - a.coords["l"].values[0]), 1e-5)
    assert np.isclose(abs(a.coords["m"].values[1] - a.coords["m"].values[0]), 2e-5)
    b = make_image_xds([8, 8], [1e-5, 1e-5], [1e9, 2e9], None, [0, 0],
                       pol=["XX", "YY"], time=[1.0, 2.0, 3.0])
    assert b["SKY"].shape == (3, 2, 2, 8, 8)
    assert "channel_width" not in b.coords["frequency"].attrs


def test_make_empty_padded_uv_image_as_reference_test():
    """test_standard_image_grid_preparation.py:82-95, plus the copy of the
    residual into the centre and the size check."""
    from astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation import (
        make_empty_padded_uv_image)
    a = _ref_test_image(which="RESIDUAL")
    a["RESIDUAL"].data[0, 0, 0, 3, 5] = 7.0
    b = make_empty_padded_uv_image(a, [250, 250], "VISIBILITY_RESIDUAL")
    assert b.sizes["u"] == 250
    assert "residual" in b.attrs["data_groups"]["base"]
    assert b["VISIBILITY_RESIDUAL"].shape[3] == 250
    assert b["VISIBILITY_RESIDUAL"].data.dtype == np.complex64
    assert b["VISIBILITY_RESIDUAL_NORMALIZATION"].shape == (1, 1, 1)
    r = b["RESIDUAL"].data
    assert r.shape == (1, 1, 1, 250, 250) and r.dtype == np.float32
    assert r[0, 0, 0, 25 + 3, 25 + 5] == 7.0 and r.sum() == 200 * 200 - 1 + 7.0
    assert b.coords["u"].values[125] == 0.0 and b.coords["v"].values[125] == 0.0
    c = make_empty_padded_uv_image(a, [250, 250], "VISIBILITY_MODEL")
    assert "MODEL" not in c.data_vars and "RESIDUAL" not in c.data_vars
    with pytest.raises(Exception, match="is larger than requested"):
        make_empty_padded_uv_image(a, [150, 250])


def test_remove_padding_as_reference_test():
    """test_standard_image_grid_preparation.py:67-80 on the l / m
    coordinates: pixel (99, 99) of 200 x 200 is pixel (89, 89) of the
    180 x 180 centre."""
    from astroviper_b200.core.imaging.imaging_utils.standard_image_grid_preparation import (
        remove_padding)
    a = _ref_test_image()
    lo, mo = a.coords["l"].values[99], a.coords["m"].values[99]
    b = remove_padding(a, [180, 180])
    assert b.coords["l"].values[89] == lo and b.coords["m"].values[89] == mo
    assert b["SKY"].shape == (1, 1, 1, 180, 180)


# ----------------------------------------------------------------- GPU ---
def _prep():
    from astroviper_b200.core.imaging.imaging_utils import standard_image_grid_preparation as P
    return P


def _image(ins, uv_names=(), to_device=False):
    import torch
    from astroviper_b200.core.imaging.sky_image import SkyImage
    img = SkyImage()
    for n, x in ins.items():
        v = x.copy()
        if to_device:
            v = torch.from_numpy(v).cuda()
        img[n] = (UV_DIMS, v) if n in uv_names or n.startswith("VISIBILITY") and v.ndim == 5 \
            else v
    return img


def _np(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True])
def test_correct_fft_to_uv_bit_exact(on_device):
    P = _prep()
    g = golden("image_prep.npz")
    for case in _cases(g, "cfu_"):
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        img = _image(ins, uv_names=tuple(ins), to_device=on_device)
        before = {n: img[n].data for n in ins}
        if "named" in case:
            P.correct_fft_to_uv(img, "VISIBILITY_MODEL")
        else:
            P.correct_fft_to_uv(img)
        for n in ins:
            assert img[n].data is before[n], "the variable must be updated in place"
            assert same_bits(_np(img[n].data), outs[n]), (case, n, on_device)


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True])
def test_correct_ifft_to_lm_bit_exact(on_device):
    P = _prep()
    g = golden("image_prep.npz")
    for case in ("cil_f64", "cil_f32", "cil_c64"):
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        img = _image(ins, to_device=on_device)
        if case == "cil_c64":
            P.correct_ifft_to_lm(img, ["RESIDUAL"])
        else:
            P.correct_ifft_to_lm(img)
        for n in ins:
            assert same_bits(_np(img[n].data), outs[n]), (case, n, on_device)


@pytest.mark.gpu
def test_correct_ifft_to_lm_spheroid():
    P = _prep()
    g = golden("image_prep.npz")
    for case, args in (("cil_sph", dict(doSpheroidCorr=True)),
                       ("cil_sph_named", dict(data_vars="RESIDUAL", doSpheroidCorr=True,
                                              convsampling=64, convsupport=9))):
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        img = _image(ins)
        P.correct_ifft_to_lm(img, **args)
        for n in ins:
            got, ref = _np(img[n].data), outs[n]
            if n.endswith("NORMALIZATION"):
                assert same_bits(got, ref)
                continue
            tol = 1e-13 if got.dtype == np.float64 else 2e-7
            assert np.max(np.abs(got - ref) / np.abs(ref)) <= tol, (case, n)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.complex64, np.complex128])
def test_plane_rescale_spheroid_bit_exact_given_the_term(dtype):
    from astroviper_b200 import _kernels as K
    import torch
    rng = np.random.default_rng(7)
    shp = (2, 3, 2, 18, 14)
    x = rng.normal(size=shp)
    if np.dtype(dtype).kind == "c":
        x = x + 1j * rng.normal(size=shp)
    x = x.astype(dtype)
    x.reshape(-1)[:3] = [-0.0, np.inf, np.nan]
    norm = rng.uniform(1, 1e5, shp[:3])
    corr = K.corr_term(18, 14)
    t = torch.from_numpy(x.copy()).cuda()
    K.plane_rescale(t, 2, 18 * 14, corr, norm)
    want = x.copy()
    with np.errstate(all="ignore"):
        OI.correct_ifft_to_lm_planes(want, 18, 14, corr.cpu().numpy(), norm)
    assert same_bits(t.cpu().numpy(), want)


@pytest.mark.gpu
def test_transforms_match_reference():
    P = _prep()
    g = golden("image_prep.npz")
    ins, outs = _vars(g, "fft", "in"), _vars(g, "fft", "out")
    img = _image({**ins, "VISIBILITY_SKY": outs["VISIBILITY_SKY"] * 0,
                  "VISIBILITY_MODEL": outs["VISIBILITY_MODEL"] * 0})
    P.fft_to_uv(img)
    for n in ("VISIBILITY_SKY", "VISIBILITY_MODEL"):
        got, ref = _np(img[n].data), outs[n]
        peak = np.max(np.abs(ref), axis=(3, 4), keepdims=True)
        assert np.max(np.abs(got - ref) / peak) <= 1e-12, n
    ins, outs = _vars(g, "ifft", "in"), _vars(g, "ifft", "out")
    img = _image({**ins, "SKY": outs["SKY"] * 0, "RESIDUAL": outs["RESIDUAL"] * 0})
    P.ifft_to_lm(img)
    for n in ("SKY", "RESIDUAL"):
        got, ref = _np(img[n].data), outs[n]
        peak = np.max(np.abs(ref), axis=(3, 4), keepdims=True)
        assert np.max(np.abs(got - ref) / peak) <= 1e-12, n


@pytest.mark.gpu
def test_errors_follow_the_reference():
    P = _prep()
    rng = np.random.default_rng(3)
    img = _image({"SKY": rng.normal(size=(1, 1, 1, 8, 8))})
    with pytest.raises(Exception, match="Do not have VISIBILITY_NORMALIZATION"):
        P.correct_ifft_to_lm(img, doSpheroidCorr=True)
    with pytest.raises(Exception, match="VISIBILITY_SKY is not in"):
        P.fft_to_uv(img)
    with pytest.raises(KeyError):
        P.correct_fft_to_uv(img)  # no u / v dims, as image.sizes["u"] fails there
    with pytest.raises(KeyError):
        P.ifft_to_lm(_image({"VISIBILITY": np.zeros((1, 1, 1, 4, 4), complex)}))


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True])
def test_apply_pb_bit_exact(on_device):
    from astroviper_b200.core.imaging.sky_image import SkyImage
    P = _prep()
    g = golden("image_prep.npz")
    for case in _pb_cases(g):
        ins, outs = _vars(g, case, "in"), _vars(g, case, "out")
        multiply = case.endswith("_mul")
        if case == "pb_separate_div":
            img = _image({"RESIDUAL": ins["RESIDUAL"]}, to_device=on_device)
            beam = SkyImage({"PRIMARY_BEAM": ins["PRIMARY_BEAM"].copy()})
            before = img["RESIDUAL"].data
            P.apply_pb(img, beam, False, "RESIDUAL")
            assert img["RESIDUAL"].data is before
            assert same_bits(_np(img["RESIDUAL"].data), outs["RESIDUAL"]), case
            continue
        img = _image(ins, to_device=on_device)
        before = {n: img[n].data for n in ins}
        P.apply_pb(img, multiply=multiply)
        for n in ins:
            assert img[n].data is before[n]
            assert same_bits(_np(img[n].data), outs[n]), (case, n, on_device)


@pytest.mark.gpu
def test_apply_pb_errors_follow_the_reference():
    P = _prep()
    rng = np.random.default_rng(5)
    img = _image({"SKY": rng.normal(size=(1, 1, 1, 8, 8))})
    with pytest.raises(Exception, match="No Primary beam information"):
        P.apply_pb(img)
    img = _image({"SKY": rng.normal(size=(1, 1, 1, 8, 8)),
                  "PRIMARY_BEAM": rng.normal(size=(1, 1, 1, 8, 6))})
    with pytest.raises(Exception, match="shapes on sky are not the same"):
        P.apply_pb(img)
    with pytest.raises(KeyError):
        P.apply_pb(img, data_vars="RESIDUAL")


class _Node:
    """Duck-typed MSv4 node: UVW, WEIGHT, FLAG, the data variables, frequency."""

    class _V:
        def __init__(self, v):
            self.data = v
            self.values = v

    def __init__(self, vis, uvw, weight, flag, freq):
        self._d = {"VISIBILITY": self._V(vis), "UV_SAMPLING": self._V(vis)}
        self.UVW, self.WEIGHT, self.FLAG = self._V(uvw), self._V(weight), self._V(flag)
        self.coords = {"frequency": self._V(freq)}

    def __getitem__(self, k):
        return self._d[k]


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_grid2xradio_spheroid_ms4_matches_reference(on_device, precision, tol):
    import torch
    from astroviper_b200.core.imaging.sky_image import SkyImage
    P = _prep()
    g = golden("image_prep.npz")
    for tag, data_var, mode in (("vis", "VISIBILITY", "continuum"),
                                ("psf", "UV_SAMPLING", "cube")):
        ref = g[f"ms4_{tag}/grid"]
        nodes = [_Node(*n) for n in _ms4_nodes(g, tag)]
        grid = np.zeros(ref.shape, complex)
        sumwt = np.zeros(ref.shape[:3])
        if on_device:
            grid, sumwt = torch.from_numpy(grid).cuda(), torch.from_numpy(sumwt).cuda()
        img = SkyImage(coords={"time": [5.0, 15.0], "l": (np.arange(64) - 32) * -MS4_CELL[0],
                               "m": (np.arange(48) - 24) * MS4_CELL[1]})
        img[data_var] = (UV_DIMS, grid)
        img[data_var + "_NORMALIZATION"] = sumwt
        P.grid2xradio_spheroid_ms4(nodes, img, data_var=data_var, chan_mode=mode,
                                   precision=precision)
        assert img[data_var].data is grid
        got, sw = _np(img[data_var].data), _np(img[data_var + "_NORMALIZATION"].data)
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)), (tag, on_device)
        assert np.allclose(sw, g[f"ms4_{tag}/sumwt"], rtol=tol, atol=0), (tag, on_device)
        for k, node in enumerate(nodes):
            assert np.array_equal(node.WEIGHT.data, g[f"ms4_{tag}/node{k}/weight_after"])
    with pytest.raises(Exception, match="VISIBILITY_MODEL is not in"):
        P.grid2xradio_spheroid_ms4(nodes, img, data_var="VISIBILITY_MODEL")
    with pytest.raises(TypeError, match="not an xarray datatree"):
        P.grid2xradio_spheroid_ms4([nodes[0], object()], img, data_var="UV_SAMPLING",
                                   chan_mode="cube")


@pytest.mark.gpu
def test_reference_unit_tests_known_answers():
    """The known answers of test_standard_image_grid_preparation.py:97-148
    (_mult_div, apply_pb, fft_to_uv + correct_fft_to_uv, ifft_to_lm).  The
    FFT values are compared to 1e-6 relative (the reference asserts numpy's
    exact values; cuFFT rounds differently)."""
    P = _prep()
    for via_apply in (False, True):
        a = _ref_test_image(npol=1, nchan=2)
        a["PRIMARY_BEAM"] = np.ones(a["SKY"].shape, dtype=np.float32)
        a["PRIMARY_BEAM"].data[0, 1, 0, :, :] = 0
        if via_apply:
            P.apply_pb(a, data_vars="SKY", multiply=True)
        else:
            P._mult_div(a["SKY"], a["PRIMARY_BEAM"], multiply=True)
        assert np.max(a["SKY"].data[0, 0, 0, :, :]) == 1.0
        assert np.max(a["SKY"].data[0, 1, 0, :, :]) == 0.0
    a = _ref_test_image(which="RESIDUAL")
    b = P.make_empty_padded_uv_image(a, image_size=[200, 200])
    P.fft_to_uv(b)
    vis = b["VISIBILITY_RESIDUAL"].data
    assert abs(vis[0, 0, 0, 100, 100] - 200 * 200) <= 1e-6 * 200 * 200
    P.correct_fft_to_uv(b)
    vis = b["VISIBILITY_RESIDUAL"].data
    assert abs(vis[0, 0, 0, 100, 100] - 1.0) <= 1e-6
    assert abs(vis[0, 0, 0, 99, 99]) <= 1e-6
    b = P.make_empty_padded_uv_image(a, image_size=[200, 200])
    b["VISIBILITY_RESIDUAL"].data[0, 0, 0, 100, 100] = 10
    P.ifft_to_lm(b)
    assert abs(float(np.max(b["RESIDUAL"].data)) - 10.0 / 200.0 / 200.0) <= 1e-6 * 2.5e-4
