"""Host logic of the imaging loop on CPU: ReturnDict, merge_return_dicts,
the ReturnDict readers and IterationController replayed against the results
of the reference's own classes (tests/golden/imager_control.json, made by
tests/golden/make_golden_imager.py), the oracle's restatements of the
polarisation products and of extract_main_lobe's sidelobe against the
reference's outputs (tests/golden/imager.npz), and the argument checks of the
Stokes conversions, which raise before any device work."""
import json
import os
import sys
import types

import numpy as np
import pytest

from conftest import ROOT, golden

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import imager_ops  # noqa: E402


def _api():
    from astroviper_b200.core.imaging.imaging_utils import iteration_control as IC
    from astroviper_b200.core.imaging.imaging_utils import return_dict as RD
    api = types.SimpleNamespace(ReturnDict=RD.ReturnDict,
                                IterationController=IC.IterationController,
                                merge_return_dicts=IC.merge_return_dicts)
    for name in imager_ops.READERS:
        setattr(api, name, getattr(IC, name))
    return api


with open(os.path.join(ROOT, "tests", "golden", "imager_control.json")) as _f:
    CONTROL = json.load(_f)


@pytest.mark.parametrize("scenario", sorted(imager_ops.SCENARIOS))
def test_control_scenario_matches_reference(scenario):
    got = imager_ops.run(scenario, _api())
    want = CONTROL[scenario]
    assert len(got) == len(want)
    for i, (g, w) in enumerate(zip(got, want)):
        assert g == w, (scenario, i, imager_ops.SCENARIOS[scenario]["ops"][i])


def test_stop_code_tables():
    from astroviper_b200.core.imaging.imaging_utils import iteration_control as IC
    assert (IC.MAJOR_CONTINUE, IC.MAJOR_ITER_LIMIT, IC.MAJOR_THRESHOLD, IC.MAJOR_ZERO_MASK,
            IC.MAJOR_CYCLE_LIMIT) == (0, 1, 2, 7, 9)
    assert (IC.MINOR_CONTINUE, IC.MINOR_ITER_LIMIT, IC.MINOR_THRESHOLD, IC.MINOR_DIVERGENCE,
            IC.MINOR_ZERO_MASK) == (0, 1, 2, 4, 7)
    c = IC.IterationController()
    assert c.stopcode == IC.StopCode(0, 0) and c.stopdescription == "Continue iterations"


def test_return_dict_history_rules():
    from astroviper_b200.core.imaging.imaging_utils.return_dict import Key, ReturnDict
    rd = ReturnDict()
    rd.add({"peakres": 1.0, "loop_gain": 0.1, "other": "a"}, 0, 1, 2)
    rd.add({"peakres": 0.5, "loop_gain": 0.2, "other": "b"}, 0, 1, 2)
    e = rd.data[Key(0, 1, 2)]
    assert e == {"peakres": [1.0, 0.5], "loop_gain": 0.2, "other": "b"}
    assert rd.sel(chan=2) is e and rd.sel(chan=3) is None and rd.to_dict() is rd.data


def test_oracle_polarisation_products_match_reference():
    import oracle.imager as OI
    g = golden("imager.npz")
    kw = {"c1": ("linear", 2, ["I", "Q", "U", "V"]), "c2": ("linear", 2, ["V", "I"]),
          "c3": ("circular", 1, ["I", "Q", "U", "V"]), "c4": ("linear", 1, ["I", "Q"]),
          "c5": ("circular", -3, ["V"]), "c6": ("linear", 1, ["I"]),
          "c7": ("circular", 2, ["I", "Q", "U", "V"])}
    for k, (ct, ax, so) in kw.items():
        out = OI.image_corr_to_stokes(g[k + "_in"], ct, ax, so)
        assert out.dtype == g[k + "_out"].dtype and np.array_equal(out, g[k + "_out"]), k
    kw = {"s1": ("linear", ["I", "Q", "U", "V"]), "s2": ("linear", ["I", "Q"]),
          "s3": ("linear", ["I"]), "s4": ("circular", ["I", "V"]),
          "s5": ("linear", ["I", "U"]), "s6": ("circular", ["I", "Q", "U", "V"])}
    for k, (ct, si) in kw.items():
        out = OI.image_stokes_to_corr(g[k + "_in"], ct, 1, si)
        assert out.dtype == g[k + "_out"].dtype and np.array_equal(out, g[k + "_out"]), k


def test_oracle_sidelobe_matches_reference():
    import oracle.imager as OI
    g = golden("imager.npz")
    for i in range(int(g["n_psf"])):
        assert OI.psf_max_sidelobe(g[f"psf{i}"]) == float(g[f"psf{i}_sidelobe"]), i


def test_stokes_argument_errors_match_reference():
    from astroviper_b200.core.imaging.imaging_utils import corr_to_stokes as CS
    x = np.zeros((2, 2, 3, 3))
    with pytest.raises(ValueError, match="corr_type is required for numpy input"):
        CS.image_corr_to_stokes(x, pol_axis=1)
    with pytest.raises(ValueError, match=r"Minimum 2 correlations required .* got 1"):
        CS.image_corr_to_stokes(np.zeros((2, 1, 3)), "linear", pol_axis=1)
    with pytest.raises(ValueError, match=r"2-pol linear data \(XX, YY\) cannot produce Stokes "
                                         r"\{'U'\}"):
        CS.image_corr_to_stokes(x, "linear", pol_axis=1, stokes_out=["U"])
    with pytest.raises(ValueError, match=r"2-pol circular data \(RR, LL\) cannot produce"):
        CS.image_corr_to_stokes(x, "circular", pol_axis=1, stokes_out=["Q"])
    with pytest.raises(ValueError, match="Invalid Stokes parameters: {'X'}"):
        CS.image_corr_to_stokes(x, "linear", pol_axis=1, stokes_out=["X"])
    with pytest.raises(ValueError, match="2-pol conversion requires corr_type"):
        CS.image_corr_to_stokes(x, "custom", pol_axis=1)
    with pytest.raises(ValueError, match=r"Cannot produce 4-pol output from 2-Stokes input"):
        CS.image_stokes_to_corr(x, "linear", pol_axis=1, corr_out=4)
    with pytest.raises(ValueError, match="corr_out must be 2 or 4, got 3"):
        CS.image_stokes_to_corr(x, "linear", pol_axis=1, corr_out=3)
    with pytest.raises(ValueError, match=r"stokes_in length \(1\) doesn't match"):
        CS.image_stokes_to_corr(x, "linear", pol_axis=1, stokes_in=["I"])
    with pytest.raises(ValueError, match="Unexpected number of Stokes parameters: 3"):
        CS.image_stokes_to_corr(np.zeros((2, 3, 2)), "linear", pol_axis=1)
    with pytest.raises(ValueError, match="without Stokes I"):
        CS.image_stokes_to_corr(x, "linear", pol_axis=1, stokes_in=["Q", "U"])
    with pytest.raises(ValueError, match="a transformation_matrix must be provided"):
        CS.corr_to_stokes(np.zeros((3, 4)), "custom")


def test_imager_parameter_defaults_and_errors():
    from astroviper_b200.core.imaging import imager
    assert imager._DEFAULT_PARAMS["nmajor"] == 10 and imager._DEFAULT_PARAMS["chan_mode"] == "cube"
    with pytest.raises(ValueError, match="cell_size must be specified in params"):
        imager.run_imaging_loop(object(), {"image_size": (8, 8)})


def test_deconvolve_argument_errors():
    from astroviper_b200.core.imaging.deconvolution import deconvolve
    from astroviper_b200.core.imaging.sky_image import make_sky_image
    d = make_sky_image((0.0, 0.0), (8, 8), (1e-5, 1e-5), [1e9], ["I", "Q"], [0.0])
    d["RESIDUAL"] = np.zeros((1, 1, 2, 8, 8))
    p = make_sky_image((0.0, 0.0), (8, 8), (1e-5, 1e-5), [1e9], ["I", "Q", "U"], [0.0])
    p["POINT_SPREAD_FUNCTION"] = np.zeros((1, 1, 3, 8, 8))
    with pytest.raises(ValueError, match=r"npol_psf = 3, npol_image = 2"):
        deconvolve(d, p)
    p2 = make_sky_image((0.0, 0.0), (8, 8), (1e-5, 1e-5), [1e9], ["I"], [0.0])
    p2["POINT_SPREAD_FUNCTION"] = np.zeros((1, 1, 1, 8, 8))
    with pytest.raises(ValueError, match="Deconvolution algorithm 'clark' not recognized."):
        deconvolve(d, p2, algorithm="clark", deconv_params={})
