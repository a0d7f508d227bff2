"""Generates the imager fixtures in this folder from the reference itself.

Run in a container that has the astroviper source tree (default
``reference/`` beside this repository, override with ``AV_REFERENCE_ROOT``):

    python tests/golden/make_golden_imager.py

Writes
* imager_control.json: the results of every scenario of imager_ops.py run
  against the reference's ReturnDict, merge_return_dicts, readers and
  IterationController (return_dict.py, iteration_control.py);
* imager_loop.json: the decisions of the reference's controller in the
  oracle's imaging loop on each of imager_ops.LOOP_CASES;
* imager.npz: inputs and outputs of the reference's corr_to_stokes,
  stokes_to_corr, image_corr_to_stokes and image_stokes_to_corr
  (corr_to_stokes.py), and PSF planes with the max_sidelobe of its
  extract_main_lobe (psf_gaussian_fit.py:46-126).
The reference modules are imported unmodified, with a stand-in module for
xarray (whose types the code only tests against).
"""
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("AV_REFERENCE_ROOT",
                     os.path.join(os.path.dirname(REPO), "reference"))
SRC = os.path.join(REF, "src", "astroviper")
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

import imager_ops  # noqa: E402
from make_golden import _DataArray, _DataTree, _mod, _pkg  # noqa: E402


def load_reference():
    xr = types.ModuleType("xarray")
    xr.DataArray = _DataArray
    xr.DataTree = _DataTree
    xr.Dataset = type("Dataset", (), {})  # annotations only
    sys.modules["xarray"] = xr
    _pkg("astroviper", SRC)
    _pkg("astroviper.core", SRC + "/core")
    _pkg("astroviper.core.imaging", SRC + "/core/imaging")
    _pkg("astroviper.core.imaging.imaging_utils", SRC + "/core/imaging/imaging_utils")
    _pkg("astroviper.core.image_analysis", SRC + "/core/image_analysis")
    iu = SRC + "/core/imaging/imaging_utils/"
    ns = types.SimpleNamespace()
    ns.rd = _mod("astroviper.core.imaging.imaging_utils.return_dict", iu + "return_dict.py")
    ns.ic = _mod("astroviper.core.imaging.imaging_utils.iteration_control",
                 iu + "iteration_control.py")
    ns.cs = _mod("astroviper.core.imaging.imaging_utils.corr_to_stokes", iu + "corr_to_stokes.py")
    ns.pg = _mod("astroviper.core.image_analysis.psf_gaussian_fit",
                 SRC + "/core/image_analysis/psf_gaussian_fit.py")
    return ns


def control(ns):
    api = types.SimpleNamespace(ReturnDict=ns.rd.ReturnDict,
                                IterationController=ns.ic.IterationController,
                                merge_return_dicts=ns.ic.merge_return_dicts)
    for name in imager_ops.READERS:
        setattr(api, name, getattr(ns.ic, name))
    out = {name: imager_ops.run(name, api) for name in imager_ops.SCENARIOS}
    with open(os.path.join(HERE, "imager_control.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)


def stokes_cases(ns, rng):
    cs = ns.cs
    d = {}
    real4 = rng.normal(size=(2, 3, 4, 5, 6))
    cplx4 = rng.normal(size=(3, 4, 7)) + 1j * rng.normal(size=(3, 4, 7))
    real2 = rng.normal(size=(2, 2, 5, 5)).astype(np.float32)
    real2b = rng.normal(size=(2, 2, 4, 4))
    cplx2 = (rng.normal(size=(3, 2, 6)) + 1j * rng.normal(size=(3, 2, 6))).astype(np.complex64)
    cases = {
        "c1": (real4, dict(corr_type="linear", pol_axis=2)),
        "c2": (real4, dict(corr_type="linear", pol_axis=2, stokes_out=["V", "I"])),
        "c3": (cplx4, dict(corr_type="circular", pol_axis=1)),
        "c4": (real2, dict(corr_type="linear", pol_axis=1)),
        "c5": (real2b, dict(corr_type="circular", pol_axis=-3, stokes_out=["V"])),
        "c6": (cplx2, dict(corr_type="linear", pol_axis=1, stokes_out=["I"])),
        "c7": (real4, dict(corr_type="circular", pol_axis=2, stokes_out=["U", "Q", "V", "I"])),
    }
    for k, (x, kw) in cases.items():
        d[k + "_in"] = x
        d[k + "_out"] = cs.image_corr_to_stokes(x, **kw)
    st4 = rng.normal(size=(2, 4, 5, 5))
    st2 = rng.normal(size=(2, 2, 4, 4)).astype(np.float32)
    st1 = rng.normal(size=(3, 1, 4, 4))
    st2c = rng.normal(size=(2, 2, 3)) + 1j * rng.normal(size=(2, 2, 3))
    cases = {
        "s1": (st4, dict(corr_type="linear", pol_axis=1)),
        "s2": (st2, dict(corr_type="linear", pol_axis=1)),
        "s3": (st1, dict(corr_type="linear", pol_axis=1)),
        "s4": (st2c, dict(corr_type="circular", pol_axis=1)),
        "s5": (st2.astype(np.float64), dict(corr_type="linear", pol_axis=1,
                                            stokes_in=["I", "U"])),
        "s6": (st4, dict(corr_type="circular", pol_axis=1)),
    }
    for k, (x, kw) in cases.items():
        d[k + "_in"] = x
        d[k + "_out"] = cs.image_stokes_to_corr(x, **kw)
    b = rng.normal(size=(5, 3, 4)) + 1j * rng.normal(size=(5, 3, 4))
    d["b_in"] = b
    d["b1_out"] = cs.corr_to_stokes(b, "linear")
    d["b2_out"] = cs.stokes_to_corr(b, "circular")
    custom = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    d["b_custom"] = custom
    d["b3_out"] = cs.corr_to_stokes(b, "custom", transformation_matrix=custom)
    return d


def sidelobe_cases(ns, rng):
    from astroviper_b200 import synthetic as S
    d = {}
    planes = []
    for n_time, size, cell_as in ((20, (128, 128), 2.0), (50, (96, 96), 1.0),
                                  (8, (64, 96), 4.0)):
        uvw, _ = S.array_uvw(64, n_time, seed=20260101 + n_time)
        pix = np.array([-cell_as, cell_as]) * np.pi / 180 / 3600
        planes.append(S.sampling_psf(uvw, np.array([1.4e9]), np.array(size), pix))
    # a Gaussian beam with ring sidelobes, peak near an edge (clipped window)
    y, x = np.mgrid[0:80, 0:80]
    r = np.hypot(y - 5, x - 70)
    planes.append(np.exp(-0.5 * (r / 2.5) ** 2) + 0.12 * np.cos(r / 1.7) * np.exp(-r / 25))
    # two lobes above the cut, the second one touching the window edge
    g = np.zeros((64, 64))
    g[32, 32] = 1.0
    g[31:34, 31:34] += 0.5
    g[32, 40:52] = 0.6
    g[10, 10] = 0.3
    planes.append(g)
    # constant zero plane
    planes.append(np.zeros((16, 16)))
    for i, p in enumerate(planes):
        d[f"psf{i}"] = p
        _, _, _, sl = ns.pg.extract_main_lobe((41, 41), 0.35, p[None, None, None])
        d[f"psf{i}_sidelobe"] = np.float64(sl)
    d["n_psf"] = len(planes)
    return d


def loop(ns):
    """The oracle's imaging loop (oracle/imager.py, imager.py:108-351 restated)
    driven by the reference's own IterationController, merge_return_dicts and
    ReturnDict on every imager_ops.LOOP_CASES case: the decisions the
    reference's controller takes on the loop's actual peaks and sidelobes."""
    import oracle.imager as OI
    out = {}
    for name in imager_ops.LOOP_CASES:
        vis, uvw, weight, flag, freq, _pols, params, init = imager_ops.loop_case(name)
        ctl = ns.ic.IterationController(niter=params["niter"], nmajor=params["nmajor"],
                                        threshold=params["threshold"], gain=params["gain"],
                                        cyclefactor=params["cyclefactor"])
        res = OI.run_imaging_loop(vis, uvw, weight, flag, freq, params, ctl,
                                  ns.ic.merge_return_dicts, ns.rd.ReturnDict, init)
        out[name] = imager_ops.loop_decisions(res)
    with open(os.path.join(HERE, "imager_loop.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)


def main():
    ns = load_reference()
    control(ns)
    loop(ns)
    rng = np.random.default_rng(20260110)
    d = {}
    d.update(stokes_cases(ns, rng))
    d.update(sidelobe_cases(ns, rng))
    np.savez_compressed(os.path.join(HERE, "imager.npz"), **d)
    print("wrote imager_control.json, imager_loop.json and imager.npz")


if __name__ == "__main__":
    main()
