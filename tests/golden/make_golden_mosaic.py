"""Generates the mosaic-gridding fixtures in this folder from the reference.

Run in a container that has the astroviper source tree (default
``reference/`` beside this repository, override with ``AV_REFERENCE_ROOT``):

    python tests/golden/make_golden_mosaic.py

Writes mosaic.npz with the inputs and outputs of the reference's
make_pb_symmetric.py beams, the convolution-function helpers of
make_gridding_convolution_function.py (create_cf_baseline_map,
create_cf_chan_map, make_baseline_patterns, resize_and_calc_support,
calc_conv_size) and its Numba kernels mosaic_grid_jit / aperture_grid_jit
(mosaic_grid.py), run on a convolution function the helpers build; and
gcf_driver.npz with the variables the driver make_gridding_convolution_function
itself builds for a duck-typed measurement set (``... make_golden_mosaic.py
gcf_driver`` writes only that one).  The reference modules are imported
unmodified, with stand-in modules for xarray and toolviper's logger.
"""
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

from make_golden import _DataArray, _DataTree, _mod, _pkg  # noqa: E402


def load_reference():
    xr = types.ModuleType("xarray")
    core = types.ModuleType("xarray.core")
    dt = types.ModuleType("xarray.core.datatree")
    dt.DataTree = _DataTree
    core.datatree = dt
    xr.core = core
    xr.DataArray = _DataArray
    xr.DataTree = _DataTree
    xr.Dataset = type("Dataset", (), {})
    sys.modules.update({"xarray": xr, "xarray.core": core, "xarray.core.datatree": dt})
    tv = types.ModuleType("toolviper")
    tvu = types.ModuleType("toolviper.utils")
    tvl = types.ModuleType("toolviper.utils.logger")
    for name in ("info", "debug", "warning", "error", "critical"):
        setattr(tvl, name, lambda *a, **k: None)
    tvu.logger = tvl
    tv.utils = tvu
    sys.modules.update({"toolviper": tv, "toolviper.utils": tvu, "toolviper.utils.logger": tvl})
    ap = types.ModuleType("astropy")
    apc = types.ModuleType("astropy.constants")
    apc.c = types.SimpleNamespace(value=299792458.0)
    ap.constants = apc
    sys.modules.update({"astropy": ap, "astropy.constants": apc})
    _pkg("astroviper", SRC)
    _pkg("astroviper.utils", SRC + "/utils")
    _pkg("astroviper.core", SRC + "/core")
    _pkg("astroviper.core.imaging", SRC + "/core/imaging")
    _pkg("astroviper.core.imaging.imaging_utils", SRC + "/core/imaging/imaging_utils")
    iu = SRC + "/core/imaging/imaging_utils/"
    ns = types.SimpleNamespace()
    ns.pb = _mod("astroviper.core.imaging.imaging_utils.make_pb_symmetric",
                 iu + "make_pb_symmetric.py")
    ns.mg = _mod("astroviper.core.imaging.imaging_utils.mosaic_grid", iu + "mosaic_grid.py")
    _mod("astroviper.core.imaging.imaging_utils.gcf_prolate_spheroidal",
         iu + "gcf_prolate_spheroidal.py")
    _mod("astroviper.core.imaging.imaging_utils.standard_grid", iu + "standard_grid.py")
    _mod("astroviper.utils.check_params", SRC + "/utils/check_params.py")
    _mod("astroviper.core.imaging.check_imaging_parameters",
         SRC + "/core/imaging/check_imaging_parameters.py")
    ns.gcf = _mod("astroviper.core.imaging.make_gridding_convolution_function",
                  SRC + "/core/imaging/make_gridding_convolution_function.py")
    return ns


class _DA:
    """xarray.DataArray stand-in: values and dims."""

    def __init__(self, data, coords=None, dims=None):
        self.data = self.values = np.asarray(data)
        self.dims = (dims,) if isinstance(dims, str) else tuple(dims or ())


class _DS:
    """xarray.Dataset stand-in for the driver: item assignment, attrs, len,
    assign_coords.  Every instance is kept in CREATED, so the dataset the
    driver fills can be read back after the call."""
    CREATED = []

    def __init__(self):
        self.vars = {}
        self.attrs = {}
        _DS.CREATED.append(self)

    def __len__(self):
        return len(self.vars)

    def __setitem__(self, name, value):
        self.vars[name] = value

    def assign_coords(self, coords):
        return self


def make_gcf_driver(ns):
    """make_gridding_convolution_function (:24-193) on a duck-typed MSv4
    dataset of 6 antennas of two types (12 m / 25 m dishes) and 15 baselines
    whose antenna-2 names are not sorted, 7 channels over 1.0-1.5 GHz, 2
    polarisations.  Its last step, make_phase_gradient, needs astropy.wcs,
    which this container lacks: the call stops there with ImportError, after
    every other variable is in the dataset, which _DS keeps.  Writes
    gcf_driver.npz."""
    import xarray
    xarray.Dataset = _DS
    xarray.DataArray = _DA
    ns.gcf.xr = xarray
    names = [f"ant{i}" for i in range(6)]
    pairs = [(i, j) for i in range(6) for j in range(i + 1, 6)]
    freq = np.linspace(1.0e9, 1.5e9, 7)
    pols = np.array(["XX", "YY"])
    ra_dec = np.array([0.31, -0.52])

    class _Field:
        def isel(self, **kw):
            return types.SimpleNamespace(data=ra_dec)

    ms = types.SimpleNamespace(
        data_vars=["VISIBILITY", "UVW", "WEIGHT", "FLAG"],
        attrs={"data_groups": {"base": {"correlated_data": "VISIBILITY", "uvw": "UVW",
                                        "weight": "WEIGHT", "flag": "FLAG"}}},
        xr_ms=types.SimpleNamespace(get_field_and_source_xds=lambda name: types.SimpleNamespace(
            FIELD_PHASE_CENTER_DIRECTION=_Field())),
        # xarray compares (antenna) with (baseline) names as a 2-D outer test
        antenna_xds=types.SimpleNamespace(antenna_name=np.array(names)[:, None]),
        baseline_antenna1_name=np.array([names[i] for i, _ in pairs]),
        baseline_antenna2_name=np.array([names[j] for _, j in pairs]),
        frequency=types.SimpleNamespace(values=freq),
        polarization=types.SimpleNamespace(values=pols))
    gcf_params = {"function": "casa_airy", "list_dish_diameters": [12.0, 25.0],
                  "list_blockage_diameters": [0.75, 0.0], "unique_ant_indx": [0, 1, 0, 1, 1, 0],
                  "oversampling": [4, 4], "max_support": [11, 11], "support_cut_level": 0.025,
                  "chan_tolerance_factor": 0.05,
                  "phase_direction": types.SimpleNamespace(values=np.array([0.3, -0.5]))}
    grid_params = {"image_size": [64, 64], "cell_size": [-1e-4, 1e-4], "fft_padding": 1.5,
                   "chan_mode": "cube"}
    _DS.CREATED.clear()
    try:
        ns.gcf.make_gridding_convolution_function(_DS(), ms, gcf_params, grid_params, {})
        raise SystemExit("expected the driver to stop at astropy.wcs")
    except ImportError:
        pass
    ds = _DS.CREATED[-1]
    d = {f"var_{k}": v.values for k, v in ds.vars.items()}
    d.update({f"dims_{k}": np.array(v.dims) for k, v in ds.vars.items()})
    d["attr_cell_uv"] = ds.attrs["cell_uv"]
    d["attr_oversampling"] = ds.attrs["oversampling"]
    d.update(names=np.array(names), pairs=np.array(pairs), freq=freq, pols=pols, ra_dec=ra_dec)
    np.savez_compressed(os.path.join(HERE, "gcf_driver.npz"), **d)
    print("wrote gcf_driver.npz", sorted(ds.vars))


def main():
    ns = load_reference()
    rng = np.random.default_rng(20260120)
    d = {}
    # primary beams
    freq = np.array([0.9e9, 1.4e9])
    pol = np.array([0, 1])
    pbp = {"list_dish_diameters": np.array([12.0, 25.0, 12.0]),
           "list_blockage_diameters": np.array([0.75, 0.0, 2.0]), "ipower": 1}
    gp = {"cell_size": np.array([-8e-4, 8e-4]), "image_size": np.array([48, 40]),
          "image_center": np.array([24, 20])}
    for name in ("airy_disk", "casa_airy_disk", "airy_disk_rorder", "casa_airy_disk_rorder"):
        for ip in (1, 2):
            pbp["ipower"] = ip
            d[f"pb_{name}_{ip}"] = getattr(ns.pb, name)(freq, pol, dict(pbp), dict(gp))
    d["pb_freq"], d["pb_cell"], d["pb_size"], d["pb_center"] = freq, gp["cell_size"], \
        gp["image_size"], gp["image_center"]
    d["pb_dish"], d["pb_block"] = pbp["list_dish_diameters"], pbp["list_blockage_diameters"]

    # convolution-function helpers
    uai = np.array([0, 1, 0, 1, 1, 0])
    bant = np.array([[i, j] for i in range(6) for j in range(i + 1, 6)])
    cbm, pairs = ns.gcf.create_cf_baseline_map(uai, bant, 2)
    d["cbm_unique_ant_indx"], d["cbm_baseline_ant"] = uai, bant
    d["cbm_map"], d["cbm_pairs"] = cbm, pairs
    for i, (fc, tol) in enumerate(((np.linspace(1.0e9, 1.2e9, 16), 0.05),
                                   (np.linspace(1.0e9, 1.5e9, 7), 0.01),
                                   (np.array([1.4e9]), 0.01),
                                   (np.linspace(0.9e9, 1.7e9, 33), 0.1))):
        m, pf = ns.gcf.create_cf_chan_map(fc, tol)
        d[f"ccm{i}_freq"], d[f"ccm{i}_tol"], d[f"ccm{i}_map"], d[f"ccm{i}_pbfreq"] = \
            fc, np.float64(tol), m, pf
    d["n_ccm"] = 4

    gcf_params = {"list_dish_diameters": np.array([12.0, 25.0]),
                  "list_blockage_diameters": np.array([0.75, 0.0]), "oversampling": np.array([4, 4]),
                  "max_support": np.array([11, 11]), "support_cut_level": 0.025}
    gcf_params["resize_conv_size"] = (gcf_params["max_support"] + 1) * gcf_params["oversampling"]
    grid_params = {"image_size": np.array([64, 64]), "image_size_padded": np.array([96, 96]),
                   "cell_size": np.array([-1e-4, 1e-4])}
    pb_freq = np.array([1.1e9, 1.4e9])
    pb_pol = np.array([0])
    pb_pairs = np.array([[0, 0], [0, 1], [1, 1]])
    gcf_params["ipower"] = 1
    bp = ns.gcf.make_baseline_patterns(pb_freq, pb_pol, pb_pairs, ns.pb.airy_disk_rorder,
                                       dict(gcf_params), dict(grid_params))
    gcf_params["ipower"] = 2
    bp2 = ns.gcf.make_baseline_patterns(pb_freq, pb_pol, pb_pairs, ns.pb.airy_disk_rorder,
                                        dict(gcf_params), dict(grid_params))
    d["bp1"], d["bp2"] = bp, bp2
    ck = np.real(np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(bp, axes=(3, 4)), axes=(3, 4)),
                                 axes=(3, 4)))
    ckc = np.real(np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(bp2, axes=(3, 4)), axes=(3, 4)),
                                  axes=(3, 4)))
    d["ck"], d["ckc"] = ck, ckc
    rk, rkc, sup = ns.gcf.resize_and_calc_support(ck, ckc, dict(gcf_params), dict(grid_params))
    d["rk"], d["rkc"], d["support"] = rk, rkc, sup
    d["conv_size_one"] = np.array(ns.gcf.calc_conv_size(
        ckc[1, 0, 0], grid_params["image_size_padded"], 0.025, gcf_params["oversampling"],
        gcf_params["max_support"]))
    d["gcf_oversampling"], d["gcf_max_support"] = gcf_params["oversampling"], \
        gcf_params["max_support"]
    d["gcf_cut"] = np.float64(0.025)
    d["grid_image_size_padded"], d["grid_cell"] = grid_params["image_size_padded"], \
        grid_params["cell_size"]

    # the Numba mosaic and aperture kernels on the function just built
    from astroviper_b200 import synthetic as S
    uvw, _ = S.array_uvw(6, 12, radius_m=40.0, seed=20260121)
    nb = uvw.shape[1]
    uvw[2, 3, 0] = np.nan
    nchan, npol = 2, 2
    fr = np.array([1.1e9, 1.38e9])
    shape = (uvw.shape[0], nb, nchan, npol)
    vis = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    wt = rng.uniform(0.5, 2.0, size=shape)
    wt[1, 2, 0, 1] = 0.0
    wt[3, 1, 1, 0] = np.nan
    cfb = np.array([k % 3 for k in range(nb)])
    cfc = np.array([0, 1])
    cfp = np.array([0, 0])
    n_uv = grid_params["image_size_padded"]
    rcs = gcf_params["resize_conv_size"]
    cx, cy = rcs // 2
    x, y = np.meshgrid(np.arange(-cx, rcs[0] - cx), np.arange(-cy, rcs[1] - cy), indexing="ij")
    pg = np.exp(1j * (x * 0.013 - y * 0.021))[None]
    for tag, chan_map in (("cube", np.arange(nchan)), ("cont", np.zeros(nchan, dtype=int))):
        nic = nchan if tag == "cube" else 1
        for do_psf in (False, True):
            g = np.zeros((nic, npol, n_uv[0], n_uv[1]), dtype=np.complex128)
            sw = np.zeros((nic, npol))
            ns.mg.mosaic_grid_jit(g, sw, do_psf, vis, uvw, fr, chan_map, np.arange(npol), cfb,
                                  cfc, cfp, wt, rk, n_uv, grid_params["cell_size"], sup,
                                  gcf_params["oversampling"], pg)
            d[f"mg_{tag}_{int(do_psf)}_grid"], d[f"mg_{tag}_{int(do_psf)}_sw"] = g, sw
        g = np.zeros((nic, npol, n_uv[0], n_uv[1]), dtype=np.complex128)
        sw = np.zeros((nic, npol))
        ns.mg.aperture_grid_jit(g, sw, uvw, fr, chan_map, np.arange(npol), cfb, cfc, cfp, wt,
                                rkc, n_uv, grid_params["cell_size"], sup,
                                gcf_params["oversampling"], pg)
        d[f"ag_{tag}_grid"], d[f"ag_{tag}_sw"] = g, sw
    d.update(mg_uvw=uvw, mg_vis=vis, mg_wt=wt, mg_freq=fr, mg_cfb=cfb, mg_cfc=cfc, mg_cfp=cfp,
             mg_pg=pg)
    np.savez_compressed(os.path.join(HERE, "mosaic.npz"), **d)
    print("wrote mosaic.npz")


if __name__ == "__main__":
    if sys.argv[1:] == ["gcf_driver"]:
        make_gcf_driver(load_reference())
    else:
        main()
        make_gcf_driver(load_reference())
