"""Generates the golden fixtures in this folder from the reference itself.

Run in a container that has the astroviper source tree (default
``reference/`` beside this repository, override with ``AV_REFERENCE_ROOT``) and the reference's
Hogbom extension built by ``oracle/build_ref.sh``:

    python tests/golden/make_golden.py

The reference's Numba kernels are imported unmodified from the source tree,
with small stand-ins for the modules this container lacks (``xarray``'s
DataTree / DataArray types, ``astropy.constants.c``).  Outputs are written as
compressed ``.npz`` files holding both the inputs and the reference outputs,
so the tests never need the reference tree.
"""
import glob
import importlib.util
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


class _DataTree:
    """Stand-in for xarray.core.datatree.DataTree (type checks only)."""


class _DataArray:
    def __init__(self, data, coords=None, dims=None):
        self.data = data
        self.values = data


def _pkg(name, path):
    m = types.ModuleType(name)
    m.__path__ = [path]
    sys.modules[name] = m
    return m


def _mod(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


def load_reference():
    xr = types.ModuleType("xarray")
    core = types.ModuleType("xarray.core")
    dt = types.ModuleType("xarray.core.datatree")
    dt.DataTree = _DataTree
    core.datatree = dt
    xr.core = core
    xr.DataArray = _DataArray
    xr.DataTree = _DataTree
    sys.modules.update({"xarray": xr, "xarray.core": core, "xarray.core.datatree": dt})
    ap = types.ModuleType("astropy")
    apc = types.ModuleType("astropy.constants")
    apc.c = types.SimpleNamespace(value=299792458.0)
    ap.constants = apc
    sys.modules.update({"astropy": ap, "astropy.constants": apc})
    _pkg("astroviper", SRC)
    _pkg("astroviper.core", SRC + "/core")
    _pkg("astroviper.core.imaging", SRC + "/core/imaging")
    _pkg("astroviper.core.imaging.imaging_utils", SRC + "/core/imaging/imaging_utils")
    _pkg("astroviper.core.imaging.imaging_weighting", SRC + "/core/imaging/imaging_weighting")
    iu = SRC + "/core/imaging/imaging_utils/"
    iw = SRC + "/core/imaging/imaging_weighting/"
    ns = types.SimpleNamespace()
    ns.gcf = _mod("astroviper.core.imaging.imaging_utils.gcf_prolate_spheroidal",
                  iu + "gcf_prolate_spheroidal.py")
    ns.sg = _mod("astroviper.core.imaging.imaging_utils.standard_grid", iu + "standard_grid.py")
    ns.sd = _mod("astroviper.core.imaging.imaging_utils.standard_degrid",
                 iu + "standard_degrid.py")
    ns.giw = _mod("astroviper.core.imaging.imaging_weighting.grid_imaging_weights",
                  iw + "grid_imaging_weights.py")
    ns.bw = _mod("astroviper.core.imaging.imaging_weighting.briggs_weighting",
                 iw + "briggs_weighting.py")
    ns.fft = _mod("astroviper.core.imaging.fft", SRC + "/core/imaging/fft.py")
    ns.ifft = _mod("astroviper.core.imaging.ifft", SRC + "/core/imaging/ifft.py")
    so = glob.glob(os.path.join(REPO, "oracle", "_ref", "_hogbom_ext*.so"))
    if not so:
        raise SystemExit("build the reference Hogbom module first: sh oracle/build_ref.sh")
    spec = importlib.util.spec_from_file_location("_hogbom_ext", so[0])
    ns.hog = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ns.hog)
    return ns


class _Coord:
    def __init__(self, v):
        self.values = v
        self.data = v


class MS4Double(_DataTree):
    """Duck-typed MSv4 node for grid2image_spheroid_ms4 (standard_grid.py:657-670)."""

    def __init__(self, vis, uvw, weight, flag, freq):
        self._d = {"VISIBILITY": _Coord(vis)}
        self.UVW = _Coord(uvw)
        self.WEIGHT = _Coord(weight)
        self.FLAG = _Coord(flag)
        self.coords = {"frequency": _Coord(freq)}

    def __getitem__(self, k):
        return self._d[k]


def _edge_case_inputs(rng, nt, n_ant, nchan, npol, cell, freq, extent=1.2):
    """uvw / vis / weight with NaN rows, NaN and zero samples, zero weights
    and samples beyond the grid edge."""
    from astroviper_b200 import synthetic as S
    uvw, _ = S.array_uvw(n_ant, nt, radius_m=600.0, seed=int(rng.integers(1 << 30)))
    nb = uvw.shape[1]
    # stretch a few baselines beyond the grid edge
    uvw[:, -2:, :2] *= 40.0 * extent
    uvw[1, 2, 0] = np.nan
    uvw[2, 3, 1] = np.nan
    shape = (nt, nb, nchan, npol)
    vis = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    vis[0, 1, 0, 0] = np.nan + 0j
    vis[0, 2, 0, npol - 1] = complex(0.0, np.nan)
    vis[1, 1, :, :] = 0.0
    vis[3, 4, 1, 0] = complex(0.0, 1.5)
    weight = rng.uniform(0.5, 2.0, size=shape)
    weight[2, 1, :, 0] = 0.0
    weight[0, 5, nchan - 1, npol - 1] = np.nan
    return uvw, vis, weight


def make_pswf(R):
    out = {}
    for os_, sup in [(100, 7), (64, 9), (100, 8), (50, 5), (128, 6)]:
        out[f"cgk_{os_}_{sup}"] = R.gcf.create_prolate_spheroidal_kernel_1D(os_, sup)
    for n in [(64, 64), (96, 128), (101, 77)]:
        _, ct = R.gcf.create_prolate_spheroidal_kernel(100, 7, np.array(n))
        out[f"corr_{n[0]}_{n[1]}"] = ct
    u = np.concatenate([np.linspace(-1.2, 1.2, 241), [0.75, 1.0, -0.75, 1.0 + 1e-12]])
    g, k = R.gcf.prolate_spheroidal_function(u)
    out.update(u=u, grdsf=g, kern=k)
    np.savez_compressed(os.path.join(HERE, "pswf.npz"), **out)


def make_grid(R):
    rng = np.random.default_rng(1001)
    cases = {}
    specs = [
        # name, nt, n_ant, nchan, npol, (nu, nv), support, oversampling
        ("a", 5, 7, 3, 2, (48, 64), 7, 100),
        ("b", 4, 6, 2, 1, (40, 40), 9, 64),
        ("c", 4, 6, 2, 4, (36, 44), 8, 100),
    ]
    for name, nt, na, nchan, npol, (nu, nv), sup, os_ in specs:
        freq = np.linspace(1.2e9, 1.6e9, nchan)
        cell = np.array([-25.0, 25.0]) * np.pi / (180 * 3600)
        uvw, vis, weight = _edge_case_inputs(rng, nt, na, nchan, npol, cell, freq)
        cgk = R.gcf.create_prolate_spheroidal_kernel_1D(os_, sup)
        d = dict(uvw=uvw, vis=vis, weight=weight, freq=freq, cell=cell,
                 image_size=np.array([nu, nv]), support=sup, oversampling=os_, cgk=cgk)
        for do_psf in (False, True):
            for mode in ("continuum", "cube"):
                g, s = R.sg.standard_grid_numpy_wrap_input_checked(
                    vis, np.array([]), np.array([]), uvw, weight, freq, cgk,
                    np.array([nu, nv]), cell, os_, sup, True, do_psf, mode)
                key = f"{'psf' if do_psf else 'vis'}_{mode}"
                d["grid_" + key] = g
                d["sumwt_" + key] = s
        # accumulate into an existing grid (standard_grid.py:133 takes the
        # given arrays when they are not empty)
        g0 = rng.normal(size=d["grid_vis_continuum"].shape) + 0j
        s0 = rng.uniform(size=d["sumwt_vis_continuum"].shape)
        g, s = R.sg.standard_grid_numpy_wrap_input_checked(
            vis, g0.copy(), s0.copy(), uvw, weight, freq, cgk, np.array([nu, nv]), cell, os_,
            sup, True, False, "continuum")
        d.update(acc_grid0=g0, acc_sumwt0=s0, acc_grid=g, acc_sumwt=s)
        if npol >= 2:
            # the do_imaging_weight branch of standard_grid_jit (conjugate
            # gridding of pol-averaged weights), called directly
            gg = np.zeros((1, npol, nu, nv), dtype=np.complex128)
            ss = np.zeros((1, npol))
            w2 = np.nan_to_num(weight, nan=0.0)
            R.sg.standard_grid_jit(gg, ss, True, True, np.zeros((1, 1, 1, 1), dtype=np.complex128),
                                   uvw, freq, np.zeros(nchan, dtype=np.int64),
                                   np.arange(npol, dtype=np.int64), w2, cgk, np.array([nu, nv]),
                                   cell, sup, os_)
            d.update(iw_weight=w2, iw_grid=gg, iw_sumwt=ss)
        cases[name] = d
        np.savez_compressed(os.path.join(HERE, f"grid_{name}.npz"), **d)


def make_image(R):
    """grid2image_spheroid_ms4 (standard_grid.py:607-708) through a duck-typed
    MSv4 node, for the dirty image and the PSF, continuum and cube."""
    rng = np.random.default_rng(2002)
    from astroviper_b200 import synthetic as S
    uvw, _ = S.array_uvw(12, 6, radius_m=500.0, seed=77)
    freq = np.array([1.3e9, 1.4e9])
    nt, nb = uvw.shape[:2]
    vis = rng.normal(size=(nt, nb, 2, 2)) + 1j * rng.normal(size=(nt, nb, 2, 2))
    weight = rng.uniform(0.5, 1.5, size=vis.shape)
    flag = rng.uniform(size=vis.shape) < 0.1
    uvw[2, 5, 0] = np.nan
    cell = np.array([-30.0, 30.0]) * np.pi / (180 * 3600)
    out = dict(uvw=uvw, freq=freq, vis=vis, weight=weight, flag=flag, cell=cell)
    for dopsf in (False, True):
        for mode, nci in (("continuum", 1), ("cube", 2)):
            w = weight.copy()
            ms = MS4Double(vis.copy(), uvw.copy(), w, flag.copy(), freq)
            img = np.zeros((nci, 2, 64, 64))
            R.sg.grid2image_spheroid_ms4(ms, img, cell, 7, 100, dopsf, "VISIBILITY", mode)
            out[f"img_{'psf' if dopsf else 'vis'}_{mode}"] = img
            out[f"weight_after_{'psf' if dopsf else 'vis'}_{mode}"] = w
    # the reference's FFT helpers (fft.py:5, ifft.py:5)
    a = rng.normal(size=(2, 3, 32, 30))
    out["fft_in"] = a
    out["fft_out"] = R.fft.fft_lm_to_uv(a, axes=[2, 3])
    out["ifft_out"] = R.ifft.ifft_uv_to_lm(out["fft_out"], axes=[2, 3])
    np.savez_compressed(os.path.join(HERE, "image.npz"), **out)


def make_psf_planes(R):
    """The PSF planes make_psf (make_point_spread_function.py:41-53) computes
    before xradio wraps them: grid2image_spheroid_ms4 with dopsf=True and
    pixel increment [-cell0, cell1] into a zero array of shape
    (n_freq, n_pol, image_size[1], image_size[0]).  xradio is absent here, so
    the function itself cannot run; its call is made exactly as it makes it.
    Non-square sizes show the transposed array shape."""
    rng = np.random.default_rng(2112)
    from astroviper_b200 import synthetic as S
    uvw, _ = S.array_uvw(12, 6, radius_m=500.0, seed=78)
    freq = np.array([1.3e9, 1.4e9])
    nt, nb = uvw.shape[:2]
    vis = rng.normal(size=(nt, nb, 2, 2)) + 1j * rng.normal(size=(nt, nb, 2, 2))
    weight = rng.uniform(0.5, 1.5, size=vis.shape)
    flag = rng.uniform(size=vis.shape) < 0.1
    uvw[3, 4, 1] = np.nan
    cell = np.array([25.0, 30.0]) * np.pi / (180 * 3600)
    out = dict(uvw=uvw, freq=freq, vis=vis, weight=weight, flag=flag, cell=cell)
    for mode, nch, image_size in (("cube", 2, (64, 48)), ("continuum", 1, (48, 64))):
        w = weight[:, :, :nch].copy()
        ms = MS4Double(vis[:, :, :nch].copy(), uvw.copy(), w, flag[:, :, :nch].copy(), freq[:nch])
        psf = np.zeros([nch, 2, image_size[1], image_size[0]], dtype=float)
        R.sg.grid2image_spheroid_ms4(ms, psf, np.array([-cell[0], cell[1]]), 7, 100, True,
                                     "VISIBILITY", mode)
        out[f"psf_{mode}"] = psf
        out[f"image_size_{mode}"] = np.array(image_size)
        out[f"weight_after_{mode}"] = w
    np.savez_compressed(os.path.join(HERE, "psf_dropin.npz"), **out)


def make_degrid(R):
    rng = np.random.default_rng(3003)
    from astroviper_b200 import synthetic as S
    uvw, _ = S.array_uvw(10, 5, radius_m=800.0, seed=99)
    uvw[:, -1, :2] *= 30.0  # off-grid
    nt, nb = uvw.shape[:2]
    freq = np.array([1.1e9, 1.25e9, 1.4e9])
    nvpol = 4
    grid = (rng.normal(size=(2, 2, 64, 64)) + 1j * rng.normal(size=(2, 2, 64, 64)))
    cell = np.array([-20.0, 20.0]) * np.pi / (180 * 3600)
    nx, ny = 64, 64
    scale = np.array([-cell[0] * nx, -cell[1] * ny, 0.0])
    offset = np.array([nx / 2, ny / 2, 0.0])
    flag = rng.uniform(size=(nt, nb, 3, nvpol)) < 0.15
    dphase = rng.uniform(-0.3, 0.3, size=(nt, nb))
    chanmap = (np.arange(3) / 3 * 2).astype(int)
    polmap = np.round(np.arange(nvpol) % 2).astype(int)
    out = dict(uvw=uvw, freq=freq, grid=grid, cell=cell, scale=scale, offset=offset,
               flag=flag, dphase=dphase, chanmap=chanmap, polmap=polmap)
    for sup, os_ in ((7, 100), (9, 64), (8, 100)):
        cf = R.gcf.create_prolate_spheroidal_kernel_1D(os_, sup)
        for dp_name, dp in (("zero", np.zeros((nt, nb))), ("phase", dphase)):
            v0 = np.zeros((nt, nb, 3, nvpol), dtype=complex)
            if (sup, os_, dp_name) == (7, 100, "zero"):
                # values += (standard_degrid.py:483): start from non-zero values once
                v0 = rng.normal(size=v0.shape) + 1j * rng.normal(size=v0.shape)
            v = v0.copy()
            R.sd.dgrid_numba(uvw, dp, v, flag, scale, offset, grid, freq, 299792458.0, sup, os_,
                             cf, chanmap, polmap)
            out[f"v0_{sup}_{os_}_{dp_name}"] = v0
            out[f"v_{sup}_{os_}_{dp_name}"] = v
    # the reference's own known answer: a 2 Jy centre source degrids to
    # |vis| = 2 everywhere (test_standard_degrid.py:122-240), seeded here
    npix = 200
    maxuv = 2e3
    c = 299792458.0
    cellk = 0.5 * c / 1.4e9 / maxuv
    mod = np.zeros((npix, npix))
    mod[100, 100] = 2.0
    gk = np.zeros((1, 1, npix, npix), dtype=complex)
    gk[0, 0] = np.conj(R.fft.fft_lm_to_uv(mod, axes=[0, 1]))
    uvk = np.zeros((1, 64 * 64, 3))
    uvk[0, :, 0] = rng.uniform(-maxuv, maxuv, 64 * 64)
    uvk[0, :, 1] = rng.uniform(-maxuv, maxuv, 64 * 64)
    vk = np.zeros((1, 64 * 64, 1, 1), dtype=complex)
    R.sd.dgrid_numba(uvk, np.zeros((1, 64 * 64)), vk, np.zeros(vk.shape, bool),
                     np.array([cellk, cellk]), np.array([npix // 2, npix // 2]), gk,
                     np.array([1.4e9]), c, 7, 100,
                     R.gcf.create_prolate_spheroidal_kernel_1D(100, 7), np.zeros(1, int),
                     np.zeros(1, int))
    out.update(kat_uvw=uvk, kat_cell=np.array([cellk, cellk]), kat_vis=vk)
    np.savez_compressed(os.path.join(HERE, "degrid.npz"), **out)


def make_weights(R):
    rng = np.random.default_rng(4004)
    from astroviper_b200 import synthetic as S
    out = {}
    for npol in (1, 2, 4):
        uvw, _ = S.array_uvw(9, 6, radius_m=700.0, seed=10 + npol)
        uvw[:, -1, :2] *= 50.0
        uvw[3, 2, 0] = np.nan
        nt, nb = uvw.shape[:2]
        freq = np.array([1.2e9, 1.5e9])
        w = rng.uniform(0.2, 3.0, size=(nt, nb, 2, npol))
        flag = rng.uniform(size=w.shape) < 0.1
        cell = np.array([-15.0, 15.0]) * np.pi / (180 * 3600)
        n = np.array([64, 48])
        wd = w.copy()
        wd[flag] = np.nan
        if npol == 2:
            wd = ((wd[..., 0] + wd[..., 1]) / 2)[..., None]
        if npol == 4:
            wd = ((wd[..., 0] + wd[..., 3]) / 2)[..., None]
        G = np.zeros((2, 1, n[0], n[1]))
        sw = np.zeros((2, 1))
        R.giw.grid_imaging_weights(G, sw, uvw, wd, freq, {"image_size": n, "cell_size": cell})
        d = dict(uvw=uvw, freq=freq, w=w, flag=flag, cell=cell, n=n, wd=wd, G=G, sw=sw)
        for robust in (-1.0, 0.5, 2.0):
            bf = R.bw.calculate_briggs_params(G, sw, {"weighting": "briggs", "robust": robust})
            iw = R.giw.degrid_imaging_weights(G, uvw, wd, bf, freq, {"image_size": n,
                                                                    "cell_size": cell})
            d[f"bf_{robust}"] = bf
            d[f"iw_{robust}"] = np.tile(iw, (1, 1, 1, npol))
        d["bf_abs"] = R.bw.calculate_briggs_params(
            G, sw, {"weighting": "briggs_abs", "robust": 0.7, "briggs_abs_noise": 0.3})
        d["bf_nat"] = R.bw.calculate_briggs_params(G, sw, {"weighting": "natural"})
        for k, v in d.items():
            out[f"p{npol}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "weights.npz"), **out)


def make_iw_degrid(R):
    """standard_imaging_weight_degrid_numpy_wrap (standard_grid.py:441-484) and
    standard_imaging_weight_degrid_jit (:487-604) with permuted maps into a
    prefilled array: NaN / zero natural weights, NaN / zero grid cells, NaN
    uv, samples off the grid and one just below index 0 (int() truncation)."""
    rng = np.random.default_rng(6006)
    from astroviper_b200 import synthetic as S
    out = {}
    c = 299792458.0
    for npol in (1, 2, 4):
        uvw, _ = S.array_uvw(9, 6, radius_m=700.0, seed=20 + npol)
        nt, nb = uvw.shape[:2]
        uvw[:, -1, :2] *= 50.0
        uvw[3, 2, 0] = np.nan
        freq = np.array([1.2e9, 1.35e9, 1.5e9])
        nchan = len(freq)
        cell = np.array([-15.0, 15.0]) * np.pi / (180 * 3600)
        n = np.array([40, 32])
        # sample (4, 1) at channel 0 lands at u_pos = -0.7: int(-0.2) = 0 is kept
        us0 = -(freq[0] * cell[0] * n[0]) / c
        uvw[4, 1, 0] = (-0.7 - n[0] // 2) / us0
        nat = rng.uniform(0.2, 3.0, size=(nt, nb, nchan, npol))
        nat[rng.uniform(size=nat.shape) < 0.08] = 0.0
        nat[rng.uniform(size=nat.shape) < 0.05] = np.nan
        G = 0.5 * rng.integers(1, 9, size=(nchan, npol, n[0], n[1]))  # compresses
        G[rng.uniform(size=G.shape) < 0.15] = 0.0
        G[rng.uniform(size=G.shape) < 0.05] = np.nan
        bf = np.stack([rng.uniform(0.1, 2.0, size=(nchan, npol)),
                       rng.uniform(0.5, 1.5, size=(nchan, npol))])
        params = {"image_size_padded": n, "cell_size": cell}
        iw = R.sg.standard_imaging_weight_degrid_numpy_wrap(G, uvw, nat, bf, freq, params)
        Gf = G.astype(np.float32)
        iw32 = R.sg.standard_imaging_weight_degrid_numpy_wrap(Gf, uvw, nat, bf, freq, params)
        cm = np.array([2, 0, 1])
        pm = np.arange(npol)[::-1].copy()
        jit = np.full(nat.shape, -7.0)
        R.sg.standard_imaging_weight_degrid_jit(jit, G, bf, uvw, freq, cm, pm, nat, n, cell)
        d = dict(uvw=uvw, freq=freq, nat=nat, G=G, bf=bf, cell=cell, n=n, iw=iw, iw32=iw32,
                 cm=cm, pm=pm, jit=jit)
        for k, v in d.items():
            out[f"p{npol}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "iw_degrid.npz"), **out)


def make_hogbom(R):
    from astroviper_b200 import synthetic as S
    cw = S.clean_workload(nx=64, psf_factor=2, n_src=12, n_time=12, seed=5005)
    dirty = cw["dirty"]
    psf2 = cw["psf"]
    psf = psf2[32:96, 32:96].copy()
    rng = np.random.default_rng(5005)
    mask = (rng.uniform(size=dirty.shape) > 0.25).astype(np.float32)
    out = dict(dirty=dirty, psf=psf, psf2=psf2, mask=mask)
    runs = {
        "default": dict(max_iter=100),
        "box_thr": dict(max_iter=400, gain=0.2, threshold=0.02, clean_box=(5, 50, 10, 60)),
        "mask_speed": dict(max_iter=150, start_iter=3, speedup=40.0, threshold=0.005,
                           mask=mask),
        "long": dict(max_iter=1000, gain=0.05),
    }
    for dt in (np.float32, np.float64):
        tag = "f32" if dt == np.float32 else "f64"
        for name, kw in runs.items():
            kw = dict(kw)
            if "mask" in kw:
                kw["mask"] = kw["mask"].astype(dt)
            r = R.hog.clean(dirty.astype(dt), psf.astype(dt), **kw)
            for k in ("model_image", "residual_image", "iterations_performed", "final_peak",
                      "total_flux_cleaned", "converged"):
                out[f"{tag}_{name}_{k}"] = np.asarray(r[k])
        out[f"{tag}_maximg"] = np.asarray(R.hog.maximg(dirty.astype(dt)))
        out[f"{tag}_maximg_mask"] = np.asarray(R.hog.maximg(dirty.astype(dt), mask.astype(dt)))
    np.savez_compressed(os.path.join(HERE, "hogbom.npz"), **out)


MAKERS = {"pswf": make_pswf, "grid": make_grid, "image": make_image,
          "psf_dropin": make_psf_planes, "degrid": make_degrid, "weights": make_weights,
          "hogbom": make_hogbom, "iw_degrid": make_iw_degrid}


def main(names=None):
    """Writes every fixture, or only the named ones
    (``python tests/golden/make_golden.py psf_dropin``)."""
    R = load_reference()
    for name in (names or list(MAKERS)):
        MAKERS[name](R)
    for f in sorted(glob.glob(os.path.join(HERE, "*.npz"))):
        print(os.path.basename(f), os.path.getsize(f))


if __name__ == "__main__":
    main(sys.argv[1:])
