"""Generates image_prep.npz in this folder from the reference itself.

Run in a container that has the astroviper source tree (default
``reference/`` beside this repository, override with ``AV_REFERENCE_ROOT``):

    python tests/golden/make_golden_image_prep.py

Runs the reference's remove_padding, apply_pb, fft_to_uv, ifft_to_lm,
correct_fft_to_uv, correct_ifft_to_lm and grid2xradio_spheroid_ms4
(standard_image_grid_preparation.py:99-580), imported unmodified, on a small
dataset stand-in (the xarray surface those functions use: sizes, data_vars,
item get / set, .data, in-place *= and /=, ==, coords, .sel and .isel
returning views), with stand-in modules for xarray and xradio;
grid2xradio_spheroid_ms4 grids duck-typed MSv4 nodes with the reference's
own Numba gridder.  The inputs and the outputs go into image_prep.npz, keyed
<case>/<variable>/{in,out}.
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
sys.path.insert(0, HERE)

from make_golden import MS4Double, _DataArray, _DataTree, _mod, _pkg  # noqa: E402

IMAGE_DIMS = ("time", "frequency", "polarization", "l", "m")
UV_DIMS = ("time", "frequency", "polarization", "u", "v")


class _Coord:
    def __init__(self, v):
        self.values = np.asarray(v)


class _DA:
    """A data variable: .data (a numpy buffer), .dims, .coords, in-place *=
    on the buffer, and .sel by coordinate value returning a view."""

    def __init__(self, data, dims, coords):
        self._data = data
        self.dims = tuple(dims)
        self.coords = {d: _Coord(coords[d]) for d in self.dims if d in coords}

    @property
    def data(self):
        return self._data

    @data.setter
    def data(self, v):
        if v.shape != self._data.shape:
            raise ValueError("shape change")
        self._data = v

    @property
    def shape(self):
        return self._data.shape

    def __array__(self, dtype=None, copy=None):
        return self._data

    def _raw(self, k):
        return k._data if isinstance(k, _DA) else k

    def __imul__(self, k):
        self._data *= self._raw(k)
        return self

    def __itruediv__(self, k):
        self._data /= self._raw(k)
        return self

    def __eq__(self, k):
        return self._data == self._raw(k)

    def __getitem__(self, idx):
        return _DA(self._data[idx], self.dims[-self._data[idx].ndim:] if self._data[idx].ndim
                   else (), {})

    def __setitem__(self, idx, value):
        self._data[idx] = self._raw(value)

    def sel(self, **kw):
        idx = []
        for d in self.dims:
            if d in kw:
                idx.append(int(np.flatnonzero(self.coords[d].values == kw[d])[0]))
            else:
                idx.append(slice(None))
        rest = [d for d in self.dims if d not in kw]
        return _DA(self._data[tuple(idx) + (Ellipsis,)], rest, {})


class _DS:
    def __init__(self, variables, coords):
        self.coords = coords
        self.data_vars = {}
        for name, (dims, data) in variables.items():
            self.data_vars[name] = _DA(data, dims, coords)

    @property
    def sizes(self):
        out = {}
        for v in self.data_vars.values():
            out.update(zip(v.dims, v.data.shape))
        return out

    def __getitem__(self, name):
        return self.data_vars[name]

    def __contains__(self, name):
        return name in self.data_vars or name in self.coords

    def isel(self, **kw):
        out = _DS({}, {})
        for n, v in self.data_vars.items():
            idx = tuple(kw.get(d, slice(None)) for d in v.dims)
            out.data_vars[n] = _DA(v.data[idx], v.dims, {})
        return out

    def __setitem__(self, name, value):
        self.data_vars[name] = value

    def __getattr__(self, name):
        coords = self.__dict__.get("coords", {})
        if name in coords:
            return _DA(np.asarray(coords[name]), (name,), {})
        raise AttributeError(name)

    def __repr__(self):
        return "<image>"


def load_reference():
    xr = types.ModuleType("xarray")
    core = types.ModuleType("xarray.core")
    dt = types.ModuleType("xarray.core.datatree")
    dt.DataTree = _DataTree
    core.datatree = dt
    xr.core = core
    xr.DataArray = _DataArray
    xr.DataTree = _DataTree
    xr.Dataset = _DS
    sys.modules.update({"xarray": xr, "xarray.core": core, "xarray.core.datatree": dt})
    xd = types.ModuleType("xradio")
    xdi = types.ModuleType("xradio.image")
    xdii = types.ModuleType("xradio.image.image")
    xdii.make_empty_lmuv_image = xdii.make_empty_sky_image = None
    sys.modules.update({"xradio": xd, "xradio.image": xdi, "xradio.image.image": xdii})
    _pkg("astroviper", SRC)
    _pkg("astroviper.core", SRC + "/core")
    _pkg("astroviper.core.imaging", SRC + "/core/imaging")
    _pkg("astroviper.core.imaging.imaging_utils", SRC + "/core/imaging/imaging_utils")
    iu = SRC + "/core/imaging/imaging_utils/"
    _mod("astroviper.core.imaging.imaging_utils.standard_grid", iu + "standard_grid.py")
    _mod("astroviper.core.imaging.fft", SRC + "/core/imaging/fft.py")
    _mod("astroviper.core.imaging.ifft", SRC + "/core/imaging/ifft.py")
    _mod("astroviper.core.imaging.imaging_utils.gcf_prolate_spheroidal",
         iu + "gcf_prolate_spheroidal.py")
    return _mod("astroviper.core.imaging.imaging_utils.standard_image_grid_preparation",
                iu + "standard_image_grid_preparation.py")


def _coords(shape):
    return {"time": np.arange(shape[0]) * 10.0 + 5.0,
            "frequency": 1.0e9 + np.arange(shape[1]) * 1.0e6,
            "polarization": np.array(["XX", "XY", "YX", "YY"][:shape[2]])}


def _cplx(rng, shape, dtype):
    x = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(dtype)
    flat = x.reshape(-1)
    ft = flat.real.dtype
    specials = [(-0.0, 1.0), (1.0, -0.0), (-0.0, -0.0), (np.inf, 1.0), (1.0, -np.inf),
                (np.nan, 2.0), (3.0e-39 if ft == np.float32 else 3.0e-310, -1.0)]
    for k, (a, b) in enumerate(specials):
        flat.real[k * 7] = a
        flat.imag[k * 7] = b
    return x


def run(ref):
    rng = np.random.default_rng(20261203)
    out = {}

    def record(case, ds, names_in, call):
        for n in names_in:
            out[f"{case}/{n}/in"] = ds[n].data.copy()
        call(ds)
        for n, v in ds.data_vars.items():
            out[f"{case}/{n}/out"] = v.data.copy()

    # correct_fft_to_uv on complex grids, u x v = 12 x 10 (not a power of 2)
    for tag, dt in (("c128", np.complex128), ("c64", np.complex64)):
        shp = (2, 2, 2, 12, 10)
        ds = _DS({"VISIBILITY": (UV_DIMS, _cplx(rng, shp, dt)),
                  "VISIBILITY_RESIDUAL": (UV_DIMS, _cplx(rng, shp, dt)),
                  "OTHER": (UV_DIMS, _cplx(rng, shp, dt))}, _coords(shp))
        record(f"cfu_{tag}", ds, list(ds.data_vars), lambda d: ref.correct_fft_to_uv(d))
        ds = _DS({"VISIBILITY_MODEL": (UV_DIMS, _cplx(rng, shp, dt))}, _coords(shp))
        record(f"cfu_named_{tag}", ds, list(ds.data_vars),
               lambda d: ref.correct_fft_to_uv(d, "VISIBILITY_MODEL"))

    # correct_ifft_to_lm without the spheroid correction: real and complex
    for tag, dt in (("f64", np.float64), ("f32", np.float32)):
        shp = (2, 3, 2, 14, 10)
        sky = rng.normal(size=shp).astype(dt)
        sky.reshape(-1)[:4] = [-0.0, np.inf, np.nan, 1e-39 if dt == np.float32 else 1e-310]
        ds = _DS({"SKY": (IMAGE_DIMS, sky),
                  "RESIDUAL": (IMAGE_DIMS, rng.normal(size=shp).astype(dt)),
                  "MODEL": (IMAGE_DIMS, rng.normal(size=shp).astype(dt))}, _coords(shp))
        record(f"cil_{tag}", ds, list(ds.data_vars), lambda d: ref.correct_ifft_to_lm(d))
    shp = (1, 2, 2, 9, 11)
    ds = _DS({"RESIDUAL": (IMAGE_DIMS, _cplx(rng, shp, np.complex64))}, _coords(shp))
    record("cil_c64", ds, list(ds.data_vars), lambda d: ref.correct_ifft_to_lm(d, ["RESIDUAL"]))

    # correct_ifft_to_lm with the spheroid correction (default 100 / 7 kernel)
    shp = (2, 2, 2, 16, 12)
    ds = _DS({"SKY": (IMAGE_DIMS, rng.normal(size=shp)),
              "RESIDUAL": (IMAGE_DIMS, rng.normal(size=shp).astype(np.float32)),
              "VISIBILITY_NORMALIZATION": (IMAGE_DIMS[:3], rng.uniform(10, 1e4, shp[:3])),
              "VISIBILITY_RESIDUAL_NORMALIZATION":
                  (IMAGE_DIMS[:3], rng.uniform(10, 1e4, shp[:3]).astype(np.float32))},
             _coords(shp))
    record("cil_sph", ds, list(ds.data_vars),
           lambda d: ref.correct_ifft_to_lm(d, doSpheroidCorr=True))
    shp = (1, 3, 1, 20, 20)
    ds = _DS({"RESIDUAL": (IMAGE_DIMS, rng.normal(size=shp)),
              "VISIBILITY_RESIDUAL_NORMALIZATION": (IMAGE_DIMS[:3], rng.uniform(1, 9, shp[:3]))},
             _coords(shp))
    record("cil_sph_named", ds, list(ds.data_vars),
           lambda d: ref.correct_ifft_to_lm(d, "RESIDUAL", True, 64, 9))
    out["cil_sph_named/corr"] = sys.modules[
        "astroviper.core.imaging.imaging_utils.gcf_prolate_spheroidal"
    ].create_prolate_spheroidal_kernel(64, 9, np.array([20, 20]))[1]

    # the transforms
    shp = (1, 2, 2, 16, 12)
    ds = _DS({"SKY": (IMAGE_DIMS, rng.normal(size=shp)),
              "MODEL": (IMAGE_DIMS, rng.normal(size=shp)),
              "VISIBILITY_SKY": (UV_DIMS, np.zeros(shp, complex)),
              "VISIBILITY_MODEL": (UV_DIMS, np.zeros(shp, complex))}, _coords(shp))
    record("fft", ds, ["SKY", "MODEL"], lambda d: ref.fft_to_uv(d))
    ds = _DS({"VISIBILITY": (UV_DIMS, _cplx(rng, shp, np.complex128)),
              "VISIBILITY_RESIDUAL": (UV_DIMS, _cplx(rng, shp, np.complex128)),
              "SKY": (IMAGE_DIMS, np.zeros(shp)),
              "RESIDUAL": (IMAGE_DIMS, np.zeros(shp))}, _coords(shp))
    for n in ("VISIBILITY", "VISIBILITY_RESIDUAL"):
        ds[n].data[~np.isfinite(ds[n].data)] = 0.5
    record("ifft", ds, ["VISIBILITY", "VISIBILITY_RESIDUAL"], lambda d: ref.ifft_to_lm(d))

    # apply_pb: equal shapes and planes broadcast from index 0, multiply and
    # divide (NaN where the beam is 0), real and complex images
    shp = (2, 3, 2, 10, 8)

    def beam(shape, dtype):
        b = rng.uniform(0.0, 1.0, shape).astype(dtype)
        b.reshape(-1)[::9] = 0.0
        b.reshape(-1)[4::23] = -0.0
        return b

    for tag, pshape, dt, pdt in (("eq_f64", shp, np.float64, np.float64),
                                 ("eq_f32_pb64", shp, np.float32, np.float64),
                                 ("bc_f64", (1, 3, 1, 10, 8), np.float64, np.float64),
                                 ("bc_f32", (1, 1, 1, 10, 8), np.float32, np.float32),
                                 ("bc_mixed", (2, 2, 2, 10, 8), np.float64, np.float32),
                                 ("eq_c64", shp, np.complex64, np.float32),
                                 ("bc_c128_pb32", (1, 3, 2, 10, 8), np.complex128, np.float32),
                                 ("bc_c64_pb64", (2, 1, 1, 10, 8), np.complex64, np.float64)):
        for mult in (True, False):
            if np.dtype(dt).kind == "c":
                sky = _cplx(rng, shp, dt)
            else:
                sky = rng.normal(size=shp).astype(dt)
                sky.reshape(-1)[:3] = [-0.0, np.inf, np.nan]
            ds = _DS({"SKY": (IMAGE_DIMS, sky),
                      "MODEL": (IMAGE_DIMS, rng.normal(size=shp).astype(dt)),
                      "PRIMARY_BEAM": (IMAGE_DIMS, beam(pshape, pdt))}, _coords(shp))
            record(f"pb_{tag}_{'mul' if mult else 'div'}", ds, list(ds.data_vars),
                   lambda d: ref.apply_pb(d, multiply=mult))
    ds = _DS({"RESIDUAL": (IMAGE_DIMS, rng.normal(size=shp))}, _coords(shp))
    pbds = _DS({"PRIMARY_BEAM": (IMAGE_DIMS, beam(shp, np.float64))}, _coords(shp))
    out["pb_separate_div/PRIMARY_BEAM/in"] = pbds["PRIMARY_BEAM"].data.copy()
    record("pb_separate_div", ds, ["RESIDUAL"],
           lambda d: ref.apply_pb(d, pbds, False, "RESIDUAL"))

    # remove_padding: the centre of odd and even padded sizes
    for tag, (pl, pm), size in (("even", (16, 12), (10, 7)), ("odd", (15, 13), (8, 9))):
        shp = (1, 2, 1, pl, pm)
        ds = _DS({"SKY": (IMAGE_DIMS, rng.normal(size=shp))}, _coords(shp))
        out[f"pad_{tag}/SKY/in"] = ds["SKY"].data.copy()
        out[f"pad_{tag}/size"] = np.array(size)
        out[f"pad_{tag}/SKY/out"] = ref.remove_padding(ds, np.array(size))["SKY"].data.copy()

    # grid2xradio_spheroid_ms4: two MSv4 nodes into two time planes, the
    # visibilities in continuum mode and the weights (UV_SAMPLING) as a cube
    for tag, data_var, chan_mode in (("vis", "VISIBILITY", "continuum"),
                                     ("psf", "UV_SAMPLING", "cube")):
        nodes = []
        nchan, npol, nt, nb = 3, 2, 4, 15
        freq = 1.0e9 + np.arange(nchan) * 2.0e7
        for k in range(2):
            uvw = rng.uniform(-900.0, 900.0, (nt, nb, 3))
            shape = (nt, nb, nchan, npol)
            vis = rng.normal(size=shape) + 1j * rng.normal(size=shape)
            weight = rng.uniform(0.5, 2.0, (nt, nb, nchan, npol))
            flag = rng.uniform(size=(nt, nb, nchan, npol)) < 0.1
            node = MS4Double(vis, uvw, weight, flag, freq)
            node._d["UV_SAMPLING"] = node._d["VISIBILITY"]
            nodes.append(node)
            for n, a in (("vis", vis), ("uvw", uvw), ("weight", weight), ("flag", flag)):
                out[f"ms4_{tag}/node{k}/{n}"] = a.copy()
            out[f"ms4_{tag}/freq"] = freq
        n_img_chan = nchan if chan_mode == "cube" else 1
        shp = (2, n_img_chan, npol, 64, 48)
        coords = _coords(shp)
        coords["l"] = (np.arange(64) - 32) * -2.0e-5
        coords["m"] = (np.arange(48) - 24) * 2.4e-5
        ds = _DS({data_var: (UV_DIMS, np.zeros(shp, complex)),
                  data_var + "_NORMALIZATION": (UV_DIMS[:3], np.zeros(shp[:3]))}, coords)
        ref.grid2xradio_spheroid_ms4(nodes, ds, data_var=data_var, chan_mode=chan_mode)
        out[f"ms4_{tag}/grid"] = ds[data_var].data.copy()
        out[f"ms4_{tag}/sumwt"] = ds[data_var + "_NORMALIZATION"].data.copy()
        for k, node in enumerate(nodes):
            out[f"ms4_{tag}/node{k}/weight_after"] = node.WEIGHT.data.copy()

    np.savez_compressed(os.path.join(HERE, "image_prep.npz"), **out)
    return out


if __name__ == "__main__":
    with np.errstate(all="ignore"):
        run(load_reference())
