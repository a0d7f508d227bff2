"""A minimal sky-image dataset for the imager and deconvolve.

The reference builds its images with xradio's make_empty_sky_image (an
xarray Dataset with dims (time, frequency, polarization, l, m)) and reads
them through .sizes, ds[name].values, .coords[name].values, .copy(deep=True)
and .rename_vars.  xradio and xarray are not dependencies of this package, so
SkyImage offers exactly that surface; data variables may be numpy arrays or
torch tensors on the device, so images stay resident between the steps of a
major cycle.  An xarray Dataset passed in its place works the same way.
"""
import numpy as np
import torch

DIMS = ("time", "frequency", "polarization", "l", "m")


class _Var:
    """A data variable or coordinate: .values / .data and .dims."""

    def __init__(self, values, dims, attrs=None):
        self.values = values
        self.dims = tuple(dims)
        self.attrs = dict(attrs or {})

    @property
    def data(self):
        return self.values

    @data.setter
    def data(self, values):
        if tuple(values.shape) != tuple(self.values.shape):
            raise ValueError("replacement data must keep the variable's shape")
        self.values = values

    @property
    def shape(self):
        return tuple(self.values.shape)

    @property
    def size(self):
        return int(np.prod(self.values.shape))

    def __len__(self):
        return int(self.values.shape[0]) if len(self.values.shape) else 1


def _copy(v):
    if isinstance(v, torch.Tensor):
        return v.clone()
    return np.array(v, copy=True)


class SkyImage:
    """Data variables over DIMS, 1-D coordinates and attributes."""

    def __init__(self, data_vars=None, coords=None, attrs=None):
        self._vars = {}
        self._coords = {}
        self.attrs = dict(attrs or {})
        for name, v in (coords or {}).items():
            self._coords[name] = v if isinstance(v, _Var) else _Var(np.asarray(v), (name,))
        for name, v in (data_vars or {}).items():
            self[name] = v

    # dataset surface -------------------------------------------------------
    @property
    def dims(self):
        return DIMS

    @property
    def sizes(self):
        if self._vars:
            out = {}
            for v in self._vars.values():
                out.update(zip(v.dims, (int(s) for s in v.values.shape)))
            # dimension coordinates of dims no variable uses, as xarray lists them
            for name, c in self._coords.items():
                if c.dims == (name,) and name not in out:
                    out[name] = len(c)
            return out
        return {d: len(self._coords[d]) for d in DIMS if d in self._coords}

    @property
    def coords(self):
        return self._coords

    @property
    def data_vars(self):
        return self._vars

    def __contains__(self, name):
        return name in self._vars or name in self._coords

    def __getitem__(self, name):
        if name in self._vars:
            return self._vars[name]
        return self._coords[name]

    def __setitem__(self, name, value):
        """ds[name] = array (dims DIMS, or their first three for a per-plane
        variable such as a normalisation) or (dims, array), as xarray takes
        it; a uv image is ("time", "frequency", "polarization", "u", "v")."""
        dims = None
        if isinstance(value, tuple) and len(value) == 2:
            dims, value = tuple(value[0]), value[1]
        vals = value.values if hasattr(value, "values") and not isinstance(
            value, (np.ndarray, torch.Tensor)) else value
        if not isinstance(vals, (np.ndarray, torch.Tensor)):
            vals = np.asarray(vals)
        if dims is None:
            if len(vals.shape) == len(DIMS):
                dims = DIMS
            elif len(vals.shape) == 3:
                dims = DIMS[:3]
            else:
                raise ValueError(f"{name}: data variables have dims {DIMS} (or {DIMS[:3]})")
        if len(dims) != len(vals.shape):
            raise ValueError(f"{name}: {len(dims)} dims for a {len(vals.shape)}-d array")
        self._vars[name] = _Var(vals, dims)

    def copy(self, deep=True):
        out = SkyImage(attrs=self.attrs)
        out._coords = {k: _Var(_copy(c.values) if deep else c.values, c.dims, c.attrs)
                       for k, c in self._coords.items()}
        out._vars = {k: _Var(_copy(v.values) if deep else v.values, v.dims)
                     for k, v in self._vars.items()}
        return out

    def load(self):
        return self

    def isel(self, **indexers):
        """Views of the variables and coordinates with the named dims indexed
        by the given slices (xarray's isel for slices)."""
        for d, sl in indexers.items():
            if not isinstance(sl, slice):
                raise TypeError(f"isel: {d} must be indexed by a slice")

        def cut(v):
            idx = tuple(indexers.get(d, slice(None)) for d in v.dims)
            return _Var(v.values[idx], v.dims, v.attrs)

        out = SkyImage(attrs=self.attrs)
        out._coords = {k: cut(c) for k, c in self._coords.items()}
        out._vars = {k: cut(v) for k, v in self._vars.items()}
        return out

    def rename_vars(self, mapping):
        out = self.copy(deep=False)
        out._vars = {mapping.get(k, k): v for k, v in self._vars.items()}
        return out

    def __repr__(self):
        return f"SkyImage(sizes={self.sizes}, vars={list(self._vars)})"


def make_sky_image(phase_center, image_size, cell_size, frequency_coords, pol_coords,
                   time_coords):
    """An image with the coordinates of make_empty_sky_image (time,
    frequency, polarization; l / m offsets of the pixel centres from the
    phase centre in radians) and no data variables."""
    ny, nx = int(image_size[0]), int(image_size[1])
    cell = np.asarray(cell_size, dtype=float)
    coords = {
        "time": np.atleast_1d(np.asarray(time_coords, dtype=float)),
        "frequency": np.atleast_1d(np.asarray(frequency_coords, dtype=float)),
        "polarization": np.asarray(list(pol_coords)),
        "l": (np.arange(ny) - ny // 2) * -abs(float(cell[0])),
        "m": (np.arange(nx) - nx // 2) * abs(float(cell[1])),
    }
    return SkyImage(coords=coords, attrs={"phase_center": tuple(phase_center),
                                          "cell_size": tuple(float(c) for c in cell)})


def make_uv_coords(image_size, cell_size):
    """u / v coordinates of the uv grid paired by the FFT with an (l, m)
    image of image_size pixels of cell_size radians: spacing
    1 / (n * cell) wavelengths, 0 at pixel n // 2."""
    out = {}
    for name, n, c in (("u", int(image_size[0]), float(cell_size[0])),
                       ("v", int(image_size[1]), float(cell_size[1]))):
        out[name] = (np.arange(n) - n // 2) / (n * abs(c))
    return out
