"""A minimal dataset for the convolution-function driver.

make_gridding_convolution_function (make_gridding_convolution_function.py:
24-193) fills an xarray Dataset: data variables set as (dims, array), .attrs,
len() (the number of data variables) and a dimension's size read as
``ds.<dim>.size``.  xarray is not a dependency of this package, so Dataset
offers that surface; with xarray installed the driver uses xarray's own.
"""
import numpy as np

from .sky_image import _Var


class Dataset:
    """Named data variables over named dims, coordinates and attributes."""

    def __init__(self, attrs=None):
        self.__dict__["_vars"] = {}
        self.__dict__["_coords"] = {}
        self.__dict__["attrs"] = dict(attrs or {})

    def __len__(self):
        return len(self._vars)

    def __contains__(self, name):
        return name in self._vars or name in self._coords

    def __getitem__(self, name):
        if name in self._vars:
            return self._vars[name]
        return self._coords[name]

    def __setitem__(self, name, value):
        """ds[name] = (dims, array), or a variable with .dims and .values."""
        if isinstance(value, tuple) and len(value) == 2:
            dims, vals = tuple(value[0]), np.asarray(value[1])
        else:
            dims, vals = tuple(value.dims), np.asarray(value.values)
        if len(dims) != vals.ndim:
            raise ValueError(f"{name}: {len(dims)} dims for a {vals.ndim}-d array")
        for d, n in zip(dims, vals.shape):
            have = self.sizes.get(d)
            if have is not None and have != n and not (name in self._vars and
                                                      d in self._vars[name].dims):
                raise ValueError(f"{name}: dim {d} of size {n} conflicts with {have}")
        self._vars[name] = _Var(vals, dims)

    @property
    def data_vars(self):
        return self._vars

    @property
    def coords(self):
        return self._coords

    @property
    def sizes(self):
        out = {}
        for v in list(self._vars.values()) + list(self._coords.values()):
            out.update(zip(v.dims, (int(s) for s in np.shape(v.values))))
        return out

    def __getattr__(self, name):
        # data variables, coordinates and, for a dim without a coordinate,
        # its default index (as xarray gives it)
        if name.startswith("_"):
            raise AttributeError(name)
        if name in self._vars:
            return self._vars[name]
        if name in self._coords:
            return self._coords[name]
        sizes = self.sizes
        if name in sizes:
            return _Var(np.arange(sizes[name]), (name,))
        raise AttributeError(name)

    def assign_coords(self, coords):
        """A new dataset sharing the variables, with the given 1-D
        coordinates added."""
        out = Dataset(self.attrs)
        out._vars.update(self._vars)
        out._coords.update(self._coords)
        for k, v in coords.items():
            out._coords[k] = _Var(np.asarray(v), (k,))
        return out

    def __repr__(self):
        return f"Dataset(sizes={self.sizes}, vars={list(self._vars)})"


def new_dataset():
    """xarray's Dataset when xarray is installed, else this module's."""
    try:
        import xarray as xr
    except ImportError:
        return Dataset()
    return xr.Dataset()
