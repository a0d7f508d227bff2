"""Standard (PSWF) degridder on B200.

Drop-in for src/astroviper/core/imaging/imaging_utils/standard_degrid.py.  The
four reference variants (dgrid, dgrid_optimized, dgrid2, dgrid_numba) compute
the same sum; all run the libav200 degridder (av_degrid_tiled in "fp32",
av_degrid_plain in "fp64", which reproduces dgrid_numba bit for bit).  The
variants differ only in the bounds axes used for non-square grids
(dgrid_numba tests x against shape[3], standard_degrid.py:407); the kernel
applies dgrid_numba's test and the array's true extents.

``values`` is updated in place (+=), like the reference.
"""
import math

import numpy as np
import torch

from .... import _host as H
from .... import _kernels as K
from ....config import resolve_precision
from .gcf_prolate_spheroidal import create_prolate_spheroidal_kernel_1D

C_LIGHT = 299792458.0


def sgrid(uvw, dphase, freq, c, scale, offset, sampling, pos, loc, off):
    """standard_degrid.py:8-29: position, cell, kernel offset and phasor of one
    sample (writes pos, loc, off in place, returns the phasor)."""
    pos[:2] = scale[:2] * uvw[:2] * freq / c + (offset[:2])
    loc[:2] = np.round(pos[:2]).astype(int)
    off[:2] = np.round((loc[:2] - pos[:2]) * sampling).astype(int)
    phase = -2.0 * np.pi * dphase * freq / c
    return complex(np.cos(phase), np.sin(phase))


def sgrid_numba(uvw, dphase, freq, c, scale, offset, sampling):
    """standard_degrid.py:367-385: returns (phasor, loc, off)."""
    pos = np.empty(2, dtype=np.float64)
    loc = np.empty(2, dtype=np.int32)
    off = np.empty(2, dtype=np.int32)
    pos[0] = scale[0] * uvw[0] * freq / c + offset[0]
    pos[1] = scale[1] * uvw[1] * freq / c + offset[1]
    loc[0] = int(np.round(pos[0]))
    loc[1] = int(np.round(pos[1]))
    off[0] = int(np.round((float(loc[0]) - pos[0]) * float(sampling)))
    off[1] = int(np.round((float(loc[1]) - pos[1]) * float(sampling)))
    phase = -2.0 * np.pi * dphase * freq / c
    phasor = np.cos(phase) + 1j * np.sin(phase)
    return phasor, loc, off


def _degrid_inplace(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                    convFunc, chanmap, polmap, precision=None):
    precision = resolve_precision(precision)
    if (isinstance(values, np.ndarray) and values.flags.c_contiguous and values.flags.writeable
            and np.iscomplexobj(values) and np.ndim(grid) == 4
            and H.streamable(values, uvw, None if flag is None else np.asarray(flag))
            and K.degrid_tiled_ok(precision, int(support), int(sampling),
                                  int(np.shape(grid)[1]), c)):
        # large host arrays: values / flags / uvw in time chunks, copied in
        # and back while neighbouring chunks are degridded
        dph = None
        if dphase is not None and np.any(np.asarray(dphase) != 0):
            dph = np.asarray(dphase, dtype=np.float64)
        K.degrid_streamed(grid, uvw, freq, scale, offset, chanmap, polmap, convFunc,
                          int(support), int(sampling), values,
                          flag=None if flag is None else np.asarray(flag), dphase=dph)
        return
    vals = H.dev(values)
    if not vals.is_complex():
        raise TypeError("values must be complex")
    dph = None
    if dphase is not None:
        d = np.asarray(dphase) if not H.is_torch(dphase) else dphase
        if H.is_torch(d) or np.any(d != 0):
            dph = H.dev(d, torch.float64)
    acc = vals
    K.degrid(grid, uvw, freq, scale, offset, chanmap, polmap, convFunc, int(support),
             int(sampling), values=acc, flag=None if flag is None else H.dev(flag),
             dphase=dph, c=float(c), precision=precision)
    if H.is_torch(values):
        if values.data_ptr() != acc.data_ptr():
            values.copy_(acc)
    else:
        H.write_back(values, acc)


def dgrid_numba(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                convFunc, chanmap, polmap, *, precision=None):
    """standard_degrid.py:388-485: values[t, b, chan, pol] += degridded model."""
    _degrid_inplace(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                    convFunc, chanmap, polmap, precision)


def dgrid(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling, convFunc,
          chanmap, polmap, *, precision=None):
    """standard_degrid.py:32-138 (same sum as dgrid_numba)."""
    _degrid_inplace(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                    convFunc, chanmap, polmap, precision)


def dgrid_optimized(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                    convFunc, chanmap, polmap, *, precision=None):
    """standard_degrid.py:144-278 (same sum as dgrid_numba)."""
    _degrid_inplace(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                    convFunc, chanmap, polmap, precision)


def dgrid2(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling, convFunc,
           chanmap, polmap, *, precision=None):
    """standard_degrid.py:281-361 (same sum as dgrid_numba)."""
    _degrid_inplace(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                    convFunc, chanmap, polmap, precision)


class _ModelArray:
    """Result holder used when xarray is not installed (data / values / dims /
    coords like an xarray.DataArray)."""

    def __init__(self, data, coords=None, dims=None):
        self.data = data
        self.values = data
        self.coords = coords
        self.dims = dims


def degrid_spheroid_ms4(vis, grid, pixelincr, support: int = 7, sampling: int = 100,
                        incremental: bool = False, whichFunc=0, *, precision=None):
    """standard_degrid.py:488-608: degrids `grid` onto the node's samples and
    stores VISIBILITY_MODEL.  As the reference, NaN-uvw rows are flagged and
    their uvw set to 1e9 in the caller's arrays."""
    uvw = vis.UVW.data
    dims = vis.dims
    dphase = None  # the reference grids at the phase centre: zero phase
    fresh = not incremental or "VISIBILITY_MODEL" not in vis
    modvis = None if fresh else vis.VISIBILITY_MODEL.data
    flag = vis.FLAG.data
    uvwmask = np.isnan(np.asarray(uvw))
    nan_it, nan_ib = np.where(uvwmask.any(axis=-1))
    for k in range(len(nan_it)):
        flag[nan_it[k], nan_ib[k], :, :] = True
        uvw[nan_it[k], nan_ib[k], :] = 1e9
    nx, ny = grid.shape[-2:]
    scale = np.array([-pixelincr[0] * nx, -pixelincr[1] * ny, 0.0]).astype(np.float64)
    offset = np.array([nx / 2, ny / 2, 0.0]).astype(np.float64)
    freq = vis.frequency.data
    convFunc = create_prolate_spheroidal_kernel_1D(sampling, support)
    nchan = grid.shape[0]
    npol = grid.shape[1]
    chanmap = (np.arange(dims["frequency"]) / dims["frequency"] * nchan).astype(int)
    polmap = np.round(np.arange(dims["polarization"]) % npol).astype(int)
    if fresh:
        # a fresh model (np.zeros then += in the reference): the tiled kernel
        # stores every sample (zeros where skipped) straight into a complex128
        # device array, which is copied back once
        p = resolve_precision(precision)
        shape = (dims["time"], dims["baseline_id"], dims["frequency"], dims["polarization"])
        vals = torch.empty(shape, dtype=torch.complex128, device=K.device())
        K.degrid(grid, uvw, freq, scale, offset, chanmap, polmap, convFunc, int(support),
                 int(sampling), values=vals, flag=H.dev(flag), precision=p,
                 accumulate=False)
        modvis = H.host(vals)
    else:
        _degrid_inplace(uvw, dphase, modvis, flag, scale, offset, grid, freq, C_LIGHT, support,
                        sampling, convFunc, chanmap, polmap, precision)
    datdims = vis.VISIBILITY.dims
    datcoords = vis.VISIBILITY.coords
    try:
        import xarray
        modvis_da = xarray.DataArray(modvis, coords=datcoords, dims=datdims)
    except ImportError:
        modvis_da = _ModelArray(modvis, coords=datcoords, dims=datdims)
    vis["VISIBILITY_MODEL"] = modvis_da
