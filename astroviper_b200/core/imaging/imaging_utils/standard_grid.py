"""Standard (PSWF) gridder and image formation on B200.

Drop-in for src/astroviper/core/imaging/imaging_utils/standard_grid.py:
same function names, arguments, defaults, in-place updates and errors.  The
numerical work runs in libav200 (av_grid_tiled / av_grid_plain /
av_grid_to_image); host arrays are staged to the device and results copied
back into the caller's arrays, as the reference updates them in place.

Accepts numpy arrays (results are numpy) or torch tensors (results stay
torch tensors on the device).
"""
from typing import List, Tuple, Union

import numpy as np
import torch

from .... import _host as H
from .... import _kernels as K
from ....config import resolve_precision
from .gcf_prolate_spheroidal import create_prolate_spheroidal_kernel_1D


def _grid_into(grid, sum_weight, do_psf, do_imaging_weight, vis_data, uvw, freq_chan, chan_map,
               pol_map, weight, cgk_1D, n_uv, delta_lm, support, oversampling, precision):
    """Accumulate into grid / sum_weight (host or device arrays) in place."""
    precision = resolve_precision(precision)
    n_img_chan, n_img_pol = int(grid.shape[0]), int(grid.shape[1])
    g_dev = H.dev(grid)
    real_grid = not g_dev.is_complex()
    if real_grid and not do_psf:
        raise TypeError("a real grid can only hold do_psf=True gridding")
    sw_dev = H.dev(sum_weight, torch.float64)
    if precision == "fp32" and real_grid:
        precision = "fp64"  # the tiled kernel writes complex grids only
    target = g_dev
    vis_in = None if do_psf else vis_data
    if (not real_grid and H.streamable(vis_in, weight, uvw)
            and K.grid_tiled_ok(precision, do_imaging_weight, support, oversampling,
                                int(weight.shape[3]), n_img_pol)):
        # large host inputs: copied in time chunks that overlap the gridding
        K.grid_streamed(vis_in, weight, uvw, freq_chan, chan_map, pol_map, cgk_1D, n_uv,
                        delta_lm, support, oversampling, n_img_chan, n_img_pol,
                        grid_out=target, sum_weight=sw_dev, do_psf=do_psf)
    else:
        K.grid(vis_in, H.dev(weight), uvw, freq_chan, chan_map, pol_map,
               cgk_1D, n_uv, delta_lm, support, oversampling, n_img_chan, n_img_pol,
               grid_out=target, sum_weight=sw_dev, do_psf=do_psf,
               do_imaging_weight=do_imaging_weight, precision=precision)
    if H.is_torch(grid):
        if grid.data_ptr() != target.data_ptr():
            grid.copy_(target)
    else:
        H.write_back(grid, target)
    if H.is_torch(sum_weight):
        if sum_weight.data_ptr() != sw_dev.data_ptr():
            sum_weight.copy_(sw_dev)
    else:
        H.write_back(sum_weight, sw_dev)


def standard_grid_numpy_wrap_input_checked(
    vis_data,
    grid,
    sum_weight,
    uvw,
    weight,
    freq_chan,
    cgk_1D,
    image_size,
    cell_size,
    oversampling: int = 100,
    support: int = 7,
    complex_grid: bool = True,
    do_psf: bool = False,
    chan_mode: str = "continuum",
    *,
    precision=None,
) -> Tuple[np.ndarray, np.ndarray]:
    """standard_grid.py:15-85: builds the parameter dict and calls
    standard_grid_numpy_wrap.  Returns (grid, sum_weight)."""
    params = {
        "image_size_padded": image_size,
        "cell_size": cell_size,
        "complex_grid": complex_grid,
        "oversampling": oversampling,
        "support": support,
        "do_psf": do_psf,
        "chan_mode": chan_mode,
    }
    return standard_grid_numpy_wrap(vis_data, grid, sum_weight, uvw, weight, freq_chan, cgk_1D,
                                    params, precision=precision)


def _maps(weight, chan_mode):
    n_chan = weight.shape[2]
    if chan_mode == "cube":
        n_imag_chan = n_chan
        chan_map = np.arange(0, n_chan).astype(int)
    else:
        n_imag_chan = 1
        chan_map = np.zeros(n_chan).astype(int)
    n_imag_pol = weight.shape[3]
    pol_map = np.arange(0, n_imag_pol).astype(int)
    return n_imag_chan, chan_map, n_imag_pol, pol_map


def standard_grid_numpy_wrap(vis_data, grid, sum_weight, uvw, weight, freq_chan, cgk_1D,
                             grid_params, *, precision=None):
    """standard_grid.py:88-165: grids vis (or weights for do_psf) into grid,
    creating a complex128 (or float64) grid and sum_weight when both given
    arrays are empty, else accumulating into them."""
    n_imag_chan, chan_map, n_imag_pol, pol_map = _maps(weight, grid_params["chan_mode"])
    n_uv = grid_params["image_size_padded"]
    delta_lm = grid_params["cell_size"]
    oversampling = grid_params["oversampling"]
    support = grid_params["support"]
    torch_io = H.is_torch(vis_data) or H.is_torch(weight)
    if np.size(grid) == 0 and np.size(sum_weight) == 0:
        # fresh arrays (standard_grid.py:133-143): made on the device and
        # returned to the host once
        shape = (n_imag_chan, n_imag_pol, int(n_uv[0]), int(n_uv[1]))
        dt = torch.complex128 if grid_params["complex_grid"] else torch.float64
        g_dev = torch.zeros(shape, dtype=dt, device=K.device())
        s_dev = torch.zeros((n_imag_chan, n_imag_pol), dtype=torch.float64, device=K.device())
        _grid_into(g_dev, s_dev, grid_params["do_psf"], False, vis_data, uvw, freq_chan,
                   chan_map, pol_map, weight, cgk_1D, n_uv, delta_lm, support, oversampling,
                   precision)
        if torch_io:
            return g_dev, s_dev
        return H.host(g_dev), H.host(s_dev)
    _grid_into(grid, sum_weight, grid_params["do_psf"], False, vis_data, uvw, freq_chan, chan_map,
               pol_map, weight, cgk_1D, n_uv, delta_lm, support, oversampling, precision)
    return grid, sum_weight


def standard_grid_psf_numpy_wrap(uvw, weight, freq_chan, cgk_1D, grid_params, *,
                                 precision=None):
    """standard_grid.py:168-239: grids weights onto a fresh float64 grid
    (do_imaging_weight per grid_params).  Returns (grid, sum_weight)."""
    n_imag_chan, chan_map, n_imag_pol, pol_map = _maps(weight, grid_params["chan_mode"])
    n_uv = grid_params["image_size_padded"]
    grid = np.zeros((n_imag_chan, n_imag_pol, int(n_uv[0]), int(n_uv[1])), dtype=np.double)
    sum_weight = np.zeros((n_imag_chan, n_imag_pol), dtype=np.double)
    _grid_into(grid, sum_weight, grid_params["do_psf"], grid_params["do_imaging_weight"], None,
               uvw, freq_chan, chan_map, pol_map, weight, cgk_1D, n_uv,
               grid_params["cell_size"], grid_params["support"], grid_params["oversampling"],
               precision)
    return grid, sum_weight


def standard_grid_jit(grid, sum_weight, do_psf, do_imaging_weight, vis_data, uvw, freq_chan,
                      chan_map, pol_map, weight, cgk_1D, n_uv, delta_lm, support, oversampling,
                      *, precision=None):
    """standard_grid.py:246-432: accumulates into grid and sum_weight in place
    (grid (n_chan, n_pol, n_u, n_v), sum_weight (n_chan, n_pol))."""
    _grid_into(grid, sum_weight, do_psf, do_imaging_weight, vis_data, uvw, freq_chan, chan_map,
               pol_map, weight, cgk_1D, n_uv, delta_lm, support, oversampling, precision)


def standard_imaging_weight_degrid_numpy_wrap(grid_imaging_weight, uvw, natural_imaging_weight,
                                              briggs_factors, freq_chan, grid_params):
    """standard_grid.py:441-484: per-sample, per-polarisation imaging weights
    (float64, the shape of natural_imaging_weight) read from a cube of
    imaging-weight grids (n_chan, n_pol, n_u, n_v) with the Briggs factors
    (2, n_chan, n_pol); zero for samples off the grid.  Channel c and
    polarisation p read grid (c, p), as the reference's identity maps."""
    n_chan = natural_imaging_weight.shape[2]
    n_imag_pol = natural_imaging_weight.shape[3]
    out = torch.zeros(tuple(int(s) for s in natural_imaging_weight.shape), dtype=torch.float64,
                      device=K.device())
    K.imaging_weight_degrid(out, grid_imaging_weight, briggs_factors, uvw, freq_chan,
                            np.arange(0, n_chan), np.arange(0, n_imag_pol),
                            natural_imaging_weight, grid_params["image_size_padded"],
                            grid_params["cell_size"])
    if H.is_torch(natural_imaging_weight) or H.is_torch(grid_imaging_weight):
        return out
    return H.host(out)


def standard_imaging_weight_degrid_jit(imaging_weight, grid_imaging_weight, briggs_factors, uvw,
                                       freq_chan, chan_map, pol_map, natural_imaging_weight,
                                       n_uv, delta_lm):
    """standard_grid.py:487-604: writes the imaging weights of the samples on
    the grid into imaging_weight in place (entries of samples off the grid
    keep their values).  chan_map / pol_map entries index the grid's
    channels / polarisations (ValueError otherwise)."""
    iw = H.dev(imaging_weight, torch.float64)
    K.imaging_weight_degrid(iw, grid_imaging_weight, briggs_factors, uvw, freq_chan, chan_map,
                            pol_map, natural_imaging_weight, n_uv, delta_lm)
    if H.is_torch(imaging_weight):
        if imaging_weight.data_ptr() != iw.data_ptr():
            imaging_weight.copy_(iw)
    else:
        H.write_back(imaging_weight, iw)


def _is_datatree(x):
    try:
        import xarray  # noqa: F401
        from xarray.core.datatree import DataTree
        return isinstance(x, DataTree)
    except Exception:
        # without xarray, accept objects shaped like an MSv4 node
        return all(hasattr(x, a) for a in ("UVW", "WEIGHT", "FLAG", "coords")) and \
            hasattr(x, "__getitem__")


def grid2image_spheroid_ms4(
    vis,
    resid_array: np.ndarray,
    pixelincr: np.ndarray,
    support: int = 7,
    sampling: int = 100,
    dopsf: bool = False,
    column: str = "VISIBILITY",
    chan_mode: str = "continuum",
    *,
    precision=None,
):
    """standard_grid.py:607-708: grids one MSv4 node (or a list) and writes the
    grid-corrected dirty image (or PSF with dopsf) into resid_array in place.
    As the reference, flagged samples and NaN-uvw rows get weight 0 in the
    caller's WEIGHT array."""
    listvis = [vis] if _is_datatree(vis) else vis
    nx, ny = resid_array.shape[-2:]
    cgk_1D = create_prolate_spheroidal_kernel_1D(sampling, support)
    gridvis = None
    sumwt = None
    for elvis in listvis:
        if not _is_datatree(elvis):
            raise TypeError("One of the elements of vis is not an xarray datatree")
        vis_data = elvis[column].data
        uvw = elvis.UVW.data
        weight = elvis.WEIGHT.data
        flag = elvis.FLAG.data
        weight[flag] = 0.0
        nan_uvw = np.isnan(uvw[:, :, 0]) | np.isnan(uvw[:, :, 1])
        weight[nan_uvw] = 0.0
        freq_chan = elvis.coords["frequency"].values
        n_imag_chan, chan_map, n_imag_pol, pol_map = _maps(weight, chan_mode)
        if gridvis is None:
            # complex128 in both precisions: the fp32 kernel accumulates in FP64
            gridvis = torch.zeros((n_imag_chan, n_imag_pol, nx, ny), dtype=torch.complex128,
                                  device=K.device())
            sumwt = torch.zeros((n_imag_chan, n_imag_pol), dtype=torch.float64,
                                device=K.device())
        _grid_into(gridvis, sumwt, dopsf, False, vis_data, uvw, freq_chan, chan_map, pol_map,
                   weight, cgk_1D, np.array([nx, ny]), pixelincr, support, sampling, precision)
        if tuple(gridvis.shape) != tuple(resid_array.shape):
            raise RuntimeError(
                f"Shapes of gridded vis and image do no match {tuple(gridvis.shape)} and "
                f"{tuple(resid_array.shape)}")
    img = K.grid_to_image(gridvis, sumwt, apply_corr=True, out_dtype=torch.float64)
    H.write_back(resid_array, img)
