"""The image <-> uv-grid transforms, their normalisations and the primary
beam on B200.

Drop-in for make_image_xds, remove_padding, make_empty_padded_uv_image,
apply_pb, fft_to_uv, ifft_to_lm, correct_fft_to_uv, correct_ifft_to_lm and
grid2xradio_spheroid_ms4 of
src/astroviper/core/imaging/imaging_utils/standard_image_grid_preparation.py
(:19-580): same arguments, defaults, variable-name rules, exceptions and
in-place updates of the image dataset.  The transforms are this package's
cuFFT fft_lm_to_uv / ifft_uv_to_lm; the normalisations (av_plane_rescale)
and the primary-beam product or quotient (av_apply_pb) run in libav200, one
launch per variable, in numpy's arithmetic for the reference's in-place
updates, so their results are bit-identical to the reference's for the same
inputs; the spheroid correction agrees to the 1e-14 relative of the device's
grid-correction term, and the transforms to cuFFT's rounding.  The dataset
constructors of the same file (make_image_xds, make_empty_padded_uv_image)
build SkyImage datasets here, since xradio is not a dependency: the same variables, dims, dtypes, sizes and data_groups,
with (l, m) coordinates as make_sky_image and (u, v) ones as
sky_image.make_uv_coords.

The image may be a SkyImage (its variables numpy arrays or device tensors) or
an xarray Dataset.  numpy variables are updated in place in their own
buffers, as the reference's `image[var].data /= ...` does; device tensors are
updated on the device.
"""
from typing import List, Union

import numpy as np

from .... import _host as H
from .... import _kernels as K
from ..fft import fft_lm_to_uv
from ..ifft import ifft_uv_to_lm
from ..sky_image import _Var, make_sky_image, make_uv_coords
from .gcf_prolate_spheroidal import create_prolate_spheroidal_kernel_1D
from .standard_grid import _is_datatree, standard_grid_numpy_wrap_input_checked

_DIV, _MUL, _SPHEROID = 0, 1, 2


def _try_vars(data_vars, default):
    if not data_vars:
        return list(default)
    if isinstance(data_vars, str):
        return [data_vars]
    return data_vars


def _rescale(x, mode, s, corr=None, w=None):
    """x (..., a, b) scaled in place by av_plane_rescale; returns x."""
    if H.is_torch(x) and x.is_cuda and x.is_contiguous():
        return K.plane_rescale(x, mode, s, corr, w)
    t = H.dev(x)
    K.plane_rescale(t, mode, s, corr, w)
    H.write_back(x, t)
    return x


def make_image_xds(imsize, cell, freq, freqinc, phasecent, which: str = "SKY", pol=None,
                   time=None):
    """standard_image_grid_preparation.py:19-96: an empty sky image with
    one float32 zero variable `which` (time, frequency, polarization, l, m);
    pol defaults to ["I"], time to [0.0]; freqinc, when given, is kept as the
    frequency coordinate's channel_width attribute."""
    if pol is None:
        pol = np.array(["I"])
    if time is None:
        time = np.array([0.0])
    freq_coords = np.atleast_1d(np.asarray(freq, dtype=float))
    image = make_sky_image(phasecent, imsize, cell, freq_coords, pol, time)
    if freqinc is not None:
        image.coords["frequency"].attrs["channel_width"] = {"data": freqinc, "units": "Hz"}
    shape = (len(np.atleast_1d(time)), len(freq_coords), len(pol), int(imsize[0]),
             int(imsize[1]))
    image[which] = np.zeros(shape, dtype=np.float32)
    image.attrs.setdefault("data_groups", {"base": {}})["base"][which.lower()] = which
    return image


def _phase_center(image):
    attrs = getattr(image, "attrs", {})
    if "phase_center" in attrs:
        return attrs["phase_center"]
    return image.coordinate_system_info["reference_direction"]["data"]


def make_empty_padded_uv_image(image, image_size, uv_data_array: str = "VISIBILITY_RESIDUAL",
                               insert_res_or_mod=True):
    """standard_image_grid_preparation.py:123-233: an empty uv image of
    image_size (u, v) cells for the image's time / frequency / polarization
    coordinates and cell size: uv_data_array complex64 zeros (time,
    frequency, polarization, u, v) and <uv_data_array>_NORMALIZATION float64
    zeros (time, frequency, polarization), both named in
    attrs["data_groups"]["base"]; with insert_res_or_mod, RESIDUAL (for
    VISIBILITY_RESIDUAL) or MODEL (for VISIBILITY_MODEL) of the image, when
    present, is copied as float32 into the centre of a zero (l, m) plane of
    image_size.  Raises when the image is larger than image_size."""
    image_size = np.array(image_size)
    image_size_current = np.array([image.sizes["l"], image.sizes["m"]])
    if np.any(image_size_current > image_size):
        raise Exception(
            f"current image size {image_size_current} is larger than requested {image_size}")
    lc = np.asarray(image.coords["l"].values)
    mc = np.asarray(image.coords["m"].values)
    cellsize = np.array([np.abs(lc[1] - lc[0]), np.abs(mc[1] - mc[0])])
    freq = np.asarray(image.coords["frequency"].values)
    pol = np.asarray(image.coords["polarization"].values)
    tim = np.asarray(image.coords["time"].values)
    out_im = make_sky_image(_phase_center(image), image_size, cellsize, freq, pol, tim)
    for name, values in make_uv_coords(image_size, cellsize).items():
        out_im.coords[name] = _Var(values, (name,))
    groups = out_im.attrs.setdefault("data_groups", {"base": {}})["base"]
    shape = (len(tim), len(freq), len(pol), int(image_size[0]), int(image_size[1]))
    out_im[uv_data_array] = (("time", "frequency", "polarization", "u", "v"),
                             np.zeros(shape, dtype=np.complex64))
    out_im[uv_data_array + "_NORMALIZATION"] = (("time", "frequency", "polarization"),
                                                np.zeros(shape[:3], dtype=np.float64))
    groups[uv_data_array.lower()] = uv_data_array
    groups[uv_data_array.lower() + "_normalization"] = uv_data_array + "_NORMALIZATION"
    if insert_res_or_mod:
        dat_name = {"VISIBILITY_MODEL": "MODEL",
                    "VISIBILITY_RESIDUAL": "RESIDUAL"}.get(uv_data_array, "")
        if dat_name and dat_name in image.data_vars:
            dat = image[dat_name].values
            if H.is_torch(dat):
                dat = dat.detach().cpu().numpy()
            blc = (image_size - np.array(dat.shape[-2:])) // 2
            trc = blc + np.array(dat.shape[-2:])
            plane = np.zeros(shape, dtype=np.float32)
            plane[:, :, :, blc[0]:trc[0], blc[1]:trc[1]] = dat
            out_im[dat_name] = plane
            groups[dat_name.lower()] = dat_name
    return out_im


def remove_padding(image, image_size):
    """standard_image_grid_preparation.py:99-120: the centre image_size
    (l, m) pixels of every variable, as views (image.isel)."""
    image_size = np.array(image_size)
    image_size_padded = np.array([image.sizes["l"], image.sizes["m"]])
    start_xy = image_size_padded // 2 - image_size // 2
    end_xy = start_xy + image_size
    return image.isel(l=slice(start_xy[0], end_xy[0]), m=slice(start_xy[1], end_xy[1]))


def apply_pb(image, pb=None, multiply: bool = True,
             data_vars: Union[str, List[str]] = "") -> None:
    """standard_image_grid_preparation.py:236-275: each of SKY, RESIDUAL,
    MODEL (or data_vars) present is multiplied (or divided, with NaN where
    the beam is 0) in place by PRIMARY_BEAM of pb, or of the image when pb is
    None.  The beam must be real."""
    if (pb is None) and ("PRIMARY_BEAM" not in image):
        raise Exception(f"No Primary beam information in {image}")
    pb_da = pb["PRIMARY_BEAM"] if pb is not None else image["PRIMARY_BEAM"]
    try_vars = _try_vars(data_vars, ("SKY", "RESIDUAL", "MODEL"))
    if tuple(pb_da.shape[-2:]) != tuple(image[try_vars[0]].shape[-2:]):
        raise Exception("shapes on sky are not the same")
    for sky_var in try_vars:
        if sky_var in image.data_vars:
            _mult_div(image[sky_var], pb_da, multiply=multiply)


def _mult_div(im_da, pb_da, multiply: bool = True) -> None:
    """standard_image_grid_preparation.py:278-309: im_da *= or /= pb_da,
    element by element for equal shapes, else (time, frequency,
    polarization) plane by plane with pb's index 0 along each axis whose
    extent differs."""
    x = im_da.data
    pbt = H.dev(pb_da.data)
    if H.is_torch(x) and x.is_cuda and x.is_contiguous():
        K.apply_pb(x, pbt, multiply)
        return
    t = H.dev(x)
    K.apply_pb(t, pbt, multiply)
    H.write_back(x, t)


def fft_to_uv(image, data_vars: Union[str, List[str]] = "") -> None:
    """standard_image_grid_preparation.py:312-341: VISIBILITY_<var> =
    fft_lm_to_uv(<var>) over axes 3, 4 for each of SKY, RESIDUAL, MODEL (or
    data_vars) present; the VISIBILITY_<var> variable must exist."""
    for sky_var in _try_vars(data_vars, ("SKY", "RESIDUAL", "MODEL")):
        if sky_var in image.data_vars:
            dat_name = "VISIBILITY_" + sky_var
            if dat_name not in image.data_vars:
                raise Exception(f"{dat_name} is not in {image}")
            image[dat_name].data = fft_lm_to_uv(image[sky_var].data, axes=[3, 4])


def ifft_to_lm(image, data_vars: Union[str, List[str]] = "") -> None:
    """standard_image_grid_preparation.py:344-377: SKY = ifft_uv_to_lm(
    VISIBILITY) and <name> = ifft_uv_to_lm(VISIBILITY_<name>) over axes 3, 4
    for each of VISIBILITY, VISIBILITY_RESIDUAL, VISIBILITY_MODEL (or
    data_vars) present; the target variable must exist."""
    for vis_var in _try_vars(data_vars,
                             ("VISIBILITY", "VISIBILITY_RESIDUAL", "VISIBILITY_MODEL")):
        if vis_var in image.data_vars:
            dat_name = ("SKY" if vis_var == "VISIBILITY"
                        else vis_var.split("VISIBILITY_", 1)[1])
            image[dat_name].data = ifft_uv_to_lm(image[vis_var].data, axes=[3, 4])


def correct_fft_to_uv(image, data_vars: Union[str, List[str]] = "") -> None:
    """standard_image_grid_preparation.py:380-409: each of VISIBILITY,
    VISIBILITY_RESIDUAL, VISIBILITY_MODEL (or data_vars) present is divided
    in place by the grid's u x v size."""
    try_vars = _try_vars(data_vars, ("VISIBILITY", "VISIBILITY_RESIDUAL", "VISIBILITY_MODEL"))
    u_size = image.sizes["u"]
    v_size = image.sizes["v"]
    for vis_var in try_vars:
        if vis_var in image.data_vars:
            _rescale(image[vis_var].data, _DIV, u_size * v_size)


def correct_ifft_to_lm(image, data_vars: Union[str, List[str]] = "",
                       doSpheroidCorr: bool = False, convsampling: int = 100,
                       convsupport: int = 7) -> None:
    """standard_image_grid_preparation.py:412-492: each of SKY, RESIDUAL (or
    data_vars) present is multiplied in place by l x m; with doSpheroidCorr
    each (time, frequency, polarization) plane is multiplied instead by
    l x m / (corrTerm x norm), corrTerm the grid correction of the
    prolate-spheroidal kernel for the (l, m) image and norm the plane's
    value of VISIBILITY_NORMALIZATION (for SKY) or
    VISIBILITY_<var>_NORMALIZATION, which must exist.  The correction is
    applied over the variable's dims in the order (time, frequency,
    polarization, l, m)."""
    try_vars = _try_vars(data_vars, ("SKY", "RESIDUAL"))
    nx = image.sizes["l"]
    ny = image.sizes["m"]
    corr = None
    if doSpheroidCorr:
        # create_prolate_spheroidal_kernel's kernel image depends only on the
        # image size, so the kernel itself (unused here) is not built.
        corr = K.corr_term(nx, ny)
    for sky_var in try_vars:
        if sky_var in image.data_vars:
            if not doSpheroidCorr:
                _rescale(image[sky_var].data, _MUL, nx * ny)
                continue
            sumwt = ("VISIBILITY_NORMALIZATION" if sky_var == "SKY"
                     else "VISIBILITY_" + sky_var + "_NORMALIZATION")
            if sumwt not in image.data_vars:
                raise Exception(f"Do not have {sumwt} to do image correction")
            var = image[sky_var]
            dims = tuple(getattr(var, "dims", ()))
            if dims and dims[-2:] != ("l", "m"):
                raise ValueError(f"{sky_var}: dims {dims} do not end with (l, m)")
            x = var.data
            norm = image[sumwt].data
            n_planes = int(np.prod(x.shape[:-2]))
            if int(np.prod(norm.shape)) != n_planes:
                raise ValueError(f"{sumwt} has {int(np.prod(norm.shape))} values for "
                                 f"{n_planes} planes of {sky_var}")
            _rescale(x, _SPHEROID, nx * ny, corr, norm)


def grid2xradio_spheroid_ms4(vis, image, support: int = 7, sampling: int = 100,
                             data_var: str = "VISIBILITY", chan_mode: str = "continuum", *,
                             precision=None):
    """standard_image_grid_preparation.py:495-580: grids every MSv4 node of
    vis (one node or a list) into the image's data_var uv grid and its
    <data_var>_NORMALIZATION sums, in place, for each time plane of the
    image (as the reference, every node is gridded into every time plane).
    UV_SAMPLING grids the weights (do_psf).  The cell size is the spacing of
    the image's l and m coordinates.  As the reference, flagged samples get
    weight 0 in each node's WEIGHT array.  The gridding is
    standard_grid_numpy_wrap_input_checked on the device; precision is the
    package's option ("fp32", the default of config.precision: the tiled
    FP32 gridder; "fp64": the reference's FP64 arithmetic)."""
    listvis = [vis] if _is_datatree(vis) else vis
    nx = image.sizes["u"]
    ny = image.sizes["v"]
    dopsf = data_var == "UV_SAMPLING"
    lc = np.asarray(image.coords["l"].values)
    mc = np.asarray(image.coords["m"].values)
    pixelincr = np.array([np.abs(lc[1] - lc[0]), np.abs(mc[1] - mc[0])])
    if data_var not in image.data_vars:
        raise Exception(f"{data_var} is not in {image}")
    sumwt_var = data_var + "_NORMALIZATION"
    dat_array = image[data_var]
    sumwt_array = image[sumwt_var]
    for da in (dat_array, sumwt_array):
        dims = tuple(getattr(da, "dims", ("time",)))
        if dims[0] != "time":
            raise ValueError(f"grid2xradio_spheroid_ms4: time must be the first dim, not {dims}")
    cgk_1D = create_prolate_spheroidal_kernel_1D(sampling, support)
    n_time = len(np.atleast_1d(np.asarray(image.coords["time"].values)))
    for it in range(n_time):
        gridvis = dat_array.data[it]
        sumwt = sumwt_array.data[it]
        for elvis in listvis:
            if not _is_datatree(elvis):
                raise TypeError("One of the elements of vis is not an xarray datatree")
            vis_data = elvis[data_var].data
            uvw = elvis.UVW.data
            weight = elvis.WEIGHT.data
            flag = elvis.FLAG.data
            weight[flag] = 0.0
            freq_chan = elvis.coords["frequency"].values
            gridvis, sumwt = standard_grid_numpy_wrap_input_checked(
                vis_data, gridvis, sumwt, uvw, weight, freq_chan, cgk_1D,
                image_size=np.array([nx, ny], dtype=int), cell_size=pixelincr,
                oversampling=sampling, support=support, complex_grid=True, do_psf=dopsf,
                chan_mode=chan_mode, precision=precision)
