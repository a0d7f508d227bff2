"""Deconvolution on B200.

Drop-in for src/astroviper/core/imaging/deconvolution.py: get_phase_center
(:20-43), progress_callback (:46-71), _validate_deconv_params (:74-120),
deconvolve (:123-329) and hogbom_clean (:332-426), with the same arguments,
defaults, statistics and errors.  deconvolve takes image datasets with dims
(time, frequency, polarization, l, m) - SkyImage, or an xarray Dataset where
xarray is installed - whose planes may be numpy arrays or device tensors;
every plane is cleaned, measured and written on the device.
"""
import logging
from typing import Optional

import numpy as np
import torch

from ... import _kernels as K
from .deconvolvers import hogbom
from .imaging_utils.return_dict import ReturnDict

logger = logging.getLogger("astroviper_b200")


def progress_callback(iter_num: int, px: int, py: int, peak: float, niter_log: int = 100):
    """Logs the CLEAN progress every niter_log iterations (deconvolution.py:46)."""
    if iter_num % niter_log == 0:
        logger.info(f"  Iteration {iter_num}, peak at ({px}, {py}): {peak:.6f}")


def get_phase_center(dirty_image_xds):
    """"ra,dec" of the image centre (deconvolution.py:20-43): the
    right_ascension / declination coordinates at the centre pixel when the
    image has them, else the phase_center attribute of a SkyImage."""
    coords = dirty_image_xds.coords
    if "right_ascension" in coords and "declination" in coords:
        ra = coords["right_ascension"].values
        dec = coords["declination"].values
        return f"{ra[ra.shape[0] // 2, ra.shape[1] // 2]},{dec[dec.shape[0] // 2, dec.shape[1] // 2]}"
    pc = dirty_image_xds.attrs.get("phase_center", (0.0, 0.0))
    return f"{float(pc[0])},{float(pc[1])}"


# Hogbom parameters: (name, default, test a given value passes, message when
# it fails).  Names, defaults, tests and messages are the reference's
# (deconvolution.py:86-118): callers and tests match on the messages.
_HOGBOM_PARAMS = (
    ("gain", 0.1, lambda v: 0 < v <= 1, "CLEAN gain must be between 0 and 1."),
    ("niter", 1000, lambda v: isinstance(v, int) and v > 0,
     "Maximum number of iterations must be a positive integer."),
    ("threshold", 0.0, lambda v: v is None or not v < 0,
     "Threshold must be non-negative or None."),
    ("clean_box", (-1, -1, -1, -1), lambda v: v is None or (isinstance(v, tuple) and len(v) == 4),
     "Clean box must be a 4-tuple (xmin, xmax, ymin, ymax) or None."),
)


def _validate_deconv_params(deconv_params):
    """Checks the given Hogbom parameters in table order and fills in the
    missing ones, in place (deconvolution.py:74-120): the first failing value
    raises ValueError; a missing one is logged and set to its default."""
    for name, default, passes, message in _HOGBOM_PARAMS:
        if name not in deconv_params:
            logger.info(f"Deconvolution parameter '{name}' not specified. Using default: {default}")
            deconv_params[name] = default
        elif not passes(deconv_params[name]):
            raise ValueError(message)
    return deconv_params


def _is_plane(a):
    return isinstance(a, (np.ndarray, torch.Tensor)) and a.ndim == 2


def hogbom_clean(dirty_image: np.ndarray, psf: np.ndarray, deconv_params: Optional[dict] = None,
                 output_dir: str = ".", *, progress=True):
    """One plane of Hogbom CLEAN (deconvolution.py:332-426): returns the
    result statistics (iterations_performed, final_peak, total_flux_cleaned,
    converged), the model and the residual.

    dirty_image and psf are 2-D arrays of one shape (numpy arrays, or device
    tensors, which the results then stay beside); deconv_params is checked
    and completed in place.  The CLEAN runs in FP32, as the reference's call
    selects it with an empty float32 mask.  progress=False leaves out the
    logging callback; the arithmetic, and so every result, is the same."""
    params = _validate_deconv_params(deconv_params)
    for name, plane in (("dirty_image", dirty_image), ("psf", psf)):
        if not _is_plane(plane):
            raise ValueError(f"{name} must be a 2D numpy array with shape (ny, nx)")
    if tuple(dirty_image.shape) != tuple(psf.shape):
        raise ValueError(
            f"dirty_image and psf must have same shape. Got {dirty_image.shape} and {psf.shape}")
    stats = hogbom.clean(dirty_image, psf, mask=np.array([], dtype=np.float32),
                         clean_box=params["clean_box"] or (-1, -1, -1, -1),
                         max_iter=params["niter"], gain=params["gain"],
                         threshold=params["threshold"],
                         progress_callback=progress_callback if progress else None)
    model = stats.pop("model_image")
    residual = stats.pop("residual_image")
    return stats, model, residual


# ---------------------------------------------------------------- deconvolve --
# extract_main_lobe parameters used by deconvolve (deconvolution.py:202-206)
_PSF_FIT_WINDOW = (41, 41)
_PSF_FIT_CUTOFF = 0.35
_MIN_PSF_FRACTION = 0.1
_MAX_PSF_FRACTION = 0.8


def _masksum(image, dv):
    """get_image_masksum (image_statistics.py:9-37): sum of MASK_<dv>, else
    the pixel count of one plane."""
    name = "MASK_" + dv
    if name in image:
        m = image[name].values
        return int(m.sum().item() if isinstance(m, torch.Tensor) else np.sum(m))
    shape = image[dv].values.shape
    return int(np.prod(shape[-2:]))


def _peak_residual(plane, mask=None):
    """image_peak_residual of one plane (image_statistics.py:40-88,
    per_plane_stats=False): the value at the largest |x|, masked pixels out
    (NaN, as xarray's where leaves them) when a mask is given."""
    t = K.on_device(plane)
    if mask is not None:
        m = K.on_device(mask)
        t = torch.where(m.to(torch.bool), t.to(torch.float64),
                        torch.full((), float("nan"), dtype=torch.float64, device=t.device))
    return K.argmax(t, 0)[1]


def _device_cube(values):
    t = values if isinstance(values, torch.Tensor) else torch.from_numpy(np.asarray(values))
    t = t.to(device=K.device())
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    return t.contiguous()


def _put(dst, src):
    """Write device tensor src into a dataset variable's values in place."""
    if isinstance(dst, torch.Tensor):
        dst.copy_(src.to(dst.dtype))
    else:
        dst[...] = src.detach().cpu().numpy().astype(dst.dtype, copy=False)


def deconvolve(dirty_image_xds, psf_xds, model_xds=None, algorithm: str = "hogbom",
               deconv_params: Optional[dict] = None, output_dir: str = "."):
    """deconvolution.py:123-329: cleans every (time, frequency, polarization)
    plane of RESIDUAL with POINT_SPREAD_FUNCTION (a Stokes-I PSF serves every
    polarization) and returns (ReturnDict, model image, residual image).

    As the reference: each plane's model holds the components of this call
    only (an initial model only sets start_model_flux), the PSF sidelobe is
    extract_main_lobe's over a 41 x 41 window at 0.35 of the peak, and the
    peak residuals are the signed values at the largest |x|.  The CLEAN runs
    per plane without the logging callback (same results)."""
    rd = ReturnDict()
    sizes = dirty_image_xds.sizes
    ntime, nchan, npol = sizes["time"], sizes["frequency"], sizes["polarization"]
    npol_psf = psf_xds.sizes["polarization"]
    broadcast = npol_psf == 1 and npol > 1
    if broadcast:
        logger.info(f"PSF is single-plane, will broadcast to {npol} polarizations")
    elif npol_psf != npol:
        raise ValueError(
            "PSF should have same number of polarizations as the input image, or be Stokes I "
            f"only. (npol_psf = {npol_psf}, npol_image = {npol})")
    masksum = _masksum(dirty_image_xds, "RESIDUAL")
    phase_center = get_phase_center(dirty_image_xds)
    if algorithm.lower() != "hogbom":
        raise ValueError(f"Deconvolution algorithm '{algorithm}' not recognized.")
    dirty = _device_cube(dirty_image_xds["RESIDUAL"].values)
    psf = _device_cube(psf_xds["POINT_SPREAD_FUNCTION"].values)
    mask = None
    if "MASK_RESIDUAL" in dirty_image_xds:
        mask = _device_cube(dirty_image_xds["MASK_RESIDUAL"].values)
    start_flux = None
    if model_xds is not None:
        start_flux = K.plane_sum(_device_cube(model_xds["MODEL"].values)).cpu().numpy()

    full_model = dirty_image_xds.copy(deep=True).load().rename_vars({"RESIDUAL": "MODEL"})
    full_resid = dirty_image_xds.copy(deep=True).load()
    model_out = torch.zeros(dirty.shape, dtype=torch.float64, device=dirty.device)
    resid_out = dirty.to(torch.float64).clone()
    pol_c = dirty_image_xds.coords["polarization"].values
    freq_c = dirty_image_xds.coords["frequency"].values
    time_c = dirty_image_xds.coords["time"].values
    for tt in range(ntime):
        for nn in range(nchan):
            sidelobe = K.psf_sidelobe(psf[tt, nn, 0], _PSF_FIT_WINDOW, _PSF_FIT_CUTOFF)
            for pp in range(npol):
                logger.info(f"Deconvolving time {tt+1}/{ntime}, freq {nn+1}/{nchan}, "
                            f"pol {pp+1}/{npol}")
                d = dirty[tt, nn, pp]
                ps = psf[tt, nn, 0 if broadcast else pp]
                mk = None if mask is None else mask[tt, nn, pp]
                start_peakres = _peak_residual(d, mk)
                # without a mask both statistics are the same value
                start_peakres_nomask = start_peakres if mk is None else _peak_residual(d)
                start_model_flux = float(start_flux[tt, nn, pp]) if start_flux is not None \
                    else 0.0
                results, model_arr, resid_arr = hogbom_clean(
                    dirty_image=d, psf=ps, deconv_params=deconv_params, output_dir=output_dir,
                    progress=False)
                model_out[tt, nn, pp] = model_arr
                resid_out[tt, nn, pp] = resid_arr
                flux = float(K.plane_sum(model_arr).item())
                if model_arr.dtype == torch.float32:
                    flux = float(np.float32(flux))  # np.sum of a float32 plane
                peakres = _peak_residual(resid_out[tt, nn, pp], mk)
                peakres_nomask = peakres if mk is None else _peak_residual(resid_out[tt, nn, pp])
                rd.add({
                    "niter": deconv_params.get("niter", None),
                    "threshold": deconv_params.get("threshold", None),
                    "iter_done": results.get("iterations_performed", None),
                    "loop_gain": deconv_params.get("gain", None),
                    "min_psf_fraction": _MIN_PSF_FRACTION,
                    "max_psf_fraction": _MAX_PSF_FRACTION,
                    "max_psf_sidelobe": sidelobe,
                    "stop_code": None,
                    "stokes": np.asarray(pol_c[pp]),
                    "frequency": np.asarray(freq_c[nn]),
                    "phase_center": phase_center,
                    "time": np.asarray(time_c[tt]),
                    "start_model_flux": start_model_flux,
                    "model_flux": flux,
                    "start_peakres": start_peakres,
                    "start_peakres_nomask": start_peakres_nomask,
                    "peakres": peakres,
                    "peakres_nomask": peakres_nomask,
                    "masksum": masksum,
                }, time=tt, pol=pp, chan=nn)
    _put(full_model["MODEL"].values, model_out)
    _put(full_resid["RESIDUAL"].values, resid_out)
    return rd, full_model, full_resid
