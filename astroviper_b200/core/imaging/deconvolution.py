"""hogbom_clean and its parameter validation on B200.

Drop-in for the Hogbom part of src/astroviper/core/imaging/deconvolution.py
(_validate_deconv_params :74-120, progress_callback :46-71, hogbom_clean
:332-426).  The image-level driver `deconvolve` (:123-329) iterates planes of
xarray image datasets and is outside this package; it calls hogbom_clean per
plane.
"""
import logging
from typing import Optional

import numpy as np

from .deconvolvers import hogbom

logger = logging.getLogger("astroviper_b200")


def progress_callback(iter_num: int, px: int, py: int, peak: float, niter_log: int = 100):
    """Logs the CLEAN progress every niter_log iterations (deconvolution.py:46)."""
    if iter_num % niter_log == 0:
        logger.info(f"  Iteration {iter_num}, peak at ({px}, {py}): {peak:.6f}")


def _validate_deconv_params(deconv_params):
    """deconvolution.py:74-120: fills defaults and checks gain, niter,
    threshold and clean_box (same ValueError messages)."""
    default_params = {
        "gain": 0.1,
        "niter": 1000,
        "threshold": 0.0,
        "clean_box": (-1, -1, -1, -1),
    }
    for key, default_value in default_params.items():
        if key not in deconv_params:
            logger.info(
                f"Deconvolution parameter '{key}' not specified. Using default: {default_value}")
            deconv_params[key] = default_value
        else:
            if key == "gain":
                if not (0 < deconv_params[key] <= 1):
                    raise ValueError("CLEAN gain must be between 0 and 1.")
            elif key == "niter":
                if not (isinstance(deconv_params[key], int) and deconv_params[key] > 0):
                    raise ValueError("Maximum number of iterations must be a positive integer.")
            elif key == "threshold":
                if deconv_params[key] is not None and deconv_params[key] < 0:
                    raise ValueError("Threshold must be non-negative or None.")
            elif key == "clean_box":
                if deconv_params[key] is not None and not (
                        isinstance(deconv_params[key], tuple) and len(deconv_params[key]) == 4):
                    raise ValueError(
                        "Clean box must be a 4-tuple (xmin, xmax, ymin, ymax) or None.")
    return deconv_params


def hogbom_clean(dirty_image: np.ndarray, psf: np.ndarray, deconv_params: Optional[dict] = None,
                 output_dir: str = "."):
    """deconvolution.py:332-426: returns (stats dict, model, residual) for one
    2-D plane."""
    deconv_params = _validate_deconv_params(deconv_params)
    if not isinstance(dirty_image, np.ndarray) or dirty_image.ndim != 2:
        raise ValueError("dirty_image must be a 2D numpy array with shape (ny, nx)")
    if not isinstance(psf, np.ndarray) or psf.ndim != 2:
        raise ValueError("psf must be a 2D numpy array with shape (ny, nx)")
    if dirty_image.shape != psf.shape:
        raise ValueError(
            f"dirty_image and psf must have same shape. Got {dirty_image.shape} and {psf.shape}")
    logger.debug(f"Dirty image shape: {dirty_image.shape}")
    logger.debug(f"PSF shape: {psf.shape}")
    fmin, fmax = hogbom.maximg(dirty_image)
    initial_peak = max(abs(fmin), abs(fmax))
    logger.debug(f"Initial peak flux: {initial_peak:.6f}")
    logger.info("\nRunning Hogbom CLEAN algorithm...")
    results = hogbom.clean(
        dirty_image=dirty_image,
        psf=psf,
        mask=np.array([], dtype=np.float32),
        gain=deconv_params["gain"],
        threshold=deconv_params["threshold"],
        max_iter=deconv_params["niter"],
        clean_box=(deconv_params["clean_box"] if deconv_params["clean_box"]
                   else (-1, -1, -1, -1)),
        progress_callback=progress_callback,
        stop_callback=None,
    )
    model_array = results["model_image"]
    residual_array = results["residual_image"]
    final_results = {k: v for k, v in results.items()
                     if k not in ["model_image", "residual_image"]}
    return final_results, model_array, residual_array
