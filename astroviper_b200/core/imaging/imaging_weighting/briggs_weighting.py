"""calculate_briggs_params (reference: src/astroviper/core/imaging/
imaging_weighting/briggs_weighting.py:1-31): sum(G^2) is reduced on the GPU
(av_briggs_factors)."""
import numpy as np
import torch

from .... import _host as H
from .... import _kernels as K


def calculate_briggs_params(grid_of_imaging_weights, sum_weight, imaging_weights_parms):
    """Returns briggs_factors (2, n_chan, n_pol) for "briggs" / "briggs_abs",
    else the reference's natural-weighting array."""
    if imaging_weights_parms["weighting"] == "briggs":
        bf = K.briggs_factors(H.dev(grid_of_imaging_weights, torch.float64),
                              H.dev(sum_weight, torch.float64), imaging_weights_parms["robust"])
        return H.host(bf, like=grid_of_imaging_weights)
    if imaging_weights_parms["weighting"] == "briggs_abs":
        robust = imaging_weights_parms["robust"]
        sw = np.asarray(sum_weight)
        bf = np.ones((2,) + sw.shape)
        bf[0, :, :] = bf[0, :, :] * np.square(robust)
        bf[1, :, :] = bf[1, :, :] * 2.0 * np.square(imaging_weights_parms["briggs_abs_noise"])
        return bf
    sw = np.asarray(sum_weight)
    bf = np.zeros((2, 1, 1) + sw.shape)
    bf[0, :, :] = np.ones((1, 1, 1) + sw.shape)
    return bf
