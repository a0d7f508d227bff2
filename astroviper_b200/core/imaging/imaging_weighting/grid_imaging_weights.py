"""Imaging-weight density grid and its degridding on B200.

Drop-in for src/astroviper/core/imaging/imaging_weighting/grid_imaging_weights.py
(av_weight_density / av_briggs_apply).  In-place behaviour of the reference
is kept: grid and sum_weight are accumulated into the caller's arrays.
"""
import numpy as np
import torch

from .... import _host as H
from .... import _kernels as K


def grid_imaging_weights(grid, sum_weight, uvw, data_weight, freq_chan, grid_parms):
    """grid_imaging_weights.py:6-88: weights (n_time, n_baseline, n_chan,
    n_pol <= 2, pol 0 used) onto the nearest cell and its conjugate."""
    assert data_weight.shape[3] < 3, "Polarization should be PP or PP, QQ."
    n_chan = data_weight.shape[2]
    grid_imaging_weights_jit(grid, sum_weight, uvw, freq_chan, np.arange(0, n_chan).astype(int),
                             data_weight, grid_parms["image_size"], grid_parms["cell_size"])


def grid_imaging_weights_jit(grid, sum_weight, uvw, freq_chan, chan_map, data_weights, n_uv,
                             delta_lm):
    """grid_imaging_weights.py:93-206 (pol 0 of data_weights, identity
    channel map as the wrapper passes)."""
    cm = np.asarray(chan_map)
    if not np.array_equal(cm, np.arange(len(cm))):
        raise NotImplementedError("only the identity channel map of the reference wrapper")
    w = H.dev(data_weights)[..., :1].contiguous()
    if w.dtype not in (torch.float32, torch.float64):
        w = w.to(torch.float64)
    G = H.dev(grid, torch.float64)
    sw = H.dev(sum_weight, torch.float64)
    # the kernel grids into (n_chan, 1, n_u, n_v) planes: plane c = grid[c, 0]
    dens = G[:, 0:1].contiguous()
    swc = sw[:, 0:1].contiguous()
    K.weight_density(uvw, freq_chan, w, None, n_uv, delta_lm, density=dens, sum_weight=swc)
    G[:, 0:1] = dens
    sw[:, 0:1] = swc
    H.write_back(grid, G)
    H.write_back(sum_weight, sw)


def degrid_imaging_weights(grid_imaging_weight, uvw, data_weight, briggs_factors, freq_chan,
                           grid_parms):
    """grid_imaging_weights.py:209-282: per-sample imaging weights (float64,
    shape of data_weight; single-pol degrid as the reference)."""
    n_imag_chan = data_weight.shape[2]
    imaging_weight = np.zeros(data_weight.shape, dtype=np.double)
    degrid_imaging_weights_jit(imaging_weight, grid_imaging_weight, briggs_factors, uvw,
                               freq_chan, np.arange(0, n_imag_chan).astype(int),
                               np.arange(0, 1).astype(int), data_weight,
                               grid_parms["image_size"], grid_parms["cell_size"])
    return imaging_weight


def degrid_imaging_weights_jit(imaging_weight, grid_imaging_weight, briggs_factors, uvw,
                               freq_chan, chan_map, pol_map, data_weight, n_uv, delta_lm):
    """grid_imaging_weights.py:285-443 for the reference wrapper's maps
    (identity channels, pol_map [0]): pol 0 of each sample is written."""
    if not np.array_equal(np.asarray(pol_map), np.arange(1)):
        raise NotImplementedError("only pol_map [0] of the reference wrapper")
    w = H.dev(data_weight)[..., :1].contiguous()
    if w.dtype not in (torch.float32, torch.float64):
        w = w.to(torch.float64)
    G = H.dev(grid_imaging_weight, torch.float64)
    bf = H.dev(briggs_factors, torch.float64).reshape(2, -1)
    # factors for (chan, pol 0)
    bf0 = bf.reshape(2, G.shape[0], -1)[:, :, 0].contiguous()
    out, err = K.briggs_apply(G[:, 0:1].contiguous(), bf0.reshape(2, -1), uvw, freq_chan, w,
                              None, n_uv, delta_lm)
    if int(err.item()):
        raise ValueError("NaN in briggs_factors")
    iw = H.dev(imaging_weight, torch.float64)
    iw[..., 0:1] = out
    H.write_back(imaging_weight, iw)
