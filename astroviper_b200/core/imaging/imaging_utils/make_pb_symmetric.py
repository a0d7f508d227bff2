"""Symmetric (Airy-disk) primary beams on B200.

Drop-in for src/astroviper/core/imaging/imaging_utils/make_pb_symmetric.py:
airy_disk, casa_airy_disk, airy_disk_rorder and casa_airy_disk_rorder take
the reference's arguments (freq_chan, pol, pb_params, grid_params) and
return numpy arrays of the same layouts.  The beams are evaluated on the
device (av_airy_pattern) with the reference's operation order; J1 is CUDA's
j1, which agrees with scipy's jn(1, .) to a few ulp.
"""
import numpy as np

from .... import _kernels as K


def _beams(freq_chan, pol, pb_params, grid_params, casa, rorder):
    out = K.airy_pattern(freq_chan, len(pol), pb_params["list_dish_diameters"],
                         pb_params["list_blockage_diameters"], grid_params["image_size"],
                         grid_params["image_center"], grid_params["cell_size"],
                         pb_params["ipower"], casa, rorder)
    return out.cpu().numpy()


def airy_disk(freq_chan, pol, pb_params, grid_params):
    """(nx, ny, n_freq, n_pol, n_dish) beams (make_pb_symmetric.py:1-58)."""
    return _beams(freq_chan, pol, pb_params, grid_params, False, False)


def casa_airy_disk(freq_chan, pol, pb_params, grid_params):
    """As airy_disk with CASA's blockage formula (:61-125)."""
    return _beams(freq_chan, pol, pb_params, grid_params, True, False)


def airy_disk_rorder(freq_chan, pol, pb_params, grid_params):
    """(n_dish, n_freq, n_pol, nx, ny) beams (:128-190)."""
    return _beams(freq_chan, pol, pb_params, grid_params, False, True)


def casa_airy_disk_rorder(freq_chan, pol, pb_params, grid_params):
    """As airy_disk_rorder with CASA's blockage formula (:193-280)."""
    return _beams(freq_chan, pol, pb_params, grid_params, True, True)
