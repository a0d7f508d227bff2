"""Mosaic / A-projection gridding on B200.

Drop-in for src/astroviper/core/imaging/imaging_utils/mosaic_grid.py:
mosaic_grid_jit (:307-486) and aperture_grid_jit (:13-153) update the
caller's grid and sum_weight in place, as the Numba kernels do, with the
arithmetic in libav200 (av_mosaic_grid, av_aperture_grid; the convolution
function times the phase gradient by av_cf_phase_product).
mosaic_grid_numpy_wrap and mosaic_psf_grid_numpy_wrap return fresh
(grid, sum_weight).

The reference's two wrappers do not run: numpy >= 1.24 has no np.int /
np.bool (:176, :180, :250, :254, :283), mosaic_grid_numpy_wrap passes 20
arguments to the 16-parameter aperture_grid_jit and mosaic_psf_grid_numpy_wrap
20 to the 18-parameter mosaic_grid_jit (field and field_id, which neither
kernel takes).  The wrappers here do what their arguments describe: they
grid vis_data (or, with do_psf, the weights) through mosaic_grid_jit.
"""
import numpy as np
import torch

from .... import _host as H
from .... import _kernels as K


def ndim_list(shape):
    """Nested lists of None with the given shape (mosaic_grid.py:8-9)."""
    return [ndim_list(shape[1:]) if len(shape) > 1 else None for _ in range(shape[0])]


def _grid_call(aperture, grid, sum_weight, do_psf, vis_data, uvw, freq_chan, chan_map, pol_map,
               cf_baseline_map, cf_chan_map, cf_pol_map, imaging_weight, conv_kernel, n_uv,
               delta_lm, weight_support, oversampling, phase_gradient):
    g = H.dev(grid)
    if not g.is_complex():
        raise TypeError("the grid must be complex: the convolution functions are complex")
    if g.dtype != torch.complex128:
        g = g.to(torch.complex128)
    sw = H.dev(sum_weight, torch.float64)
    pg = H.dev(phase_gradient)
    cf = K.cf_phase_product(H.dev(conv_kernel), pg[0])
    K.mosaic_grid(g, sw, do_psf, None if (do_psf or aperture) else H.dev(vis_data),
                  H.dev(imaging_weight), H.dev(uvw), np.asarray(freq_chan), chan_map, pol_map,
                  cf_baseline_map, cf_chan_map, cf_pol_map, cf, weight_support, n_uv, delta_lm,
                  oversampling, aperture=aperture)
    for dst, src in ((grid, g), (sum_weight, sw)):
        if H.is_torch(dst):
            if dst.data_ptr() != src.data_ptr():
                dst.copy_(src)
        else:
            H.write_back(dst, src)


def mosaic_grid_jit(grid, sum_weight, do_psf, vis_data, uvw, freq_chan, chan_map, pol_map,
                    cf_baseline_map, cf_chan_map, cf_pol_map, imaging_weight, conv_kernel, n_uv,
                    delta_lm, weight_support, oversampling, phase_gradient):
    """mosaic_grid.py:307-486: grid and sum_weight += every sample's window
    of conv_kernel x phase_gradient[0] (in place)."""
    _grid_call(False, grid, sum_weight, do_psf, vis_data, uvw, freq_chan, chan_map, pol_map,
               cf_baseline_map, cf_chan_map, cf_pol_map, imaging_weight, conv_kernel, n_uv,
               delta_lm, weight_support, oversampling, phase_gradient)


def aperture_grid_jit(grid, sum_weight, uvw, freq_chan, chan_map, pol_map, cf_baseline_map,
                      cf_chan_map, cf_pol_map, imaging_weight, conv_kernel_convolved, n_uv,
                      delta_lm, weight_support, oversampling, phase_gradient):
    """mosaic_grid.py:13-153: the weighted sum of the samples' functions at
    the grid centre (in place)."""
    _grid_call(True, grid, sum_weight, True, None, uvw, freq_chan, chan_map, pol_map,
               cf_baseline_map, cf_chan_map, cf_pol_map, imaging_weight, conv_kernel_convolved,
               n_uv, delta_lm, weight_support, oversampling, phase_gradient)


def _fresh(imaging_weight, grid_params):
    n_chan = imaging_weight.shape[2]
    if grid_params["chan_mode"] == "cube":
        n_imag_chan, chan_map = n_chan, np.arange(n_chan)
    else:
        n_imag_chan, chan_map = 1, np.zeros(n_chan, dtype=int)
    n_imag_pol = imaging_weight.shape[3]
    pol_map = np.arange(n_imag_pol)
    n_uv = grid_params["image_size_padded"]
    if not grid_params["complex_grid"]:
        raise TypeError("mosaic gridding needs complex_grid: the convolution functions are "
                        "complex")
    grid = np.zeros((n_imag_chan, n_imag_pol, int(n_uv[0]), int(n_uv[1])), dtype=np.complex128)
    sum_weight = np.zeros((n_imag_chan, n_imag_pol), dtype=np.double)
    return grid, sum_weight, chan_map, pol_map, n_uv


def mosaic_grid_numpy_wrap(vis_data, uvw, imaging_weight, field, cf_baseline_map, cf_chan_map,
                           cf_pol_map, conv_kernel, weight_support, phase_gradient, freq_chan,
                           grid_params):
    """mosaic_grid.py:156-227: fresh (grid, sum_weight) of vis_data (the
    weights with grid_params["do_psf"]).  field is accepted and unused, as
    in the kernels."""
    grid, sw, chan_map, pol_map, n_uv = _fresh(imaging_weight, grid_params)
    mosaic_grid_jit(grid, sw, grid_params["do_psf"], vis_data, uvw, freq_chan, chan_map, pol_map,
                    cf_baseline_map, cf_chan_map, cf_pol_map, imaging_weight, conv_kernel,
                    n_uv, grid_params["cell_size"], weight_support,
                    grid_params["oversampling"], phase_gradient)
    return grid, sw


def mosaic_psf_grid_numpy_wrap(uvw, imaging_weight, field, cf_baseline_map, cf_chan_map,
                               cf_pol_map, conv_kernel, weight_support, phase_gradient,
                               freq_chan, grid_params):
    """mosaic_grid.py:230-303: fresh (grid, sum_weight) of the weights
    (grid_params["do_psf"] as given: without it every sample is zero)."""
    grid, sw, chan_map, pol_map, n_uv = _fresh(imaging_weight, grid_params)
    if grid_params["do_psf"]:
        mosaic_grid_jit(grid, sw, True, None, uvw, freq_chan, chan_map, pol_map,
                        cf_baseline_map, cf_chan_map, cf_pol_map, imaging_weight, conv_kernel,
                        n_uv, grid_params["cell_size"], weight_support,
                        grid_params["oversampling"], phase_gradient)
    return grid, sw


def tree_sum_list(list_to_sum):
    """Pairwise sum of a list, in the reference's tree order
    (mosaic_grid.py:489-501); eager where the reference builds dask
    graphs.  Returns a one-element list."""
    while len(list_to_sum) > 1:
        nxt = []
        for i in range(0, len(list_to_sum), 2):
            nxt.append(list_to_sum[i] + list_to_sum[i + 1] if i < len(list_to_sum) - 1
                       else list_to_sum[i])
        list_to_sum = nxt
    return list_to_sum
