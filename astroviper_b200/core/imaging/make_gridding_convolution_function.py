"""Convolution functions of the mosaic / A-projection gridder on B200.

Drop-in for the helpers of
src/astroviper/core/imaging/make_gridding_convolution_function.py:
make_baseline_patterns (:196-231), create_cf_baseline_map (:234-259),
create_cf_chan_map (:262-291), find_nearest (:294-297),
resize_and_calc_support (:300-377), calc_conv_size (:380-439) and
make_phase_gradient (:442-485), with their arguments, results and
assertion messages.  The beams and their products run on the device; the
maps and the support search are small host logic.  conv_kernels computes the
two Fourier transforms the reference's driver takes of the baseline patterns
(:111-127) with cuFFT.

The driver make_gridding_convolution_function (:24-193) reads the
measurement set through the accessors xradio gives an MSv4 dataset (any
object with the same attributes works) and returns an xarray Dataset when
xarray is installed, else the minimal dataset.Dataset.
make_phase_gradient uses the SIN projection directly, where the reference
asks astropy.wcs for it.
"""
import copy
import itertools

import numpy as np
import torch

from ... import _kernels as K
from ...utils.check_params import check_sel_params
from .check_imaging_parameters import check_gcf_params, check_grid_params
from .dataset import new_dataset


def _values(x):
    return np.asarray(getattr(x, "values", x))


def make_gridding_convolution_function(gcf_xds, ms_xds, gcf_params, grid_params, sel_params):
    """The A-projection convolution functions of one measurement set
    (make_gridding_convolution_function.py:24-193).  gcf_params gives the
    beam function (airy / casa_airy), the dish and blockage diameters per
    antenna type, each antenna's type (unique_ant_indx), the phase direction
    and the kernel oversampling / support limits; the frequencies,
    polarisations, baselines' antennas and field phase centre come from
    ms_xds.  When gcf_xds holds no variables, or another number of baselines,
    the kernels are built anew: per pair of antenna types and beam frequency
    the products of the two beams (and of their squares), Fourier transformed
    on the device, cropped to (max_support + 1) x oversampling and normalised
    (SUPPORT, CONV_KERNEL, CONV_KERNEL_CONVOLVED, PS_CORR_IMAGE, the
    baseline / channel / polarisation maps and the attributes cell_uv and
    oversampling).  PHASE_GRADIENT is always (re)made.  Returns the dataset;
    the caller's parameter dicts are left as they were."""
    _gcf_params = copy.deepcopy(gcf_params)
    _grid_params = copy.deepcopy(grid_params)
    _sel_params = copy.deepcopy(sel_params)
    data_group_in, _ = check_sel_params(ms_xds, _sel_params, default_data_group_in_name="base")
    _gcf_params["field_phase_dir"] = ms_xds.xr_ms.get_field_and_source_xds(
        data_group_in["data_group_in_name"]).FIELD_PHASE_CENTER_DIRECTION.isel(field_name=0)
    # each baseline's antennas as the reference finds them: the entries of
    # antenna x baseline name matches in row-major order
    names = _values(ms_xds.antenna_xds.antenna_name).ravel()
    ids = [np.where(names[:, None] == _values(b).ravel()[None, :])[0]
           for b in (ms_xds.baseline_antenna1_name, ms_xds.baseline_antenna2_name)]
    _gcf_params["basline_ant"] = np.array(ids).T
    _gcf_params["freq_chan"] = _values(ms_xds.frequency)
    _gcf_params["pol"] = _values(ms_xds.polarization)
    assert check_gcf_params(_gcf_params), "######### ERROR: gcf_params checking failed"
    assert check_grid_params(_grid_params), "######### ERROR: grid_params checking failed"
    _gcf_params["resize_conv_size"] = (_gcf_params["max_support"] + 1) * \
        _gcf_params["oversampling"]

    if len(gcf_xds) < 1 or gcf_xds.baseline.size != len(_gcf_params["basline_ant"]):
        from .imaging_utils.make_pb_symmetric import airy_disk_rorder, casa_airy_disk_rorder
        funcs = {"airy": airy_disk_rorder, "casa_airy": casa_airy_disk_rorder}
        assert _gcf_params["function"] in funcs, \
            "######### ERROR: Only airy and casa_airy function has been implemented"
        pb_func = funcs[_gcf_params["function"]]
        gcf_xds = new_dataset()
        cf_baseline_map, pb_ant_pairs = create_cf_baseline_map(
            _gcf_params["unique_ant_indx"], _gcf_params["basline_ant"],
            len(_gcf_params["list_dish_diameters"]))
        cf_chan_map, pb_freq = create_cf_chan_map(_gcf_params["freq_chan"],
                                                  _gcf_params["chan_tolerance_factor"])
        cf_pol_map = np.zeros((len(_gcf_params["pol"]),), dtype=int)  # one beam for all pols
        pb_pol = np.array([0])
        kernels = []
        for ipower in (1, 2):  # the beams, then their squares
            _gcf_params["ipower"] = ipower
            kernels.append(conv_kernels(make_baseline_patterns(
                pb_freq, pb_pol, pb_ant_pairs, pb_func, _gcf_params, _grid_params)))
        conv_kernel, conv_kernel_convolved, conv_support = resize_and_calc_support(
            kernels[0], kernels[1], _gcf_params, _grid_params)
        lead = ("conv_baseline", "conv_chan", "conv_pol")
        gcf_xds["SUPPORT"] = (lead + ("xy",), conv_support)
        gcf_xds["CONV_KERNEL_CONVOLVED"] = (lead + ("u", "v"), conv_kernel_convolved)
        gcf_xds["CONV_KERNEL"] = (lead + ("u", "v"), conv_kernel)
        gcf_xds["PS_CORR_IMAGE"] = (("l", "m"), np.ones(_grid_params["image_size"]))
        gcf_xds["CF_BASELINE_MAP"] = (("baseline",), cf_baseline_map)
        gcf_xds["CF_CHAN_MAP"] = (("chan",), cf_chan_map)
        gcf_xds["CF_POL_MAP"] = (("pol",), cf_pol_map)
        gcf_xds.attrs["cell_uv"] = 1 / (_grid_params["image_size_padded"] *
                                        _grid_params["cell_size"] * _gcf_params["oversampling"])
        gcf_xds.attrs["oversampling"] = _gcf_params["oversampling"]
        # the reference also builds u, v, xy, field_id, l, m coordinates here
        # but drops the dataset assign_coords returns, so none are attached

    field_phase_dir = np.array(getattr(_gcf_params["field_phase_dir"], "data",
                                       _gcf_params["field_phase_dir"]))
    gcf_xds["PHASE_GRADIENT"] = (("field_id", "u", "v"),
                                 make_phase_gradient(field_phase_dir[None, :], _gcf_params,
                                                     _grid_params))
    return gcf_xds


def make_baseline_patterns(pb_freq, pb_pol, pb_ant_pairs, pb_func, gcf_params, grid_params):
    """Products of the antennas' beams per pair (:196-231): (n_pairs,
    n_freq, n_pol, nx_padded, ny_padded) float64, beams evaluated on a grid of
    cell_size x oversampling."""
    pb_grid = dict(grid_params)
    pb_grid["cell_size"] = np.asarray(grid_params["cell_size"]) * gcf_params["oversampling"]
    pb_grid["image_size"] = np.asarray(pb_grid["image_size_padded"])
    pb_grid["image_center"] = pb_grid["image_size"] // 2
    patterns = torch.as_tensor(pb_func(pb_freq, pb_pol, gcf_params, pb_grid), device=K.device())
    nx, ny = int(grid_params["image_size_padded"][0]), int(grid_params["image_size_padded"][1])
    out = torch.zeros((len(pb_ant_pairs), len(pb_freq), len(pb_pol), nx, ny),
                      dtype=torch.float64, device=patterns.device)
    for k, pair in enumerate(pb_ant_pairs):
        out[k, :, 0] = patterns[int(pair[0]), :, 0] * patterns[int(pair[1]), :, 0]
    return out.cpu().numpy()


def conv_kernels(baseline_pb):
    """Re(fftshift(fft2(ifftshift(baseline_pb)))) over the last two axes
    (the driver's conv_kernel / conv_kernel_convolved, :111-127)."""
    t = K.fft_shifted(torch.as_tensor(np.asarray(baseline_pb), device=K.device()),
                      inverse=False)
    return t.real.contiguous().cpu().numpy()


def create_cf_baseline_map(unique_ant_indx, basline_ant, n_unique_ant):
    """Index of each baseline's antenna-type pair among the n(n+1)/2
    ordered pairs (i <= j), and the pairs (:234-259)."""
    pairs = np.array([[i, j] for i in range(n_unique_ant) for j in range(i, n_unique_ant)],
                     dtype=int).reshape(-1, 2)
    typ = np.stack([np.asarray(unique_ant_indx)[np.asarray(basline_ant)[:, 0]],
                    np.asarray(unique_ant_indx)[np.asarray(basline_ant)[:, 1]]], axis=1)
    cf_map = np.zeros(len(basline_ant), dtype=int)
    for k, (i, j) in enumerate(pairs):
        cf_map[(typ[:, 0] == i) & (typ[:, 1] == j)] = k
    return cf_map, pairs


def find_nearest(array, value):
    """(index, value) of the entry of array nearest to value (:294-297)."""
    array = np.asarray(array)
    idx = (np.abs(array - value)).argmin()
    return idx, array[idx]


def create_cf_chan_map(freq_chan, chan_tolerance_factor):
    """Channel -> beam-frequency map and the beam frequencies (:262-291):
    one beam per channel when the band is narrower than the tolerance
    allows, else band-centre frequencies of equal sub-bands."""
    freq_chan = np.asarray(freq_chan)
    n_chan = len(freq_chan)
    fmax, fmin = np.max(freq_chan), np.min(freq_chan)
    tol = fmax * chan_tolerance_factor
    n_pb_chan = int(np.floor((fmax - fmin) / tol) + 0.5)
    if n_pb_chan == 0:
        n_pb_chan = 1
    if n_pb_chan >= n_chan:
        return np.arange(n_chan), freq_chan
    width = (fmax - fmin) / n_pb_chan
    pb_freq = np.arange(n_pb_chan) * width + fmin + width / 2
    cf_map = np.zeros(n_chan, dtype=int)
    for i in range(n_chan):
        cf_map[i], _ = find_nearest(pb_freq, freq_chan[i])
    return cf_map, pb_freq


def calc_conv_size(sub_a_term, imsize, support_cut_level, oversampling, max_support):
    """Odd support (x, y) of one function: where it drops below
    support_cut_level x peak walking out from the centre along each axis
    (:380-439), made square."""
    a = np.abs(sub_a_term)
    peak = a[np.unravel_index(np.argmax(a), a.shape)]
    cut = support_cut_level * peak
    msg = "######### ERROR: support_cut_level too small or imsize too small."
    assert np.min(a) < cut, msg
    sizes = []
    for axis in (0, 1):
        ix, iy = imsize[0] // 2, imsize[1] // 2
        while sub_a_term[ix, iy] > cut:
            if axis == 0:
                ix += 1
                assert ix < imsize[0], msg
            else:
                iy += 1
                assert iy < imsize[1], msg
        walked = (ix - imsize[0] // 2) if axis == 0 else (iy - imsize[1] // 2)
        sizes.append((int(0.5 + walked / oversampling[axis]) + 1) * 2 + 1)
    sx, sy = sizes
    assert sx < max_support[0], msg + str(sx) + ",*," + str(max_support[0])
    assert sy < max_support[1], msg + str(sy) + ",*," + str(max_support[1])
    s = max(sx, sy)
    return [s, s]


def resize_and_calc_support(conv_kernel, conv_kernel_convolved, gcf_params, grid_params):
    """Centre crops of the kernels to resize_conv_size, each normalised to
    unit sum over its own support window per oversampling cell, and the
    supports (:300-377)."""
    lead = conv_kernel.shape[0:3]
    support = np.zeros(lead + (2,), dtype=int)
    rcs = np.asarray(gcf_params["resize_conv_size"])
    os_ = np.asarray(gcf_params["oversampling"])
    start = np.asarray(grid_params["image_size_padded"]) // 2 - rcs // 2
    end = start + rcs
    out_k = np.zeros(lead + tuple(rcs), dtype=np.double)
    out_kc = np.zeros(lead + tuple(rcs), dtype=np.double)
    for idx in itertools.product(*[range(s) for s in lead]):
        support[idx] = calc_conv_size(conv_kernel_convolved[idx],
                                      grid_params["image_size_padded"],
                                      gcf_params["support_cut_level"], os_,
                                      gcf_params["max_support"])
        emb = (support[idx] + 1) * os_
        e0 = rcs // 2 - emb // 2
        e1 = e0 + emb
        for src, dst in ((conv_kernel, out_k), (conv_kernel_convolved, out_kc)):
            dst[idx] = src[idx[0], idx[1], idx[2], start[0]:end[0], start[1]:end[1]]
            norm = np.real(np.sum(dst[idx[0], idx[1], idx[2], e0[0]:e1[0], e0[1]:e1[1]])
                           / (os_[0] * os_[1]))
            dst[idx] = dst[idx] / norm
    return out_k, out_kc, support


def _sin_world2pix(ra, dec, ra0, dec0, crpix, cdelt):
    """FITS-convention pixel coordinates (1-based) of (ra, dec) in a SIN
    projection about (ra0, dec0); all angles in radians, cdelt in radians."""
    # direction cosines (l toward increasing RA, m toward the north pole)
    # are the SIN projection's intermediate coordinates, in degrees; the
    # pixel offset is that over cdelt (RA---SIN / DEC--SIN, no rotation)
    dra = ra - ra0
    l = np.cos(dec) * np.sin(dra)
    m = np.sin(dec) * np.cos(dec0) - np.cos(dec) * np.sin(dec0) * np.cos(dra)
    return np.stack([np.degrees(l) / np.degrees(cdelt[0]) + crpix[0],
                     np.degrees(m) / np.degrees(cdelt[1]) + crpix[1]], axis=-1)


def make_phase_gradient(field_phase_dir, gcf_params, grid_params):
    """(n_field, conv_u, conv_v) complex phase ramps that move each field's
    phase centre onto the image's (:442-485)."""
    phase_center = np.asarray(getattr(gcf_params["phase_direction"], "values",
                                      gcf_params["phase_direction"]), dtype=float)
    pad = np.asarray(grid_params["image_size_padded"])
    crpix = pad // 2
    fpd = np.atleast_2d(np.asarray(field_phase_dir, dtype=float))
    pix = _sin_world2pix(fpd[:, 0], fpd[:, 1], phase_center[0], phase_center[1], crpix,
                         np.asarray(grid_params["cell_size"], dtype=float))
    dist = pix - crpix
    ramp = -dist * 2 * np.pi / (pad * np.asarray(gcf_params["oversampling"]))
    size = np.asarray(gcf_params["resize_conv_size"])
    c = size // 2
    x = np.arange(-c[0], size[0] - c[0])
    y = np.arange(-c[1], size[1] - c[1])
    xg, yg = np.meshgrid(x, y, indexing="ij")
    pg = np.exp(1j * (xg[:, :, None] * ramp[:, 0] + yg[:, :, None] * ramp[:, 1]))
    return np.moveaxis(pg, 2, 0)
