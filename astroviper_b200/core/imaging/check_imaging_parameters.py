"""Grid and convolution-function parameter checks.

Drop-in for src/astroviper/core/imaging/check_imaging_parameters.py:
check_grid_params (:7-75) and check_gcf_params (:78-221).  Each is a table of
check_params calls, run in the reference's order (so the same messages print
and the same defaults are written), followed by the reference's conversions
to arrays when every check passes.
"""
import numbers

import numpy as np

from ...utils.check_params import check_params

_NUMS = [list, np.array]


def _run(params, table):
    ok = True
    for key, types, kw in table:
        ok = check_params(params, key, types, **kw) and ok
    return ok


def check_grid_params(grid_params):
    """image_size and cell_size (2-lists), image_center (default
    image_size // 2), fft_padding in [1, 10] (default 1.2), chan_mode cube or
    continuum (default cube); then image_size, image_size_padded =
    int(fft_padding * image_size) and image_center as arrays."""
    table = [
        ("image_size", [list], dict(list_acceptable_data_types=[int], list_len=2)),
        ("image_center", [list], dict(list_acceptable_data_types=[int], list_len=2,
                                      default=np.array(grid_params["image_size"]) // 2)),
        ("cell_size", [list], dict(list_acceptable_data_types=[numbers.Number], list_len=2)),
        ("fft_padding", [numbers.Number], dict(default=1.2, acceptable_range=[1, 10])),
        ("chan_mode", [str], dict(acceptable_data=["cube", "continuum"], default="cube")),
    ]
    ok = _run(grid_params, table)
    if ok:
        grid_params["image_size"] = np.array(grid_params["image_size"]).astype(int)
        grid_params["image_size_padded"] = (grid_params["fft_padding"] *
                                            grid_params["image_size"]).astype(int)
        grid_params["image_center"] = np.array(grid_params["image_center"])
    return ok


def check_gcf_params(gcf_params):
    """function (airy / casa_airy), the per-channel frequencies, dish and
    blockage diameters (equal lengths), antenna-type indices and
    polarisations, chan_tolerance_factor (0.005), oversampling ([10, 10]),
    max_support ([15, 15]), support_cut_level (0.025), a_chan_num_chunk (3);
    then the list entries as arrays."""
    seq = dict(list_acceptable_data_types=[numbers.Number], list_len=-1)
    table = [
        ("function", [str], dict(acceptable_data=["casa_airy", "airy"], default="casa_airy")),
        ("freq_chan", _NUMS, seq),
        ("list_dish_diameters", _NUMS, seq),
        ("list_blockage_diameters", _NUMS, seq),
        ("unique_ant_indx", _NUMS, seq),
        ("pol", _NUMS, dict(list_acceptable_data_types=[numbers.Number, str], list_len=-1)),
        ("chan_tolerance_factor", [numbers.Number], dict(default=0.005)),
        ("oversampling", _NUMS, dict(list_acceptable_data_types=[int], list_len=2,
                                     default=[10, 10])),
        ("max_support", _NUMS, dict(list_acceptable_data_types=[int], list_len=2,
                                    default=[15, 15])),
        ("support_cut_level", [numbers.Number], dict(default=2.5 * 10**-2)),
        ("a_chan_num_chunk", [int], dict(default=3)),
    ]
    ok = _run(gcf_params, table)
    if gcf_params["function"] in ("airy", "casa_airy"):
        ok = _run(gcf_params, [("list_dish_diameters", _NUMS, seq),
                               ("list_blockage_diameters", _NUMS, seq)]) and ok
        if len(gcf_params["list_dish_diameters"]) != len(gcf_params["list_blockage_diameters"]):
            print("######### ERROR:Parameter ",
                  "list_dish_diameters and list_blockage_diameters must be the same length.")
            ok = False
    if ok:
        for key in ("oversampling", "max_support"):
            gcf_params[key] = np.array(gcf_params[key]).astype(int)
        for key in ("freq_chan", "list_dish_diameters", "list_blockage_diameters",
                    "unique_ant_indx", "pol"):
            gcf_params[key] = np.array(gcf_params[key])
    return ok
