"""calculate_imaging_weights on B200.

Drop-in for src/astroviper/core/imaging/calculate_imaging_weights.py:28-275.
The arithmetic (flag -> NaN, polarisation averaging, nearest-cell density
grid with its conjugate, Briggs factors, per-sample imaging weights tiled to
every polarisation) runs in libav200 (av_weight_density, av_briggs_factors,
av_briggs_apply); the density grid stays on the device across the nodes of
the processing set.

The processing set is any mapping whose .values() are MSv4 nodes with UVW,
WEIGHT, FLAG data variables (``node[name].values``), a ``frequency``
coordinate and item assignment; xradio's DataTree is one.  Data-group
bookkeeping is kept to the keys the reference writes (names, date,
description); xradio's ``check_sel_params_ps_xdt`` is not reproduced.
"""
import copy
from datetime import datetime, timezone
from typing import Dict

import numpy as np
import torch

from ... import _host as H
from ... import _kernels as K


def _data_group_out(sel_params, weighting):
    out = {"uvw": "UVW", "weight": "WEIGHT", "flag": "FLAG",
           "weight_imaging": "WEIGHT" if weighting == "natural" else "WEIGHT_IMAGING"}
    out.update(sel_params.get("data_group_out", {}))
    out["data_group_out_name"] = sel_params.get("data_group_out_name", "imaging")
    return out


def _set_group(ms_xdt, name, group, description):
    groups = getattr(ms_xdt, "data_groups", None)
    if groups is None:
        return
    groups[name] = dict(group)
    groups[name]["date"] = datetime.now(timezone.utc).isoformat()
    groups[name]["description"] = description


def _array(x):
    return x.values if hasattr(x, "values") else np.asarray(x)


def calculate_imaging_weights(ps_xdt, grid_params: Dict, imaging_weights_params: Dict,
                              sel_params: Dict, return_weight_density_grid: bool = False):
    """Natural or Briggs imaging weights for every node of ps_xdt (see the
    module docstring).  Returns (ps_xdt, data_group_out) and, when asked, the
    (n_chan, 1, n_u, n_v) weight-density grid."""
    _sel = copy.deepcopy(sel_params)
    _iw = copy.deepcopy(imaging_weights_params)
    weighting = _iw.get("weighting")
    if weighting not in ("natural", "briggs", "briggs_abs"):
        raise AssertionError("######### ERROR: imaging_weights_params checking failed")
    group = _data_group_out(_sel, weighting)
    name = group.pop("data_group_out_name")
    nodes = list(ps_xdt.values())
    if weighting == "natural":
        for ms in nodes:
            _set_group(ms, name, group, "Data group created for natural imaging weights with .")
        group["data_group_out_name"] = name
        return ps_xdt, group
    n_uv = grid_params["image_size"]
    cell = grid_params["cell_size"]
    freq0 = _array(nodes[0].coords["frequency"]) if hasattr(nodes[0], "coords") else None
    nchan = len(freq0)
    dev = K.device()
    dens = torch.zeros((nchan, 1, int(n_uv[0]), int(n_uv[1])), dtype=torch.float64, device=dev)
    sw = torch.zeros((nchan, 1), dtype=torch.float64, device=dev)
    for ms in nodes:
        w = _array(ms[group["weight"]])
        fl = _array(ms[group["flag"]])
        w[fl == 1] = np.nan  # the reference flags its caller's WEIGHT in place
        K.weight_density(_array(ms[group["uvw"]]), _array(ms.coords["frequency"]), H.dev(w),
                         H.dev(fl), n_uv, cell, density=dens, sum_weight=sw)
    if weighting == "briggs":
        bf = K.briggs_factors(dens, sw, _iw["robust"])
    else:
        bf = torch.ones((2,) + tuple(sw.shape), dtype=torch.float64, device=dev)
        bf[0] *= float(np.square(_iw["robust"]))
        bf[1] *= 2.0 * float(np.square(_iw["briggs_abs_noise"]))
    description = ("Data group created for briggs imaging weights with robust value "
                   + str(_iw.get("robust")))
    for ms in nodes:
        w = _array(ms[group["weight"]])
        fl = _array(ms[group["flag"]])
        iw, err = K.briggs_apply(dens, bf.reshape(2, -1), _array(ms[group["uvw"]]),
                                 _array(ms.coords["frequency"]), H.dev(w), H.dev(fl), n_uv, cell)
        if int(err.item()):
            raise ValueError("NaN in briggs_factors")
        out = H.host(iw)
        try:
            import xarray as xr
            ms[group["weight_imaging"]] = xr.DataArray(out, dims=ms[group["weight"]].dims)
        except ImportError:
            ms[group["weight_imaging"]] = out
        _set_group(ms, name, group, description)
    group["data_group_out_name"] = name
    if return_weight_density_grid:
        return ps_xdt, group, H.host(dens)
    return ps_xdt, group
