"""Correlation products <-> Stokes parameters on B200.

Drop-in for src/astroviper/core/imaging/imaging_utils/corr_to_stokes.py: same
functions, arguments, defaults, validation messages and result dtypes.  The
per-pixel products run in libav200 (av_pol_transform, one complex 4x4 or
smaller matrix applied to every pixel in place of numpy's matmul after a
moveaxis).  The transformation tables are the standard linear / circular
feed relations (I = XX + YY, XX = (I + Q) / 2, ...) exactly as the reference
defines them, since they fix the scale of every Stokes image it produces.

numpy input gives numpy output; torch tensors stay on the device.  xarray
DataArrays are accepted when xarray is installed.
"""
from typing import List, Optional

import numpy as np
import torch

from .... import _host as H
from .... import _kernels as K

VALID_STOKES = {"I", "Q", "U", "V"}
STOKES_FROM_2POL_LINEAR = {"I", "Q"}
STOKES_FROM_2POL_CIRCULAR = {"I", "V"}

CORR_TYPE_MAP = {
    frozenset({"XX", "XY", "YX", "YY"}): "linear",
    frozenset({"RR", "RL", "LR", "LL"}): "circular",
    frozenset({"XX", "YY"}): "linear",
    frozenset({"RR", "LL"}): "circular",
}

# rows: I, Q, U, V from (XX, XY, YX, YY) / (RR, RL, LR, LL)
LINEAR_CORR_TO_STOKES = np.array([[1, 0, 0, 1],
                                  [1, 0, 0, -1],
                                  [0, 1, 1, 0],
                                  [0, -1j, 1j, 0]], dtype=complex)
CIRCULAR_CORR_TO_STOKES = np.array([[1, 0, 0, 1],
                                    [0, 1, 1, 0],
                                    [0, -1j, 1j, 0],
                                    [1, 0, 0, -1]], dtype=complex)
# rows: XX, XY, YX, YY / RR, RL, LR, LL from (I, Q, U, V)
LINEAR_STOKES_TO_CORR = np.array([[0.5, 0.5, 0, 0],
                                  [0, 0, 0.5, 0.5j],
                                  [0, 0, 0.5, -0.5j],
                                  [0.5, -0.5, 0, 0]], dtype=complex)
CIRCULAR_STOKES_TO_CORR = np.array([[0.5, 0, 0, 0.5],
                                    [0, 0.5, 0.5j, 0],
                                    [0, 0.5, -0.5j, 0],
                                    [0.5, 0, 0, -0.5]], dtype=complex)

_STOKES_INDEX = {"I": 0, "Q": 1, "U": 2, "V": 3}


def _xr_dataarray():
    try:
        import xarray
        return xarray.DataArray
    except Exception:
        return None


def _table(corr_type, transformation_matrix, linear, circular):
    if transformation_matrix is not None:
        return np.asarray(transformation_matrix, dtype=complex)
    if corr_type == "linear":
        return linear
    if corr_type == "circular":
        return circular
    raise ValueError("For 'custom' corr_type, a transformation_matrix must be provided.")


def _apply(data, matrix, axis, out_dtype):
    """matrix applied along axis of data (numpy or device tensor)."""
    out = K.pol_transform(H.dev(data), matrix, axis, out_dtype)
    return out if H.is_torch(data) else H.host(out)


def corr_to_stokes(data, corr_type: str = "linear",
                   transformation_matrix: Optional[np.ndarray] = None):
    """data (..., 4) correlations -> (..., 4) Stokes, complex
    (corr_to_stokes.py:71-103)."""
    m = _table(corr_type, transformation_matrix, LINEAR_CORR_TO_STOKES,
               CIRCULAR_CORR_TO_STOKES)
    return _apply(data, m, -1, torch.complex128)


def stokes_to_corr(data, corr_type: str = "linear",
                   transformation_matrix: Optional[np.ndarray] = None):
    """data (..., 4) Stokes -> (..., 4) correlations, complex
    (corr_to_stokes.py:106-138)."""
    m = _table(corr_type, transformation_matrix, LINEAR_STOKES_TO_CORR,
               CIRCULAR_STOKES_TO_CORR)
    return _apply(data, m, -1, torch.complex128)


def _is_real(data):
    if H.is_torch(data):
        return not data.is_complex()
    return not np.iscomplexobj(data)


def image_corr_to_stokes(image_data, corr_type: Optional[str] = None, pol_axis: int = 2,
                         stokes_out: Optional[List[str]] = None,
                         transformation_matrix: Optional[np.ndarray] = None):
    """Correlation image -> Stokes image along pol_axis
    (corr_to_stokes.py:141-305).  Real input gives float64 Stokes, complex
    input complex128."""
    DA = _xr_dataarray()
    is_xr = DA is not None and isinstance(image_data, DA)
    data = image_data.values if is_xr else image_data
    if corr_type is None:
        if not is_xr:
            raise ValueError(
                "corr_type is required for numpy input. "
                "Use xarray DataArray with labeled polarization coordinates for auto-detection.")
        corr_type = _detect_corr_type(image_data, pol_axis)
    ndim = len(data.shape)
    ax = pol_axis + ndim if pol_axis < 0 else pol_axis
    n_corr = int(data.shape[ax])
    if n_corr < 2:
        raise ValueError(f"Minimum 2 correlations required for Stokes conversion, got {n_corr}")
    if stokes_out is None:
        if n_corr == 2:
            if corr_type == "linear":
                stokes_out = ["I", "Q"]
            elif corr_type == "circular":
                stokes_out = ["I", "V"]
            else:
                raise ValueError(
                    f"2-pol conversion requires corr_type 'linear' or 'circular', got "
                    f"'{corr_type}'")
        else:
            stokes_out = ["I", "Q", "U", "V"]
    wanted = set(stokes_out)
    bad = wanted - VALID_STOKES
    if bad:
        raise ValueError(f"Invalid Stokes parameters: {bad}. Valid: {VALID_STOKES}")
    if n_corr == 2 and corr_type in ("linear", "circular"):
        have = STOKES_FROM_2POL_LINEAR if corr_type == "linear" else STOKES_FROM_2POL_CIRCULAR
        missing = wanted - have
        if missing:
            pair = "(XX, YY)" if corr_type == "linear" else "(RR, LL)"
            raise ValueError(
                f"2-pol {corr_type} data {pair} cannot produce Stokes {missing}. "
                f"Only {have} available.")
    full = _table(corr_type, transformation_matrix, LINEAR_CORR_TO_STOKES,
                  CIRCULAR_CORR_TO_STOKES)
    if n_corr == 2:
        # [XX, YY] is [XX, 0, 0, YY]: only the first and last columns act
        full = full[:, [0, 3]]
    if wanted == set(VALID_STOKES):
        stokes_out = ["I", "Q", "U", "V"]
    m = full[[_STOKES_INDEX[s] for s in stokes_out], :]
    out_dtype = torch.float64 if _is_real(data) else torch.complex128
    result = _apply(data, m, ax, out_dtype)
    if is_xr:
        coords = dict(image_data.coords)
        coords[image_data.dims[pol_axis]] = stokes_out
        return DA(result, dims=image_data.dims, coords=coords, attrs=image_data.attrs)
    return result


def image_stokes_to_corr(image_data, corr_type: str = "linear", pol_axis: int = 2,
                         stokes_in: Optional[List[str]] = None, corr_out: Optional[int] = None,
                         transformation_matrix: Optional[np.ndarray] = None):
    """Stokes image -> correlation image along pol_axis
    (corr_to_stokes.py:307-487).  Two-correlation output keeps the input
    dtype; four-correlation output is complex128."""
    DA = _xr_dataarray()
    is_xr = DA is not None and isinstance(image_data, DA)
    data = image_data.values if is_xr else image_data
    ndim = len(data.shape)
    ax = pol_axis + ndim if pol_axis < 0 else pol_axis
    n_stokes = int(data.shape[ax])
    if stokes_in is None:
        if n_stokes == 4:
            stokes_in = ["I", "Q", "U", "V"]
        elif n_stokes == 2:
            if corr_type == "linear":
                stokes_in = ["I", "Q"]
            elif corr_type == "circular":
                stokes_in = ["I", "V"]
            else:
                raise ValueError(
                    f"2-Stokes conversion requires corr_type 'linear' or 'circular', got "
                    f"'{corr_type}'")
        elif n_stokes == 1:
            stokes_in = ["I"]
        else:
            raise ValueError(f"Unexpected number of Stokes parameters: {n_stokes}")
    elif len(stokes_in) != n_stokes:
        raise ValueError(
            f"stokes_in length ({len(stokes_in)}) doesn't match input polarization "
            f"dimension size ({n_stokes})")
    bad = set(stokes_in) - VALID_STOKES
    if bad:
        raise ValueError(f"Invalid Stokes parameters: {bad}. Valid: {VALID_STOKES}")
    if corr_out is None:
        corr_out = 4 if n_stokes == 4 else 2
    if corr_out not in (2, 4):
        raise ValueError(f"corr_out must be 2 or 4, got {corr_out}")
    if corr_out == 4 and n_stokes < 4:
        raise ValueError(
            f"Cannot produce 4-pol output from {n_stokes}-Stokes input. "
            "Need U, V for cross-polarizations (XY, YX or RL, LR).")
    if corr_out == 2:
        if corr_type not in ("linear", "circular"):
            raise ValueError(
                f"2-pol output requires corr_type 'linear' or 'circular', got '{corr_type}'")
        pos = {s: i for i, s in enumerate(stokes_in)}
        if "I" not in pos:
            raise ValueError(f"Cannot convert to {corr_type} correlations without Stokes I")
        partner = "Q" if corr_type == "linear" else "V"
        # (I + P) / 2 and (I - P) / 2, or I / 2 twice for Stokes I alone
        m = np.zeros((2, n_stokes), dtype=complex)
        m[:, pos["I"]] = 0.5
        if partner in pos:
            m[0, pos[partner]] = 0.5
            m[1, pos[partner]] = -0.5
        src = data if H.is_torch(data) else np.asarray(data)
        tdt = src.dtype if H.is_torch(src) else H._TORCH.get(np.dtype(src.dtype), torch.float64)
        result = _apply(data, m, ax, tdt)
    else:
        full = _table(corr_type, transformation_matrix, LINEAR_STOKES_TO_CORR,
                      CIRCULAR_STOKES_TO_CORR)
        result = _apply(data, full, ax, torch.complex128)
    if corr_type == "linear":
        labels = ["XX", "XY", "YX", "YY"] if corr_out == 4 else ["XX", "YY"]
    elif corr_type == "circular":
        labels = ["RR", "RL", "LR", "LL"] if corr_out == 4 else ["RR", "LL"]
    else:
        labels = [f"CORR{i}" for i in range(corr_out)]
    if is_xr:
        coords = dict(image_data.coords)
        coords[image_data.dims[pol_axis]] = labels
        return DA(result, dims=image_data.dims, coords=coords, attrs=image_data.attrs)
    return result


def _expand_to_4stokes(data: np.ndarray, stokes_in: List[str]) -> np.ndarray:
    """Partial Stokes (..., k) -> (..., 4) in I, Q, U, V order, zeros where
    missing."""
    out = np.zeros(tuple(data.shape[:-1]) + (4,), dtype=data.dtype)
    for i, s in enumerate(stokes_in):
        out[..., _STOKES_INDEX[s]] = data[..., i]
    return out


def _expand_to_4corr(data: np.ndarray, corr_type: str) -> np.ndarray:
    """(..., 2) parallel hands -> (..., 4) with zero cross hands."""
    out = np.zeros(tuple(data.shape[:-1]) + (4,), dtype=data.dtype)
    out[..., 0] = data[..., 0]
    out[..., 3] = data[..., 1]
    return out


def _detect_corr_type(image_data, pol_axis: int) -> str:
    """'linear' / 'circular' from the polarisation coordinate labels."""
    name = image_data.dims[pol_axis]
    labels = frozenset(str(v) for v in image_data.coords[name].values)
    corr_type = CORR_TYPE_MAP.get(labels)
    if corr_type is None:
        raise ValueError(
            f"Cannot detect corr_type from polarization values: {set(labels)}. "
            f"Expected one of: {[set(k) for k in CORR_TYPE_MAP.keys()]}")
    return corr_type
