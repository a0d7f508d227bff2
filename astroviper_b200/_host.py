"""Host <-> device staging for the numpy-facing drop-in functions."""
import numpy as np
import torch

from . import _kernels as K

_NP = {torch.float32: np.float32, torch.float64: np.float64, torch.complex64: np.complex64,
       torch.complex128: np.complex128, torch.int32: np.int32, torch.int64: np.int64,
       torch.bool: np.bool_, torch.uint8: np.uint8}


def is_torch(x):
    return isinstance(x, torch.Tensor)


def dev(x, dtype=None):
    """Array-like -> contiguous CUDA tensor (dtype conversion on the device)."""
    if is_torch(x):
        t = x.to(device=K.device(), non_blocking=True)
    else:
        a = np.asarray(x)
        if not a.flags.c_contiguous:
            a = np.ascontiguousarray(a)
        t = torch.from_numpy(a).to(device=K.device(), non_blocking=True) if a.dtype != object \
            else torch.as_tensor(a)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def host(t, like=None, dtype=None):
    """CUDA tensor -> numpy array in page-locked memory (or a tensor on like's
    device when like is a tensor)."""
    if like is not None and is_torch(like):
        return t.to(like.device)
    src = t.detach()
    if dtype is not None:
        src = src.to(_TORCH[np.dtype(dtype)])
    h = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
    h.copy_(src)
    return h.numpy()


_TORCH = {np.dtype(v): k for k, v in _NP.items()}


def streamable(*arrays, min_bytes=None):
    """True when every given array (None skipped) is a numpy array and
    together they hold at least two stream chunks: such inputs are copied to
    the device in time chunks that overlap the kernels (_kernels.grid_streamed,
    _kernels.degrid_streamed)."""
    given = [a for a in arrays if a is not None]
    if not given or not all(isinstance(a, np.ndarray) and a.ndim >= 2 for a in given):
        return False
    if len({a.shape[0] for a in given}) != 1:
        return False
    need = 2 * K.STREAM_CHUNK_BYTES if min_bytes is None else min_bytes
    return sum(a.nbytes for a in given) >= need


def write_back(dst, src_t):
    """Copy a device result into a caller's array in place."""
    if is_torch(dst):
        dst.copy_(src_t.to(dst.device, dst.dtype))
    elif dst.flags.c_contiguous and np.dtype(dst.dtype) in _TORCH:
        torch.from_numpy(dst).copy_(src_t.to(_TORCH[np.dtype(dst.dtype)]))
    else:
        dst[...] = src_t.detach().cpu().numpy().astype(dst.dtype, copy=False)
