"""fft_lm_to_uv (reference: src/astroviper/core/imaging/fft.py:5-18) on cuFFT."""
from typing import List

import numpy as np

from ... import _host as H
from ... import _kernels as K


def _centred(ary, axes, inverse):
    axes = [a % np.ndim(ary) for a in axes]
    if len(axes) != 2:
        raise ValueError("axes must name two axes")
    t = H.dev(ary)
    if not t.is_complex():
        t = t.to(K.torch.complex128 if t.dtype != K.torch.float32 else K.torch.complex64)
    last = [t.ndim - 2, t.ndim - 1]
    moved = axes != last
    if moved:
        t = t.movedim(axes, last).contiguous()
    out = K.fft_shifted(t, inverse=inverse)
    if moved:
        out = out.movedim(last, axes).contiguous()
    return out


def fft_lm_to_uv(ary: np.ndarray, axes: List[int]) -> np.ndarray:
    """fftshift(fft2(ifftshift(ary, axes), axes), axes): complex result."""
    out = _centred(ary, list(axes), inverse=False)
    return H.host(out, like=ary)
