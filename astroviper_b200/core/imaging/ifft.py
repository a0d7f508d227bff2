"""ifft_uv_to_lm (reference: src/astroviper/core/imaging/ifft.py:5-18) on cuFFT."""
from typing import List

import numpy as np

from ... import _host as H
from .fft import _centred


def ifft_uv_to_lm(ary: np.ndarray, axes: List[int]) -> np.ndarray:
    """fftshift(ifft2(ifftshift(ary, axes), axes), axes).real"""
    out = _centred(ary, list(axes), inverse=True).real.contiguous()
    return H.host(out, like=ary)
