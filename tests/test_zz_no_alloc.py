"""av_briggs_factors_noalloc, the allocation-free variant of av_briggs_factors
whose partial sums live in a static device array of the library: its factors
against those of av_briggs_factors with a caller workspace, bit for bit, on
two calls in a row (the second smaller than the first, so stale partials of
the first call would show); the device's free memory unchanged by a call; and
its rejection of a plane count above the static maximum."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from astroviper_b200 import _lib


def _max_planes():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, "include", "av200.h")).read()
    return int(re.search(r"#define AV_BRIGGS_NOALLOC_MAX_PLANES (\d+)", src).group(1))


def _density(seed, nplanes, n_u, n_v):
    """Density grids shaped like natural-weight counts: mostly empty cells,
    occupied ones with counts of a few to a few hundred."""
    rng = np.random.default_rng(seed)
    g = np.zeros((nplanes, n_u, n_v))
    occ = rng.uniform(size=g.shape) < 0.15
    g[occ] = np.floor(rng.gamma(0.6, 40.0, size=int(occ.sum()))) + 1.0
    sw = g.reshape(nplanes, -1).sum(axis=1) * rng.uniform(0.9, 1.1, size=nplanes)
    return (torch.as_tensor(g, device="cuda").contiguous(),
            torch.as_tensor(sw, device="cuda").contiguous())


def _with_workspace(L, d, sw, robust):
    from astroviper_b200 import _kernels as K
    npl, nu, nv = d.shape
    out = torch.empty((2, npl), dtype=torch.float64, device="cuda")
    _buf, wptr, wbytes = K.workspace(L.av_briggs_factors_workspace_size(npl))
    _lib.check(L.av_briggs_factors(d.data_ptr(), sw.data_ptr(), out.data_ptr(), npl, nu, nv,
                                   robust, wptr, wbytes, K.stream_ptr()), "av_briggs_factors")
    return out


def _no_alloc(L, d, sw, robust, out=None):
    from astroviper_b200 import _kernels as K
    npl, nu, nv = d.shape
    if out is None:
        out = torch.full((2, npl), np.nan, dtype=torch.float64, device="cuda")
    _lib.check(L.av_briggs_factors_noalloc(d.data_ptr(), sw.data_ptr(), out.data_ptr(), npl, nu,
                                           nv, robust, K.stream_ptr()),
               "av_briggs_factors_noalloc")
    return out


@pytest.mark.gpu
def test_no_alloc_factors_match_the_workspace_entry_point_twice():
    """Both entry points launch the same kernels over the same slices, so the
    factors must be bit-identical, on the first call and on the next."""
    L = _lib.lib()
    cases = [(1, (_max_planes(), 32, 48), 0.5), (2, (3, 300, 200), -1.0)]
    for seed, shape, robust in cases:
        d, sw = _density(seed, *shape)
        ref = _with_workspace(L, d, sw, robust)
        got = _no_alloc(L, d, sw, robust)
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert np.array_equal(g, r)


@pytest.mark.gpu
def test_no_alloc_call_takes_no_device_memory():
    """After a first call (which loads the kernels and looks up the array), a
    call leaves the device's free memory exactly as it was."""
    L = _lib.lib()
    d, sw = _density(3, 16, 64, 64)
    out = torch.full((2, 16), np.nan, dtype=torch.float64, device="cuda")
    _no_alloc(L, d, sw, 0.5, out)
    torch.cuda.synchronize()
    free0, _total = torch.cuda.mem_get_info()
    _no_alloc(L, d, sw, 0.5, out)
    torch.cuda.synchronize()
    free1, _total = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.all(np.isfinite(out.cpu().numpy()))


def test_no_alloc_rejects_more_planes_than_the_static_maximum():
    """The size check comes before any device work, so it runs without a GPU
    on host buffers that are never touched."""
    L = _lib.lib()
    m = _max_planes()
    buf = (ctypes.c_double * 4)()
    rc = L.av_briggs_factors_noalloc(buf, buf, buf, m + 1, 1, 1, 0.5, None)
    assert rc == _lib.AV_ERR_ARG
    msg = L.av_last_error().decode()
    assert f"maximum of {m} planes" in msg and "av_briggs_factors_noalloc" in msg
