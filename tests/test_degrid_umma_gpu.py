"""The tensor-memory degridder (AV_DEGRID_LANES_TC05, k_degrid_umma).

Tiles of up to 128 records of one cell go through one tcgen05 MMA chain
each, with accumulators in tensor memory; these tests run it on long runs
(the 33M-sample workload's continuum grid), on short runs and runs that end
at every position of a tile (a dense uv distribution), on small chunks (many
segments per warpgroup), on a shared plan with exception samples, and check
it against the FP64 plain degridder (the reference's arithmetic,
standard_degrid.py:388-485) and against the warp-MMA kernel k_degrid_tc.
Every launch must leave the bounded-wait fault flag clear.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _set(knob, value):
    from astroviper_b200 import _lib
    L = _lib.lib()
    old = L.av_tune_get(knob)
    assert L.av_tune_set(knob, value) == _lib.AV_OK
    return old


def _fault():
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import _lib
    out = ctypes.c_int(-1)
    _lib.check(_lib.lib().av_degrid_fault_read(ctypes.byref(out), 1, K.stream_ptr()),
               "av_degrid_fault_read")
    return out.value


def _both(G, grid, **kw):
    """G.degrid under the tensor-memory kernel and under k_degrid_tc."""
    from astroviper_b200 import _lib
    old = _set(_lib.AV_TUNE_DEGRID_LANES, _lib.AV_DEGRID_LANES_TC05)
    try:
        v5 = G.degrid(grid, **kw).clone()
        torch.cuda.synchronize()
        _set(_lib.AV_TUNE_DEGRID_LANES, _lib.AV_DEGRID_LANES_TF32)
        vt = G.degrid(grid, **kw).clone()
    finally:
        _set(_lib.AV_TUNE_DEGRID_LANES, old)
    assert _fault() == 0
    return v5, vt


def _fp64(G, grid, uvw, freq, cell, nx, ny, nchan, npol):
    from astroviper_b200 import _kernels as K
    return K.degrid(grid, uvw, freq, (-cell[0] * nx, -cell[1] * ny), (nx / 2, ny / 2),
                    np.zeros(nchan, int), np.arange(npol), G.cgk, G.support, G.os,
                    nvchan=nchan, nvpol=npol, precision="fp64")


def test_fault_flag_reads_clear():
    assert _fault() == 0


@pytest.mark.parametrize("chunks_per_sm", [16, 512])
def test_long_runs_match_fp64_and_warp_mma(chunks_per_sm):
    """8 time steps of the 33M-sample workload (continuum 2048^2, 64
    channels, 4 polarisations): runs of hundreds of samples per cell; with
    512 chunks per SM the chunks are small, so segments and warpgroup slices
    start and end inside runs."""
    from astroviper_b200 import _lib
    from astroviper_b200 import synthetic as S
    from astroviper_b200.gridder import Gridder
    W = S.workload_large(n_time=8, device=torch.device("cuda"))
    nt, nb, nchan, npol = W["vis"].shape
    G = Gridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], npol)
    g, _ = G.grid(W["vis"], torch.ones(W["vis"].shape, dtype=torch.float32, device="cuda"))
    old = _set(_lib.AV_TUNE_DEGRID_CHUNKS_PER_SM, chunks_per_sm)
    try:
        v5, vt = _both(G, g)
    finally:
        _set(_lib.AV_TUNE_DEGRID_CHUNKS_PER_SM, old)
    nx, ny = (int(x) for x in W["image_size"])
    ref = _fp64(G, g, W["uvw"], W["freq"], W["pixelincr"], nx, ny, nchan, npol)
    assert rel(v5, ref) <= 1e-6
    assert rel(v5, vt) <= 5e-7


def _dense_case(seed, n=256, nt=12, nb=500, nchan=4):
    """uv positions: 40 % within 0.1 cell of a few centres (long runs), 30 %
    within a cell (runs of a few), 30 % spread over the grid (runs of one)."""
    rng = np.random.default_rng(seed)
    cell = np.array([-2.0, 2.0]) * np.pi / (180 * 3600)
    freq = np.linspace(1.4e9, 1.5e9, nchan)
    us = -(freq[0] * cell[0] * n) / 299792458.0
    vs = -(freq[0] * cell[1] * n) / 299792458.0
    m = nt * nb
    kind = rng.uniform(size=m)
    centres = rng.integers(-n // 4, n // 4, size=(8, 2)).astype(float)
    pick = rng.integers(0, 8, size=m)
    pu = np.where(kind < 0.4, centres[pick, 0] + rng.normal(0, 0.1, m),
                  np.where(kind < 0.7, centres[pick, 0] + rng.normal(0, 1.0, m),
                           rng.uniform(-0.4, 0.4, m) * n))
    pv = np.where(kind < 0.4, centres[pick, 1] + rng.normal(0, 0.1, m),
                  np.where(kind < 0.7, centres[pick, 1] + rng.normal(0, 1.0, m),
                           rng.uniform(-0.4, 0.4, m) * n))
    uvw = np.stack([pu / us, pv / vs, rng.uniform(-50, 50, m)], axis=-1).reshape(nt, nb, 3)
    uvw[0, 3, 0] = np.nan            # skipped: NaN position
    uvw[1, 7, :2] *= 1e4             # skipped: off the grid
    return uvw, freq, cell, n


@pytest.mark.parametrize("seed", [1, 2])
def test_short_and_ragged_runs(seed):
    """A dense case whose runs have every length from 1 up: tiles end at the
    third cell, so slots of one sample, tiles of two cells and full tiles
    all occur; against the FP64 degridder and k_degrid_tc."""
    from astroviper_b200.gridder import Gridder
    uvw, freq, cell, n = _dense_case(seed)
    nt, nb = uvw.shape[:2]
    nchan, npol = len(freq), 4
    G = Gridder(uvw, freq, np.array([n, n]), cell, npol, support=7, oversampling=100)
    rng = np.random.default_rng(seed + 10)
    gshape = (1, npol, n, n)
    grid = torch.as_tensor(rng.normal(size=gshape) + 1j * rng.normal(size=gshape),
                           device="cuda")
    v5, vt = _both(G, grid)
    ref = _fp64(G, grid, uvw, freq, cell, n, n, nchan, npol)
    assert rel(v5, ref) <= 1e-6
    assert rel(v5, vt) <= 5e-7
    # the skipped samples are zeros
    assert bool((v5[0, 3] == 0).all()) and bool((v5[1, 7] == 0).all())


@pytest.mark.parametrize("support", [3, 4, 5, 6, 8])
def test_other_supports(support):
    from astroviper_b200.gridder import Gridder
    uvw, freq, cell, n = _dense_case(7, nt=6)
    nchan, npol = len(freq), 4
    G = Gridder(uvw, freq, np.array([n, n]), cell, npol, support=support, oversampling=100)
    rng = np.random.default_rng(support)
    gshape = (1, npol, n, n)
    grid = torch.as_tensor(rng.normal(size=gshape) + 1j * rng.normal(size=gshape),
                           device="cuda")
    v5, vt = _both(G, grid)
    ref = _fp64(G, grid, uvw, freq, cell, n, n, nchan, npol)
    assert rel(v5, ref) <= 1e-6
    assert rel(v5, vt) <= 5e-7


def test_shared_plan_exceptions():
    """On the rounding-tie lattice a shared plan lists samples for the
    degridder's own FP64 pass: the tensor-memory kernel leaves them to it,
    and every sample matches the FP64 plain degridder."""
    from test_shared_plan_gpu import _case, _counts
    from astroviper_b200.gridder import Gridder
    c = _case("ties", seed=5)
    nt, nb, nchan, npol = c["vis"].shape
    G = Gridder(c["uvw"], c["freq"], np.array([c["n"], c["n"]]), c["cell"], npol,
                support=c["sup"], oversampling=c["os"], chan_mode="cube")
    G.plan()
    assert _counts(G, G._gplan)[1] > 100
    rng = np.random.default_rng(3)
    gshape = (nchan, npol, c["n"], c["n"])
    grid = torch.as_tensor(rng.normal(size=gshape) + 1j * rng.normal(size=gshape),
                           device="cuda")
    v5, vt = _both(G, grid)
    from astroviper_b200 import _kernels as K
    n = c["n"]
    ref = K.degrid(grid, c["uvw"], c["freq"], (-c["cell"][0] * n, -c["cell"][1] * n),
                   (n / 2, n / 2), np.arange(nchan), np.arange(npol),
                   O.create_prolate_spheroidal_kernel_1D(c["os"], c["sup"]), c["sup"], c["os"],
                   nvchan=nchan, nvpol=npol, precision="fp64")
    err = (v5.to(torch.complex128) - ref).abs().cpu().numpy()
    assert err.max() <= 1e-5 * float(ref.abs().max())
    assert rel(v5, vt) <= 5e-7


def test_inf_cell_stays_in_its_samples():
    """An infinite grid value reaches only the samples whose footprint covers
    it: a tile's second cell does not leak into the first one's samples."""
    from astroviper_b200.gridder import Gridder
    uvw, freq, cell, n = _dense_case(3, nt=6)
    nchan, npol = len(freq), 4
    G = Gridder(uvw, freq, np.array([n, n]), cell, npol, support=7, oversampling=100)
    rng = np.random.default_rng(9)
    gshape = (1, npol, n, n)
    g = rng.normal(size=gshape) + 1j * rng.normal(size=gshape)
    # a busy cell near the first centre
    u = uvw[..., 0][..., None] * freq * (-(cell[0] * n) / 299792458.0) + n / 2
    v = uvw[..., 1][..., None] * freq * (-(cell[1] * n) / 299792458.0) + n / 2
    ok = np.isfinite(u) & (np.abs(u - n / 2) < n / 2 - 8) & (np.abs(v - n / 2) < n / 2 - 8)
    cu = np.floor(u[ok] + 0.5).astype(int)
    cv = np.floor(v[ok] + 0.5).astype(int)
    vals, cnt = np.unique(cu * n + cv, return_counts=True)
    hot = int(vals[np.argmax(cnt)])
    g[0, 2, hot // n, hot % n] = np.inf
    grid = torch.as_tensor(g, device="cuda")
    v5, vt = _both(G, grid)
    a5 = v5.cpu().numpy()
    at = vt.cpu().numpy()
    assert np.array_equal(np.isfinite(a5), np.isfinite(at))
    assert (~np.isfinite(a5)).sum() > 0
    fin = np.isfinite(at)
    assert rel(a5[fin], at[fin]) <= 5e-7
