"""One binning plan for the gridder and the degridder (av_tiled_plan_shared).

The gridder rounds cells and kernel offsets with int(x + 0.5)
(standard_grid.py:337-352), the degridder with np.round, half to even
(standard_degrid.py:442-450), from FP64 positions computed in a different
order.  A shared plan sorts by the gridder's cells and lists the samples where
the degridder's rounding differs; these tests check that gridding and
degridding through it give what separate plans give, on ordinary data and on
positions placed exactly on rounding ties (where the two conventions part),
in store and accumulate mode, against the FP64 oracle too.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

C = 299792458.0


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _counts(G, ws):
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import _lib
    out = (ctypes.c_uint32 * 2)()
    _lib.check(_lib.lib().av_tiled_plan_counts(G.nt, G.nb, G.nchan, G.nx, G.ny, G.n_img_chan,
                                               G.support, ws[1], ws[2], out, K.stream_ptr()),
               "av_tiled_plan_counts")
    return int(out[0]), int(out[1])


def _tie_uvw(n, cell, freq, nt, nb, os_, rng, frac=0.5):
    """uvw whose first channel puts a fraction of the samples exactly on the
    gridder's rounding ties: cells at k + 1/2 and kernel-offset arguments at
    half-integers (positions k + odd / (2 os) with os a power of two)."""
    u = rng.uniform(-0.3, 0.3, size=(nt, nb)) * n
    v = rng.uniform(-0.3, 0.3, size=(nt, nb)) * n
    f = freq[0]
    us0 = -((f * cell[0]) * n) / C
    us1 = -((f * cell[1]) * n) / C
    pick = rng.uniform(size=(nt, nb)) < frac
    ku = rng.integers(-n // 4, n // 4, size=(nt, nb))
    kv = rng.integers(-n // 4, n // 4, size=(nt, nb))
    half = rng.uniform(size=(nt, nb)) < 0.5
    odd_u = 2 * rng.integers(0, os_, size=(nt, nb)) + 1
    odd_v = 2 * rng.integers(0, os_, size=(nt, nb)) + 1
    tu = np.where(half, ku + 0.5, ku + odd_u / (2.0 * os_))  # u position - n/2
    tv = np.where(half, kv + 0.5, kv + odd_v / (2.0 * os_))
    um = np.where(pick, tu / us0, u / us0)
    vm = np.where(pick, tv / us1, v / us1)
    w = rng.uniform(-100, 100, size=(nt, nb))
    uvw = np.stack([um, vm, w], axis=-1)
    uvw[1, 3, 0] = np.nan   # a NaN row: skipped by both conventions
    uvw[2, 5, :2] *= 1e3    # off the grid
    return np.ascontiguousarray(uvw)


def _case(kind, seed=11):
    from astroviper_b200 import synthetic as S
    rng = np.random.default_rng(seed)
    if kind == "ordinary":
        W = S.workload_large(n_time=16, n_chan=8, n_pol=4)
        uvw, freq = W["uvw"], W["freq"]
        n, os_, sup, cell = 512, 100, 7, W["pixelincr"] * 4
        vis = W["vis"]
    else:
        nt, nb, nchan, npol = 6, 600, 3, 4
        n, os_, sup = 256, 64, 7
        cell = np.array([-2.0, 2.0]) * np.pi / (180 * 3600)
        freq = np.array([1.4e9, 1.45e9, 1.5e9])
        uvw = _tie_uvw(n, cell, freq, nt, nb, os_, rng)
        shape = (nt, nb, nchan, npol)
        vis = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    shape = vis.shape
    wt = rng.uniform(0.5, 2.0, size=shape).astype(np.float32)
    wt[0, 2] = 0.0
    return dict(uvw=uvw, freq=freq, vis=vis, wt=wt, n=n, os=os_, sup=sup, cell=cell)


@pytest.mark.parametrize("kind", ["ordinary", "ties"])
@pytest.mark.parametrize("mode", ["continuum", "cube"])
def test_shared_plan_matches_separate_plans(kind, mode):
    from astroviper_b200.gridder import Gridder
    c = _case(kind)
    nt, nb, nchan, npol = c["vis"].shape
    img, cell, sup, os_ = np.array([c["n"], c["n"]]), c["cell"], c["sup"], c["os"]
    vis = torch.as_tensor(c["vis"], device="cuda")
    wt = torch.as_tensor(c["wt"], device="cuda")
    out = {}
    for shared in (True, False):
        G = Gridder(c["uvw"], c["freq"], img, cell, npol, support=sup, oversampling=os_,
                    chan_mode=mode)
        G.shared_plan = shared
        G.plan()
        g, sw = G.grid(vis, wt)
        v_store = G.degrid(g)  # store mode (fast path: complex64, 4 pols, no flags)
        flag = torch.zeros(vis.shape, dtype=torch.bool, device="cuda")
        flag[:, 1::7, :, 2] = True
        v_acc = torch.full(vis.shape, 0.25 + 0.5j, dtype=torch.complex128, device="cuda")
        G.degrid(g, values=v_acc, flag=flag, accumulate=True)
        out[shared] = (g, sw, v_store, v_acc, G)
    g1, s1, vs1, va1, G1 = out[True]
    g0, s0, vs0, va0, G0 = out[False]
    n_rec_shared, n_exc = _counts(G1, G1._gplan)
    n_rec_grid, _ = _counts(G0, G0._gplan)
    assert n_rec_shared == n_rec_grid
    if kind == "ties":
        assert n_exc > 100  # the conventions part on the ties
    # gridding: the same records; FP64 sums whose order the atomics set
    assert rel(g1, g0) <= 1e-13 and rel(s1, s0) <= 1e-13
    # degridding: separate-plan results (FP32 path) within FP32 rounding, and
    # both against the FP64 oracle on the same grid
    assert rel(vs1, vs0) <= 2e-7
    assert rel(va1, va0) <= 2e-7
    cgk = O.create_prolate_spheroidal_kernel_1D(os_, sup)
    gnp = g0.cpu().numpy()
    vo = O.degrid(gnp, c["uvw"], c["freq"], cell, flag=np.zeros(vis.shape, np.uint8),
                  support=sup, sampling=os_)
    assert rel(vs1, vo) <= 1e-6
    fo = flag.cpu().numpy().astype(np.uint8)
    vao = np.full(vis.shape, 0.25 + 0.5j) + O.degrid(gnp, c["uvw"], c["freq"], cell, flag=fo,
                                                     support=sup, sampling=os_)
    assert rel(va1, vao) <= 1e-6
    # and the grid against the oracle's gridder
    go, so = O.standard_grid(c["vis"].astype(np.complex128), c["uvw"],
                             c["wt"].astype(np.float64), c["freq"], cgk, img, cell, os_, sup,
                             chan_mode=mode)
    assert rel(g1, go) <= 1e-12


def test_shared_plan_exception_samples_are_the_degridders():
    """On the tie lattice, every sample's degridded value through the shared
    plan is the FP64 plain degridder's (the reference's exact arithmetic)
    within the FP32 path's rounding, including the ones the conventions part
    on: a wrong cell or offset would be off by far more."""
    from astroviper_b200 import _kernels as K
    from astroviper_b200.gridder import Gridder
    c = _case("ties", seed=5)
    nt, nb, nchan, npol = c["vis"].shape
    img, cell, sup, os_ = np.array([c["n"], c["n"]]), c["cell"], c["sup"], c["os"]
    G = Gridder(c["uvw"], c["freq"], img, cell, npol, support=sup, oversampling=os_,
                chan_mode="cube")
    G.plan()
    assert _counts(G, G._gplan)[1] > 100
    rng = np.random.default_rng(3)
    gshape = (nchan, npol, c["n"], c["n"])
    grid = torch.as_tensor(rng.normal(size=gshape) + 1j * rng.normal(size=gshape),
                           device="cuda")
    v = G.degrid(grid).to(torch.complex128)
    n = c["n"]
    ref = K.degrid(grid, c["uvw"], c["freq"], (-cell[0] * n, -cell[1] * n), (n / 2, n / 2),
                   np.arange(nchan), np.arange(npol), O.create_prolate_spheroidal_kernel_1D(os_, sup),
                   sup, os_, nvchan=nchan, nvpol=npol, precision="fp64")
    err = (v - ref).abs().cpu().numpy()
    scale = float(ref.abs().max())
    assert err.max() <= 1e-5 * scale


def test_clear_grid_zeroes_the_cells_a_plan_can_touch():
    """av_grid_tiled_clear (Gridder.clear_grid) zeroes every cell a plan's
    samples can reach and leaves cells beyond its tiles alone."""
    from astroviper_b200.gridder import Gridder
    c = _case("ordinary")
    nt, nb, nchan, npol = c["vis"].shape
    img = np.array([c["n"], c["n"]])
    G = Gridder(c["uvw"], c["freq"], img, c["cell"], npol, support=c["sup"],
                oversampling=c["os"])
    g, _ = G.grid(torch.as_tensor(c["vis"], device="cuda"),
                  torch.as_tensor(c["wt"], device="cuda"))
    touched = (g != 0)
    assert int(touched.sum()) > 0
    assert bool((G.clear_grid(g.clone()) == 0).all())
    ones = G.clear_grid(torch.ones_like(g))
    assert bool((ones[touched] == 0).all())
    assert ones[0, 0, 0, 0] == 1 and ones[0, 0, -1, -1] == 1  # far from the uv coverage
