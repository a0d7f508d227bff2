"""Bitwise-reproducible gridding (av_tiled_plan_order_rows +
av_grid_tiled_execute_det, Gridder(deterministic=True)).

Plans are rebuilt between the runs, so the scatter pass's atomics place a
cell's records in a different order each time; the row order and the
fixed-point sums must still give bit-identical grids and sums of weights,
within summation order of the FP64 oracle.  Cells of more than 1024 and of
more than 16384 samples exercise the CTA sorts in shared and global memory.
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


def _dense_case(seed=3, nt=40, nb=600, nchan=2, npol=4, n=64):
    """Samples packed into a few cells near the centre (hot cells hold tens
    of thousands of samples) plus a spread of ordinary ones."""
    rng = np.random.default_rng(seed)
    cell = np.array([-20.0, 20.0]) * np.pi / (180 * 3600)
    freq = np.array([1.4e9, 1.42e9])[:nchan]
    C = 299792458.0
    lam = C / freq[0]
    uv_cell = 1.0 / (n * abs(cell[0]))  # wavelengths per grid cell
    # 40 % in one hot cell, 30 % over a few cells around it, 30 % spread out
    pick = rng.uniform(size=(nt, nb))
    sig = np.where(pick < 0.4, 0.1, 1.0)
    u = rng.normal(0.0, 1.0, size=(nt, nb)) * sig * uv_cell * lam
    v = rng.normal(0.0, 1.0, size=(nt, nb)) * sig * uv_cell * lam
    spread = pick >= 0.7
    u = np.where(spread, rng.uniform(-20, 20, size=(nt, nb)) * uv_cell * lam, u)
    v = np.where(spread, rng.uniform(-20, 20, size=(nt, nb)) * uv_cell * lam, v)
    uvw = np.stack([u, v, rng.normal(size=(nt, nb))], axis=-1)
    shape = (nt, nb, nchan, npol)
    vis = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    wt = rng.uniform(0.2, 2.0, size=shape).astype(np.float32)
    wt[0, :50] = 0.0
    return dict(uvw=uvw, freq=freq, vis=vis, wt=wt, n=n, cell=cell)


def _grid(c, det, support=7, npol=None, do_psf=False, shared=False, mode="continuum"):
    from astroviper_b200.gridder import Gridder
    npol = npol or c["vis"].shape[3]
    G = Gridder(c["uvw"], c["freq"], np.array([c["n"], c["n"]]), c["cell"], npol,
                support=support, chan_mode=mode, deterministic=det)
    if shared:
        G.plan()
    vis = torch.as_tensor(c["vis"][..., :npol], device="cuda").contiguous()
    wt = torch.as_tensor(c["wt"][..., :npol], device="cuda").contiguous()
    g, sw = G.grid(vis, wt, do_psf=do_psf)
    torch.cuda.synchronize()
    return g, sw, G


def test_hot_cells_are_long():
    """Samples per cell over all channels (continuum: one plane)."""
    c = _dense_case()
    n = c["n"]
    C = 299792458.0
    keys = []
    for f in c["freq"]:
        us = -(f * c["cell"][0] * n) / C
        vs = -(f * c["cell"][1] * n) / C
        cu = np.floor(c["uvw"][..., 0] * us + n / 2 + 0.5).astype(int)
        cv = np.floor(c["uvw"][..., 1] * vs + n / 2 + 0.5).astype(int)
        keys.append((cu * n + cv).ravel())
    _, counts = np.unique(np.concatenate(keys), return_counts=True)
    assert counts.max() > 16384 and ((counts > 1024) & (counts <= 16384)).any()


@pytest.mark.parametrize("npol,support", [(4, 7), (2, 5), (1, 8)])
def test_deterministic_grid_is_bit_identical_across_plans(npol, support):
    c = _dense_case()
    runs = [_grid(c, True, support=support, npol=npol) for _ in range(3)]
    g0, s0, _ = runs[0]
    for g, s, _ in runs[1:]:
        assert torch.equal(g, g0) and torch.equal(s, s0)
    # the same values as the FP64 oracle, within summation order
    cgk = O.create_prolate_spheroidal_kernel_1D(100, support)
    go, so = O.standard_grid(c["vis"][..., :npol].astype(np.complex128), c["uvw"],
                             c["wt"][..., :npol].astype(np.float64), c["freq"], cgk,
                             np.array([c["n"], c["n"]]), c["cell"], 100, support)
    assert rel(g0, go) <= 1e-13 and rel(s0, so) <= 1e-13
    # the default path sums in FP64 in arrival order: same values
    gd, sd, _ = _grid(c, False, support=support, npol=npol)
    assert rel(g0, gd) <= 1e-13


def test_deterministic_psf_and_cube_and_accumulation():
    c = _dense_case(seed=9)
    a, sa, G = _grid(c, True, do_psf=True, mode="cube")
    b, sb, _ = _grid(c, True, do_psf=True, mode="cube")
    assert torch.equal(a, b) and torch.equal(sa, sb)
    # accumulating into a grid adds one fixed-point result per cell
    vis = torch.as_tensor(c["vis"], device="cuda")
    wt = torch.as_tensor(c["wt"], device="cuda")
    g1, s1 = G.grid(vis, wt)
    g2, s2 = G.grid(vis, wt, grid=g1.clone(), sum_weight=s1.clone())
    assert rel(g2, 2 * g1) <= 1e-15 and rel(s2, 2 * s1) <= 1e-15


def test_ordered_shared_plan_keeps_the_degridders_marks():
    """A shared plan ordered by row still degrids like separate plans: the
    degridder's marks moved with their records."""
    from astroviper_b200 import synthetic as S
    from astroviper_b200.gridder import Gridder
    W = S.workload_large(n_time=8, n_chan=16, n_pol=4)
    img, cell = np.array([512, 512]), W["pixelincr"] * 4
    vis = torch.as_tensor(W["vis"], device="cuda")
    out = {}
    for det in (True, False):
        G = Gridder(W["uvw"], W["freq"], img, cell, 4, deterministic=det)
        G.shared_plan = det
        G.plan()
        g, _ = G.grid(vis, torch.ones(vis.shape, dtype=torch.float32, device="cuda"))
        out[det] = (g, G.degrid(g))
    assert rel(out[True][0], out[False][0]) <= 1e-13
    assert rel(out[True][1], out[False][1]) <= 2e-7


def test_execute_det_refuses_an_unordered_plan_and_infinite_values():
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import _lib
    c = _dense_case(nt=4, nb=100)
    L = _lib.lib()
    nt, nb, nchan, npol = c["vis"].shape
    n = c["n"]
    uvw = torch.as_tensor(c["uvw"], device="cuda")
    freq = torch.as_tensor(c["freq"], device="cuda")
    cm = torch.zeros(nchan, dtype=torch.int32, device="cuda")
    pm = torch.arange(npol, dtype=torch.int32, device="cuda")
    cgk = K.pswf_table(100, 7)
    ws = K.workspace(L.av_grid_tiled_workspace_size(nt, nb, nchan, n, n, 1, 7))
    _lib.check(L.av_grid_tiled_plan(K.p(uvw), K.p(freq), K.p(cm), n, n, float(c["cell"][0]),
                                    float(c["cell"][1]), 7, 100, nt, nb, nchan, 1, ws[1], ws[2],
                                    K.stream_ptr()), "plan")
    dws = K.workspace(L.av_grid_tiled_det_workspace_size(1, npol, n, n))
    grid = torch.zeros((1, npol, n, n), dtype=torch.complex128, device="cuda")
    sw = torch.zeros((1, npol), dtype=torch.float64, device="cuda")
    vis = torch.as_tensor(c["vis"], device="cuda")
    wt = torch.as_tensor(c["wt"], device="cuda")

    def run():
        return L.av_grid_tiled_execute_det(K.p(grid), K.dcode(grid), K.p(sw), 0, K.p(vis),
                                           _lib.AV_C64, K.p(wt), _lib.AV_F32, K.p(pm), K.p(cgk),
                                           n, n, 7, 100, nt, nb, nchan, npol, 1, npol, ws[1],
                                           ws[2], dws[1], dws[2], K.stream_ptr())
    assert run() == _lib.AV_ERR_ARG and "ordered by row" in _lib.last_error()
    assert bool((grid == 0).all())
    _lib.check(L.av_tiled_plan_order_rows(nt, nb, nchan, n, n, 1, 7, ws[1], ws[2],
                                          K.stream_ptr()), "order")
    assert run() == _lib.AV_OK
    wt[0, 3, 0, 1] = float("inf")
    assert run() == _lib.AV_ERR_ARG and "infinite" in _lib.last_error()
    with pytest.raises(ValueError):
        from astroviper_b200.gridder import Gridder
        Gridder(c["uvw"], c["freq"], np.array([n, n]), c["cell"], npol, support=9,
                deterministic=True)
