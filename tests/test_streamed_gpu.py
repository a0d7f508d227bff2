"""Streamed host-input paths of the numpy drop-ins: large numpy inputs go to
the device in time chunks on a copy stream while neighbouring chunks are
gridded / degridded (and, for the degridder, copied back on a third stream).
Chunking changes only the order in which the FP64 grid sums are formed, and
the degridder's per-sample arithmetic not at all, so the streamed results are
checked against the single-launch ones: grid within 1e-12 relative, degridded
values bit-identical; and against the golden outputs with the chunk size forced
down so the golden cases stream in several pieces."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (nb if nb else 1.0)


def pinned(a):
    t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1].copy()).dtype, pin_memory=True)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
    return t.numpy()


@pytest.fixture
def small_chunks(monkeypatch):
    from astroviper_b200 import _kernels as K
    monkeypatch.setattr(K, "STREAM_CHUNK_BYTES", 1024)
    return K


@pytest.mark.parametrize("case", ["a", "b", "c"])
def test_streamed_grid_dropin_matches_golden_and_single_launch(small_chunks, case):
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG
    g = golden(f"grid_{case}.npz")
    sup, os_ = int(g["support"]), int(g["oversampling"])
    for pin in (False, True):
        vis = pinned(g["vis"]) if pin else g["vis"]
        w = pinned(g["weight"]) if pin else g["weight"]
        for do_psf in (False, True):
            for mode in ("continuum", "cube"):
                key = f"{'psf' if do_psf else 'vis'}_{mode}"
                gr, sw = SG.standard_grid_numpy_wrap_input_checked(
                    vis, np.array([]), np.array([]), g["uvw"], w, g["freq"], g["cgk"],
                    g["image_size"], g["cell"], os_, sup, True, do_psf, mode, precision="fp32")
                assert rel(gr, g["grid_" + key]) <= 1e-6, key
                assert np.allclose(sw, g["sumwt_" + key], rtol=1e-7)
                one, sw1 = SG.standard_grid_numpy_wrap_input_checked(
                    torch.as_tensor(vis, device="cuda"), np.array([]), np.array([]),
                    g["uvw"], torch.as_tensor(w, device="cuda"), g["freq"], g["cgk"],
                    g["image_size"], g["cell"], os_, sup, True, do_psf, mode, precision="fp32")
                assert rel(gr, one.cpu().numpy()) <= 1e-12, key
                assert np.allclose(sw, sw1.cpu().numpy(), rtol=1e-12)


def test_streamed_grid_accumulates_in_place(small_chunks):
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG
    g = golden("grid_a.npz")
    gr = g["acc_grid0"].copy()
    sw = g["acc_sumwt0"].copy()
    out = SG.standard_grid_numpy_wrap_input_checked(
        g["vis"], gr, sw, g["uvw"], g["weight"], g["freq"], g["cgk"], g["image_size"], g["cell"],
        int(g["oversampling"]), int(g["support"]), True, False, "continuum", precision="fp32")
    assert out[0] is gr and out[1] is sw
    assert rel(gr, g["acc_grid"]) <= 1e-6 and np.allclose(sw, g["acc_sumwt"], rtol=1e-7)


@pytest.mark.parametrize("phase", ["zero", "phase"])
def test_streamed_dgrid_numba_matches_golden_and_single_launch(small_chunks, phase):
    from astroviper_b200.core.imaging.imaging_utils import standard_degrid as SD
    g = golden("degrid.npz")
    nt, nb = g["uvw"].shape[:2]
    dph = np.zeros((nt, nb)) if phase == "zero" else g["dphase"]
    for sup, os_ in ((7, 100), (9, 64), (8, 100)):
        cf = O.create_prolate_spheroidal_kernel_1D(os_, sup)
        v0 = g[f"v0_{sup}_{os_}_{phase}"]
        ref = g[f"v_{sup}_{os_}_{phase}"]
        for pin in (False, True):
            v = pinned(v0) if pin else v0.copy()
            SD.dgrid_numba(g["uvw"], dph, v, g["flag"], g["scale"], g["offset"], g["grid"],
                           g["freq"], 299792458.0, sup, os_, cf, g["chanmap"], g["polmap"],
                           precision="fp32")
            assert rel(v - v0, ref - v0) <= 1e-6
            one = torch.as_tensor(v0, device="cuda").clone()
            SD.dgrid_numba(g["uvw"], dph, one, g["flag"], g["scale"], g["offset"], g["grid"],
                           g["freq"], 299792458.0, sup, os_, cf, g["chanmap"], g["polmap"],
                           precision="fp32")
            assert np.array_equal(v, one.cpu().numpy())


def test_streamed_kernels_on_a_multichannel_four_pol_workload():
    """Direct calls with a few-hundred-kB chunk size on 16 steps x 2016
    baselines x 8 channels x 4 polarisations (complex64, float32 weights,
    complex64 model values, without flags and with 5% flagged): streamed against single-launch."""
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import synthetic as S
    W = S.workload_large(n_time=16, n_chan=8, device=torch.device("cuda"))
    vis_d = W["vis"]
    nt, nb, nchan, npol = vis_d.shape
    rng = np.random.default_rng(7)
    w_h = pinned(rng.uniform(0.5, 2.0, size=vis_d.shape).astype(np.float32))
    vis_h = pinned(vis_d.cpu().numpy())
    uvw = W["uvw"]
    nx = int(W["image_size"][0])
    cgk = O.create_prolate_spheroidal_kernel_1D(100, 7)
    cm = np.zeros(nchan, dtype=np.int32)
    pm = np.arange(npol, dtype=np.int32)
    args = (W["freq"], cm, pm, cgk, (nx, nx), W["pixelincr"], 7, 100, 1, npol)
    g1 = torch.zeros((1, npol, nx, nx), dtype=torch.complex128, device="cuda")
    s1 = torch.zeros((1, npol), dtype=torch.float64, device="cuda")
    K.grid(vis_d, torch.as_tensor(w_h, device="cuda"), uvw, *args, grid_out=g1, sum_weight=s1)
    g2 = torch.zeros_like(g1)
    s2 = torch.zeros_like(s1)
    K.grid_streamed(vis_h, w_h, uvw, *args, grid_out=g2, sum_weight=s2, chunk_bytes=300_000)
    torch.cuda.synchronize()
    assert rel(g2.cpu().numpy(), g1.cpu().numpy()) <= 1e-12
    assert np.allclose(s2.cpu().numpy(), s1.cpu().numpy(), rtol=1e-12)

    scale = np.array([-W["pixelincr"][0] * nx, -W["pixelincr"][1] * nx, 0.0])
    offset = np.array([nx / 2, nx / 2, 0.0])
    v0 = (rng.normal(size=vis_d.shape) + 1j * rng.normal(size=vis_d.shape)).astype(np.complex64)
    for flag in (None, rng.uniform(size=vis_d.shape) < 0.05):
        one = torch.as_tensor(v0, device="cuda").clone()
        K.degrid(g1, uvw, W["freq"], scale, offset, cm, pm, cgk, 7, 100, values=one,
                 flag=None if flag is None else torch.as_tensor(flag, device="cuda"))
        v = pinned(v0)
        K.degrid_streamed(g1, uvw, W["freq"], scale, offset, cm, pm, cgk, 7, 100, v, flag=flag,
                          chunk_bytes=300_000)
        assert np.array_equal(v, one.cpu().numpy())
