"""Batched uneven gridding (cube mode, many independent grids with their own
flag fractions) in one persistent launch under a CUDA graph: against the
oracle in cube mode, against one launch per grid, across graph replays with
new inputs, and with the autotuner choosing the launch knob."""
import numpy as np
import pytest
import torch

import oracle as O
from astroviper_b200 import _lib

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def _work(seed=3, support=7):
    from astroviper_b200 import synthetic as S
    W = S.workload_batched(seed=seed, n_time=24, n_chan=6, n_pol=2, image=128, device="cuda")
    W["support"] = support
    return W


def _oracle(W, vis, wt):
    cf = O.create_prolate_spheroidal_kernel_1D(100, W["support"])
    v = vis.cpu().numpy().astype(np.complex128)
    w = wt.cpu().numpy().astype(np.float64)
    return O.standard_grid(v, W["uvw"], w, W["freq"], cf, W["image_size"], W["pixelincr"],
                           support=W["support"], chan_mode="cube")


@pytest.mark.parametrize("drop_flagged", [False, True])
@pytest.mark.parametrize("support", [7, 9])
def test_batched_graph_matches_oracle_and_replays(support, drop_flagged):
    """Three calls in a row (so the touched-tile clears run between them):
    with drop_flagged the graph rebuilds the plan from each batch's weights
    and leaves the fully flagged samples out."""
    from astroviper_b200.batched import BatchedGridder
    W = _work(support=support)
    frac = W["flag_fraction"]
    assert frac.min() >= 0.0 and frac.max() < 0.6
    B = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], 2, support=support,
                       graph=True, drop_flagged=drop_flagged)
    g, sw = B(W["vis"], W["weight"])
    rg, rs = _oracle(W, W["vis"], W["weight"])
    assert rel(g.cpu().numpy(), rg) <= 1e-12
    assert np.allclose(sw.cpu().numpy(), rs, rtol=1e-12)
    # uneven: the per-grid sums of weights follow the flag fractions
    counts = W["weight"].sum(dim=(0, 1)).cpu().numpy()
    assert counts.min() < 0.75 * counts.max()
    # replay with other inputs
    w2 = torch.flip(W["weight"], dims=[2]).contiguous()
    v2 = (W["vis"] * 0.5j).contiguous()
    g2, sw2 = B(v2, w2)
    rg2, rs2 = _oracle(W, v2, w2)
    assert rel(g2.cpu().numpy(), rg2) <= 1e-12
    assert np.allclose(sw2.cpu().numpy(), rs2, rtol=1e-12)
    # and back
    g3, _ = B(W["vis"], W["weight"])
    assert rel(g3.cpu().numpy(), rg) <= 1e-12


def test_per_grid_launches_equal_batched():
    from astroviper_b200.batched import BatchedGridder, PerGridGridder
    W = _work(seed=5)
    B = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], 2, graph=False)
    g, sw = B(W["vis"], W["weight"])
    P = PerGridGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], 2)
    gp, swp = P(P.split(W["vis"], W["weight"]))
    assert rel(gp.cpu().numpy(), g.cpu().numpy()) <= 1e-12
    assert np.allclose(swp.cpu().numpy(), sw.cpu().numpy(), rtol=1e-12)


def test_batched_with_autotuner(tmp_path, monkeypatch):
    from astroviper_b200 import autotune
    from astroviper_b200.batched import BatchedGridder
    monkeypatch.setenv("AV200_TUNE_CACHE", str(tmp_path / "tune.json"))
    W = _work(seed=7)
    B = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], 2, graph=True,
                       tune=True)
    autotune._applied.pop(B.tune_key(), None)
    g, _ = B(W["vis"], W["weight"])
    rg, _ = _oracle(W, W["vis"], W["weight"])
    assert rel(g.cpu().numpy(), rg) <= 1e-12
    entries = autotune.load(str(tmp_path / "tune.json"))
    assert B.tune_key() in entries
    best = entries[B.tune_key()]["value"]
    assert best["chunks_per_sm"] in autotune.CANDIDATES
    assert best["lanes"] in (_lib.AV_GRID_LANES_MMA, _lib.AV_GRID_LANES_ROWS)
    assert len(entries[B.tune_key()]["ms"]) == 2 * len(autotune.CANDIDATES)
    assert _lib.lib().av_tune_get(_lib.AV_TUNE_GRID_LANES) == best["lanes"]
    # put the process-wide knobs back for the tests that follow
    _lib.lib().av_tune_set(_lib.AV_TUNE_GRID_LANES, _lib.AV_GRID_LANES_AUTO)
    _lib.lib().av_tune_set(_lib.AV_TUNE_GRID_CHUNKS_PER_SM, 16)
    autotune._applied.pop(B.tune_key(), None)


def test_batched_support_auto_picks_the_less_aliasing_kernel():
    """support="auto" takes the smallest of 7 and 9 whose aliasing in the
    inner 80 % of the field meets the tolerance: 7, which aliases less than 9
    with the reference's kernel; the grids are then support 7's."""
    from astroviper_b200.batched import BatchedGridder
    W = _work(seed=9)
    B = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], 2, support="auto",
                       graph=False)
    assert B.support == 7 and B.alias[7] < 1e-2 < B.alias[9]
    g, _ = B(W["vis"], W["weight"])
    rg, _ = _oracle(W, W["vis"], W["weight"])
    assert rel(g.cpu().numpy(), rg) <= 1e-12
