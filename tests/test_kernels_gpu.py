"""CUDA kernels (through the C ABI) against the CPU oracle and the reference's
golden outputs.  Tolerances: FP64 paths 1e-12 relative (norm-wise), the plain
FP64 degridder and Hogbom bit-exact, FP32 paths 1e-5 relative (norm-wise)."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu


def K():
    from astroviper_b200 import _kernels
    return _kernels


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def test_pswf_tables_match_reference():
    g = golden("pswf.npz")
    for os_, sup in [(100, 7), (64, 9), (100, 8), (50, 5), (128, 6)]:
        t = K().pswf_table(os_, sup).cpu().numpy()
        ref = g[f"cgk_{os_}_{sup}"]
        assert np.max(np.abs(t - ref)) <= 1e-15 * np.max(np.abs(ref))
    for n in [(64, 64), (96, 128), (101, 77)]:
        c = K().corr_term(*n).cpu().numpy()
        ref = g[f"corr_{n[0]}_{n[1]}"]
        assert np.max(np.abs(c - ref) / np.abs(ref)) <= 1e-14
    gr, kk = K().pswf(g["u"])
    assert np.allclose(gr.cpu().numpy(), g["grdsf"], rtol=1e-14, atol=1e-300)
    assert np.allclose(kk.cpu().numpy(), g["kern"], rtol=1e-14, atol=1e-300)


def _grid_case(case, precision, do_psf, mode):
    g = golden(f"grid_{case}.npz")
    sup, os_ = int(g["support"]), int(g["oversampling"])
    nchan, npol = g["weight"].shape[2:]
    n_img_chan = nchan if mode == "cube" else 1
    cm = np.arange(nchan) if mode == "cube" else np.zeros(nchan, int)
    gr, sw = K().grid(g["vis"], torch.as_tensor(g["weight"]), g["uvw"], g["freq"], cm,
                      np.arange(npol), g["cgk"], g["image_size"], g["cell"], sup, os_,
                      n_img_chan, npol, do_psf=do_psf, precision=precision)
    key = f"{'psf' if do_psf else 'vis'}_{mode}"
    return gr.cpu().numpy(), sw.cpu().numpy(), g["grid_" + key], g["sumwt_" + key]


@pytest.mark.parametrize("case", ["a", "b", "c"])
@pytest.mark.parametrize("do_psf", [False, True])
@pytest.mark.parametrize("mode", ["continuum", "cube"])
def test_grid_plain_fp64(case, do_psf, mode):
    gr, sw, rg, rs = _grid_case(case, "fp64", do_psf, mode)
    assert rel(gr, rg) <= 1e-12
    assert np.allclose(sw, rs, rtol=1e-12, atol=0)


@pytest.mark.parametrize("case", ["a", "b", "c"])
@pytest.mark.parametrize("do_psf", [False, True])
@pytest.mark.parametrize("mode", ["continuum", "cube"])
def test_grid_tiled_fp32(case, do_psf, mode, grid_lanes):
    """The tiled gridder on the reference's golden cases (data and PSF
    gridding), under both lane mappings."""
    gr, sw, rg, rs = _grid_case(case, "fp32", do_psf, mode)
    assert rel(gr, rg) <= 1e-5
    assert np.allclose(sw, rs, rtol=1e-6, atol=0)


def test_grid_imaging_weight_branch_fp64():
    g = golden("grid_a.npz")
    nchan, npol = g["weight"].shape[2:]
    gr, sw = K().grid(None, torch.as_tensor(g["iw_weight"]), g["uvw"], g["freq"],
                      np.zeros(nchan, int), np.arange(npol), g["cgk"], g["image_size"],
                      g["cell"], 7, 100, 1, npol, do_psf=True, do_imaging_weight=True,
                      precision="fp64")
    assert rel(gr.cpu().numpy(), g["iw_grid"]) <= 1e-12
    assert np.allclose(sw.cpu().numpy(), g["iw_sumwt"], rtol=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_degrid_golden(precision):
    g = golden("degrid.npz")
    nt, nb = g["uvw"].shape[:2]
    for sup, os_ in ((7, 100), (9, 64), (8, 100)):
        cf = g["grid"]  # noqa
        cgk = O.create_prolate_spheroidal_kernel_1D(os_, sup)
        for dp_name in ("zero", "phase"):
            dph = None if dp_name == "zero" else g["dphase"]
            v0 = g[f"v0_{sup}_{os_}_{dp_name}"]
            vals = torch.as_tensor(v0.astype(np.complex128 if precision == "fp64"
                                              else np.complex64)).cuda()
            K().degrid(g["grid"], g["uvw"], g["freq"], g["scale"], g["offset"], g["chanmap"],
                       g["polmap"], cgk, sup, os_, values=vals, flag=g["flag"], dphase=dph,
                       precision=precision)
            out = vals.cpu().numpy()
            ref = g[f"v_{sup}_{os_}_{dp_name}"]
            if precision == "fp64":
                if dp_name == "zero":
                    assert np.array_equal(out, ref), (sup, os_)
                else:
                    assert rel(out, ref) <= 1e-14, (sup, os_)
            else:
                assert rel(out - v0, ref - v0) <= 1e-5, (sup, os_, dp_name)


def test_image_golden():
    g = golden("image.npz")
    cgk = O.create_prolate_spheroidal_kernel_1D(100, 7)
    for dopsf in (False, True):
        for mode in ("continuum", "cube"):
            tag = f"{'psf' if dopsf else 'vis'}_{mode}"
            w = g["weight_after_" + tag]
            nci = 2 if mode == "cube" else 1
            cm = np.arange(2) if mode == "cube" else np.zeros(2, int)
            for precision, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
                gr, sw = K().grid(g["vis"], torch.as_tensor(w), g["uvw"], g["freq"], cm,
                                  np.arange(2), cgk, (64, 64), g["cell"], 7, 100, nci, 2,
                                  do_psf=dopsf, precision=precision)
                img = K().grid_to_image(gr, sw).cpu().numpy()
                assert rel(img, g["img_" + tag]) <= tol, (tag, precision)


def test_fft_helpers():
    g = golden("image.npz")
    f = K().fft_shifted(torch.as_tensor(g["fft_in"]).to(torch.complex128), inverse=False)
    assert rel(f.cpu().numpy(), g["fft_out"]) <= 1e-13
    b = K().fft_shifted(torch.as_tensor(g["fft_out"]), inverse=True)
    assert rel(b.cpu().numpy().real, g["ifft_out"]) <= 1e-13


def test_weights_golden():
    g = golden("weights.npz")
    for npol in (1, 2, 4):
        q = lambda k: g[f"p{npol}_{k}"]
        G, sw = K().weight_density(q("uvw"), q("freq"), torch.as_tensor(q("w")),
                                   torch.as_tensor(q("flag")), q("n"), q("cell"))
        assert rel(G.cpu().numpy(), q("G")) <= 1e-13
        assert np.allclose(sw.cpu().numpy(), q("sw"), rtol=1e-13)
        for robust in (-1.0, 0.5, 2.0):
            bf = K().briggs_factors(G, sw, robust)
            assert np.allclose(bf.cpu().numpy(), q(f"bf_{robust}"), rtol=1e-12)
            iw, err = K().briggs_apply(G, bf, q("uvw"), q("freq"), torch.as_tensor(q("w")),
                                       torch.as_tensor(q("flag")), q("n"), q("cell"))
            assert int(err.item()) == 0
            assert np.allclose(iw.cpu().numpy(), q(f"iw_{robust}"), rtol=1e-12, atol=0,
                               equal_nan=True)


RUNS = {
    "default": dict(max_iter=100),
    "box_thr": dict(max_iter=400, gain=0.2, threshold=0.02, clean_box=(5, 50, 10, 60)),
    "mask_speed": dict(max_iter=150, start_iter=3, speedup=40.0, threshold=0.005, mask=True),
    "long": dict(max_iter=1000, gain=0.05),
}


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("name", list(RUNS))
def test_hogbom_kernel_golden(tag, name):
    g = golden("hogbom.npz")
    dt = np.float32 if tag == "f32" else np.float64
    kw = dict(RUNS[name])
    ny, nx = g["dirty"].shape
    box = kw.get("clean_box", (0, nx, 0, ny))
    mask = g["mask"].astype(dt) if kw.get("mask") else None
    run = K().HogbomRun(torch.as_tensor(g["dirty"].astype(dt)), torch.as_tensor(g["psf"].astype(dt)),
                        mask=None if mask is None else torch.as_tensor(mask), box=box,
                        niter=kw["max_iter"], siter=kw.get("start_iter", 0),
                        gain=kw.get("gain", 0.1), threshold=kw.get("threshold", 0.0),
                        speedup=kw.get("speedup", 0.0))
    run.run(kw.get("start_iter", 0), kw["max_iter"])
    st = run.read_state()
    assert st["err"] == 0
    assert st["iter"] == int(g[f"{tag}_{name}_iterations_performed"])
    assert np.array_equal(run.model.cpu().numpy(), g[f"{tag}_{name}_model_image"])
    assert np.array_equal(run.resid.cpu().numpy(), g[f"{tag}_{name}_residual_image"])


def test_maximg_and_abs_sum():
    g = golden("hogbom.npz")
    for tag, dt in (("f32", np.float32), ("f64", np.float64)):
        m = K().maximg(torch.as_tensor(g["dirty"].astype(dt))).cpu().numpy()
        assert np.array_equal(m, g[f"{tag}_maximg"])
        m = K().maximg(torch.as_tensor(g["dirty"].astype(dt)),
                       torch.as_tensor(g["mask"].astype(dt))).cpu().numpy()
        assert np.array_equal(m, g[f"{tag}_maximg_mask"])
        model = g[f"{tag}_long_model_image"]
        s = K().abs_sum_ordered(torch.as_tensor(model)).cpu().numpy()[0]
        assert s == g[f"{tag}_long_total_flux_cleaned"]


def test_small_workload_grid_degrid_vs_oracle():
    """The small workload (64 antennas, 50 steps, 2 pols, 512^2): FP32 tiled
    grid and degrid within 1e-5 of the FP64 oracle; FP64 within 1e-12."""
    from astroviper_b200 import synthetic as S
    W = S.workload_small()
    cgk = O.create_prolate_spheroidal_kernel_1D(100, 7)
    rg, rs = O.standard_grid(W["vis"], W["uvw"], W["weight"], W["freq"], cgk, W["image_size"],
                             W["pixelincr"])
    for precision, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
        gr, sw = K().grid(W["vis"], torch.as_tensor(W["weight"]), W["uvw"], W["freq"],
                          np.zeros(1, int), np.arange(2), cgk, W["image_size"], W["pixelincr"],
                          7, 100, 1, 2, precision=precision)
        assert rel(gr.cpu().numpy(), rg) <= tol
        assert np.allclose(sw.cpu().numpy(), rs, rtol=tol)
    rv = O.degrid(rg, W["uvw"], W["freq"], W["pixelincr"], flag=W["flag"])
    nx, ny = 512, 512
    scale = (-W["pixelincr"][0] * nx, -W["pixelincr"][1] * ny)
    for precision, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
        v = K().degrid(torch.as_tensor(rg), W["uvw"], W["freq"], scale, (nx / 2, ny / 2),
                       np.zeros(1, int), np.arange(2), cgk, 7, 100, flag=W["flag"],
                       nvchan=1, nvpol=2, precision=precision)
        assert rel(v.cpu().numpy(), rv) <= tol, precision


@pytest.mark.parametrize("support", [3, 4, 5, 6, 7, 8, 9])
@pytest.mark.parametrize("os_", [32, 100])
def test_tiled_degrid_every_support(support, os_):
    """The tiled degridder against the oracle for every support and two
    oversamplings on the golden degrid case (a 2-polarisation grid read by 4
    visibility polarisations, 2 grid channels).  The block sizes make the
    staging loops end mid-warp for some supports, which the kernels must
    survive at their block barriers."""
    g = golden("degrid.npz")
    nt, nb = g["uvw"].shape[:2]
    cf = O.create_prolate_spheroidal_kernel_1D(os_, support)
    ref = np.zeros((nt, nb, 3, 4), complex)
    O.dgrid_numba(g["uvw"], np.zeros((nt, nb)), ref, g["flag"], g["scale"], g["offset"],
                  g["grid"], g["freq"], 299792458.0, support, os_, cf, g["chanmap"], g["polmap"])
    v = K().degrid(torch.as_tensor(g["grid"]), g["uvw"], g["freq"], g["scale"][:2],
                   g["offset"][:2], g["chanmap"], g["polmap"], cf, support, os_,
                   flag=g["flag"], dphase=np.zeros((nt, nb)), nvchan=3, nvpol=4,
                   precision="fp32", accumulate=True)
    assert rel(v.cpu().numpy(), ref) <= 1e-6


@pytest.fixture(params=["tf32", "fp32", "tc05"])
def degrid_lanes(request):
    """Runs a test under each setting of the tiled degridder's fast store
    path: TF32 tensor-core tiles with split operands (warp MMAs, or MMAs with
    tensor-memory accumulators), and FP32 FMA."""
    from astroviper_b200 import _lib
    L = _lib.lib()
    old = L.av_tune_get(_lib.AV_TUNE_DEGRID_LANES)
    want = {"tf32": _lib.AV_DEGRID_LANES_TF32, "fp32": _lib.AV_DEGRID_LANES_FP32,
            "tc05": _lib.AV_DEGRID_LANES_TC05}[request.param]
    assert L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, want) == _lib.AV_OK
    yield request.param
    L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, old)


@pytest.mark.parametrize("polmap", [(0, 1, 2, 3), (2, 0, 3, 1)])
@pytest.mark.parametrize("support", [3, 4, 5, 6, 7, 8])
def test_degrid_fast_store_every_support(support, polmap, degrid_lanes):
    """The fast store path (complex64 values, 4 visibility and 4 grid
    polarisations, no flags or phase) against the oracle's dgrid_numba on a
    random 4-polarisation grid, for every support it covers and a permuted
    polarisation map; samples the degridder skips get zeros."""
    g = golden("degrid.npz")
    rng = np.random.default_rng(100 + support)
    nt, nb = g["uvw"].shape[:2]
    n2, n3 = g["grid"].shape[2:]
    grid = rng.normal(size=(2, 4, n2, n3)) + 1j * rng.normal(size=(2, 4, n2, n3))
    cf = O.create_prolate_spheroidal_kernel_1D(100, support)
    pm = np.array(polmap, dtype=np.int32)
    ref = np.zeros((nt, nb, 3, 4), complex)
    O.dgrid_numba(g["uvw"], np.zeros((nt, nb)), ref, np.zeros((nt, nb, 3, 4), bool),
                  g["scale"], g["offset"], grid, g["freq"], 299792458.0, support, 100, cf,
                  g["chanmap"], pm)
    v = K().degrid(torch.as_tensor(grid), g["uvw"], g["freq"], g["scale"][:2], g["offset"][:2],
                   g["chanmap"], pm, cf, support, 100, nvchan=3, nvpol=4, precision="fp32",
                   accumulate=False)
    assert v.dtype == torch.complex64
    assert rel(v.cpu().numpy(), ref) <= 1e-6


@pytest.mark.parametrize("polmap", [(0, -1, 2, 7), (1, 1, 0, 0)])
def test_degrid_fast_store_unmapped_and_repeated_polarisations(polmap, degrid_lanes):
    """The fast store path with a polarisation map that leaves outputs
    unmapped (-1, or past the grid's polarisations: zeros) or reads one grid
    polarisation twice: the mapped outputs match the FP64 degridder on the
    same grid polarisation, the unmapped ones are exactly zero."""
    g = golden("degrid.npz")
    rng = np.random.default_rng(7)
    nt, nb = g["uvw"].shape[:2]
    n2, n3 = g["grid"].shape[2:]
    grid = rng.normal(size=(2, 4, n2, n3)) + 1j * rng.normal(size=(2, 4, n2, n3))
    cf = O.create_prolate_spheroidal_kernel_1D(100, 7)
    pm = np.array(polmap, dtype=np.int32)
    v = K().degrid(torch.as_tensor(grid), g["uvw"], g["freq"], g["scale"][:2], g["offset"][:2],
                   g["chanmap"], pm, cf, 7, 100, nvchan=3, nvpol=4, precision="fp32",
                   accumulate=False).cpu().numpy()
    ident = np.arange(4, dtype=np.int32)
    ref = np.zeros((nt, nb, 3, 4), complex)
    O.dgrid_numba(g["uvw"], np.zeros((nt, nb)), ref, np.zeros((nt, nb, 3, 4), bool),
                  g["scale"], g["offset"], grid, g["freq"], 299792458.0, 7, 100, cf,
                  g["chanmap"], ident)
    for p, src in enumerate(polmap):
        if 0 <= src < 4:
            assert rel(v[..., p], ref[..., src]) <= 1e-6
        else:
            assert np.all(v[..., p] == 0)


@pytest.fixture(params=["mma", "rows"])
def grid_lanes(request):
    """Runs a test under each of the tiled gridder's lane mappings: FP64
    tensor-core tiles (supports up to 8) and a footprint row per lane."""
    from astroviper_b200 import _lib
    L = _lib.lib()
    old = L.av_tune_get(_lib.AV_TUNE_GRID_LANES)
    want = _lib.AV_GRID_LANES_MMA if request.param == "mma" else _lib.AV_GRID_LANES_ROWS
    assert L.av_tune_set(_lib.AV_TUNE_GRID_LANES, want) == _lib.AV_OK
    yield request.param
    L.av_tune_set(_lib.AV_TUNE_GRID_LANES, old)


@pytest.mark.parametrize("npol", [1, 2, 3, 4])
@pytest.mark.parametrize("support", [3, 4, 5, 6, 7, 8, 9])
def test_tiled_grid_every_support(support, npol, grid_lanes):
    """The tiled gridder against the oracle for every support and
    polarisation count (3 channels into 3 image channels)."""
    g = golden("degrid.npz")
    rng = np.random.default_rng(support * 10 + npol)
    nt, nb = g["uvw"].shape[:2]
    vis = (rng.normal(size=(nt, nb, 3, npol)) + 1j * rng.normal(size=(nt, nb, 3, npol)))
    wt = rng.uniform(0.5, 2.0, size=(nt, nb, 3, npol))
    cf = O.create_prolate_spheroidal_kernel_1D(100, support)
    cell = np.array([-1.0, 1.0]) * 20.0 * np.pi / (180 * 3600)
    rg, rs = O.standard_grid(vis, g["uvw"], wt, g["freq"], cf, np.array([64, 64]), cell,
                             support=support, chan_mode="cube")
    gr, sw = K().grid(vis.astype(np.complex64), torch.as_tensor(wt.astype(np.float32)), g["uvw"],
                      g["freq"], np.arange(3), np.arange(npol), cf, np.array([64, 64]), cell,
                      support, 100, 3, npol, precision="fp32")
    vis32 = vis.astype(np.complex64).astype(complex)
    wt32 = wt.astype(np.float32).astype(float)
    rg32, rs32 = O.standard_grid(vis32, g["uvw"], wt32, g["freq"], cf, np.array([64, 64]), cell,
                                 support=support, chan_mode="cube")
    assert rel(gr.cpu().numpy(), rg32) <= 1e-12
    assert np.allclose(sw.cpu().numpy(), rs32, rtol=1e-12)
    assert rel(gr.cpu().numpy(), rg) <= 1e-6


@pytest.mark.parametrize("npol", [2, 4])
def test_tiled_grid_unaligned_rows(npol, grid_lanes):
    """Visibility and weight arrays that start 8 / 4 bytes past a 16-byte
    boundary (views one element into larger buffers): the gridder copies
    them one polarisation at a time and must match the aligned result."""
    g = golden("degrid.npz")
    rng = np.random.default_rng(40 + npol)
    nt, nb = g["uvw"].shape[:2]
    shape = (nt, nb, 3, npol)
    vis = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    wt = rng.uniform(0.5, 2.0, size=shape).astype(np.float32)
    cf = O.create_prolate_spheroidal_kernel_1D(100, 7)
    cell = np.array([-1.0, 1.0]) * 20.0 * np.pi / (180 * 3600)
    args = (g["uvw"], g["freq"], np.arange(3), np.arange(npol), cf, np.array([64, 64]), cell,
            7, 100, 3, npol)
    va = torch.as_tensor(vis).cuda()
    wa = torch.as_tensor(wt).cuda()
    vbuf = torch.zeros(vis.size + 1, dtype=torch.complex64, device="cuda")
    wbuf = torch.zeros(wt.size + 1, dtype=torch.float32, device="cuda")
    vu = vbuf[1:].view(shape)
    wu = wbuf[1:].view(shape)
    vu.copy_(va)
    wu.copy_(wa)
    assert vu.data_ptr() % 16 == 8 and wu.data_ptr() % 16 == 4
    g0, s0 = K().grid(va, wa, *args, precision="fp32")
    g1, s1 = K().grid(vu, wu, *args, precision="fp32")
    assert rel(g1.cpu().numpy(), g0.cpu().numpy()) <= 1e-14
    assert np.allclose(s1.cpu().numpy(), s0.cpu().numpy(), rtol=1e-14)


def test_tiled_grid_long_runs_match_fp64(grid_lanes):
    """Runs of one cell that span many staged rounds (8 time steps of the
    33M-sample workload, continuum 2048^2, 4 polarisations): the tiled
    gridder against the plain FP64 gridder on the same complex64 inputs."""
    from astroviper_b200 import synthetic as S
    W = S.workload_large(n_time=8, n_chan=16, device=torch.device("cuda"))
    nt, nb, nchan, npol = W["vis"].shape
    cf = O.create_prolate_spheroidal_kernel_1D(100, 7)
    wt = torch.rand(W["vis"].shape, dtype=torch.float32, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(5)) + 0.5
    args = (W["uvw"], W["freq"], np.zeros(nchan, int), np.arange(npol), cf, W["image_size"],
            W["pixelincr"], 7, 100, 1, npol)
    g32, s32 = K().grid(W["vis"], wt, *args, precision="fp32")
    g64, s64 = K().grid(W["vis"].to(torch.complex128), wt.double(), *args, precision="fp64")
    assert rel(g32.cpu().numpy(), g64.cpu().numpy()) <= 1e-12
    assert np.allclose(s32.cpu().numpy(), s64.cpu().numpy(), rtol=1e-12)


def test_degrid_store_mode_four_pol_fast_output(degrid_lanes):
    """Store mode, complex64, 4 polarisations, no flags / phase: the kernel
    writes each sample's 4 values as two 16-byte stores with FP32 scaling;
    against the FP64 plain degridder on a slice of the 33M workload."""
    from astroviper_b200 import synthetic as S
    from astroviper_b200.gridder import Gridder
    W = S.workload_large(n_time=4, device=torch.device("cuda"))
    nt, nb, nchan, npol = W["vis"].shape
    G = Gridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], npol)
    wt = torch.ones(W["vis"].shape, dtype=torch.float32, device="cuda")
    g, _ = G.grid(W["vis"], wt)
    v = G.degrid(g)  # store mode, fresh complex64 values
    nx, ny = (int(x) for x in W["image_size"])
    ref = K().degrid(g, W["uvw"], W["freq"], (-W["pixelincr"][0] * nx, -W["pixelincr"][1] * ny),
                     (nx / 2, ny / 2), np.zeros(nchan, int), np.arange(npol), G.cgk, 7, 100,
                     nvchan=nchan, nvpol=npol, precision="fp64")
    assert rel(v.cpu().numpy(), ref.cpu().numpy()) <= 1e-6


def test_fp64_mma_probe_reports_a_rate():
    """The FP64 tensor-rate probe runs and returns a plausible B200 figure."""
    import ctypes
    from astroviper_b200 import _lib
    v = ctypes.c_double(0.0)
    assert _lib.lib().av_probe_fp64_mma(ctypes.byref(v), None) == _lib.AV_OK
    assert 5.0 < v.value < 200.0
    assert _lib.lib().av_probe_fp64_mma(None, None) == _lib.AV_ERR_ARG
