#!/usr/bin/env python
"""Benchmark of the standard-gridder imaging path on B200.

Workload (the reference's 33M-visibility imaging case, synthetic data of its
shape): 64 antennas in a 2 km disk, 2016 baselines x 256 time steps of 10 s x
64 channels (1.0-1.5 GHz) x 4 polarisations = 33.03 M visibilities
(132 M correlations), complex64, Briggs robust 0.5 imaging weights, one
continuum 2048^2 grid of 1 arcsec cells, PSWF support 7, oversampling 100.

One step = grid (binning plan + FP64-accumulating tiled gridder) + degrid
(binning plan + tiled degridder) of all samples, inputs resident in HBM
(1.06 GB of visibilities per step, larger than L2).  Metric: Mvis/s of the
grid+degrid pair.  Also reported: the plain FP64 GPU gridder on the same GPU,
relative errors against the FP64 path (grid, dirty image, degridded
visibilities), Hogbom CLEAN iterations/s, the CPU oracle timed on this host
and an end-to-end number through the numpy drop-in API with host buffers.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mvis/s grid+degrid on 1 B200 at <=1e-5 rel err vs FP64; CLEAN iter/s"
WORKLOAD = ("64 ant (2016 bl) x 256 t x 64 ch x 4 pol = 33.03M vis, complex64, Briggs 0.5, "
            "2048^2 continuum, 1 arcsec, support 7, oversampling 100")
N_TIME = 256          # time steps of the full workload
CPU_SAMPLE_T = 64     # time steps of one CPU step: 8.26M vis, 33.0M corr
CPU_SINGLE_T = 8      # time steps for the one-thread rate


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n-time", type=int, default=N_TIME)
    ap.add_argument("--quick", action="store_true", help="skip CPU baseline / CLEAN / e2e")
    ap.add_argument("--no-clean", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-forward", action="store_true")
    ap.add_argument("--no-imager", action="store_true")
    ap.add_argument("--no-mosaic", action="store_true")
    ap.add_argument("--clean-iters", type=int, default=20000)
    ap.add_argument("--degrid-lanes", default="auto", choices=["auto", "tf32", "fp32", "tc05"],
                    help="the degridder's fast store path: the library's choice (auto), warp "
                         "TF32 MMAs, FP32 FMA, or tcgen05 MMAs with tensor-memory accumulators")
    return ap.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled every 2 ms during
    the timed region through NVML (read-only queries), in a thread; falls
    back to nvidia-smi polling when NVML is unavailable."""
    NAMES = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, gpu_index, period_s=0.002):
        self.gpu_index = gpu_index
        self.period = period_s
        self.rows = []
        self.nv = None
        self.h = None
        self._stop = threading.Event()
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            uuid = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
            self.h = nv.nvmlDeviceGetHandleByUUID(uuid)
            self.nv = nv
        except Exception:
            self.nv = None

    def _poll(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.rows.append((sm, mx, rs))
            except Exception:
                pass
            self._stop.wait(self.period)

    def start(self):
        if self.nv is None:
            return
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

    def stop(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable"],
                    "samples": 0}
        self._stop.set()
        self.t.join(timeout=2)
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows]
        reasons = set()
        for _, _, rs in self.rows:
            for nm, attr in self.NAMES.items():
                if rs & getattr(self.nv, attr, 0):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows), "source": "NVML, 2 ms"}


# DRAM bytes read + written per launch and per visibility of the main
# kernels, from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum)
# of the 8.26M-visibility case (64 time steps): k_grid_mma 481.40 MB,
# k_grid_tiled (row lanes) 484.11 MB, k_degrid_tc 286.43 MB, k_degrid_tiled
# 286.84 MB.  The traffic is per record, so it scales with the visibilities.
NCU_VIS = 64 * 2016 * 64
DRAM_BYTES_PER_VIS = {"k_grid_mma": 481.40e6 / NCU_VIS, "k_grid_tiled": 484.11e6 / NCU_VIS,
                      "k_degrid_tc": 286.43e6 / NCU_VIS, "k_degrid_tiled": 286.84e6 / NCU_VIS}


def max_over_ranks(ms, world, device=None):
    """The slowest rank's time (every rank calls this; one rank: unchanged)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def max_elem_err(a, b):
    """max |a - b| / max(|b|, 1e-7 max |b|) over the elements: the per-element
    error with an absolute floor of 1e-7 of the largest reference value."""
    import torch
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    mag = b.abs()
    floor = 1e-7 * float(mag.max())
    return float(((a - b).abs() / torch.clamp(mag, min=floor)).max()) if floor > 0 else 0.0


def rel(a, b):
    import torch
    if isinstance(a, torch.Tensor):
        a = a.double() if not a.is_complex() else a.to(torch.complex128)
        b = b.double() if not b.is_complex() else b.to(torch.complex128)
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


# ---------------------------------------------------------------------------
# CPU side (oracle port on the host cores)
# ---------------------------------------------------------------------------
def bench_config(world, n_time=None):
    """The workload description, the same in both arms."""
    n_vis = (n_time or N_TIME) * 2016 * 64
    return {"workload": WORKLOAD, "n_vis": n_vis, "n_corr": 4 * n_vis,
            "l2": "inputs larger than L2 (1.06 GB visibilities per step)",
            "step": "plan (one for both directions)+grid+degrid; grid cleared, model "
                    "visibilities written each step",
            "parallelism": f"replicas x{world}"}


def host_threads():
    """Host threads this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_sample(uvw, vis, weight, freq, image_size, pixelincr):
    """A host sample for the CPU legs, converted once to the oracle's dtypes
    (complex128 visibilities, float64 weights) outside any timing."""
    return {"uvw": np.ascontiguousarray(uvw, dtype=np.float64),
            "vis": np.ascontiguousarray(vis, dtype=np.complex128),
            "wt": np.ascontiguousarray(weight, dtype=np.float64),
            "flag": np.zeros(vis.shape, np.uint8), "freq": np.asarray(freq, np.float64),
            "image_size": image_size, "pixelincr": pixelincr}


def cpu_grid_degrid(smp, nthreads, t_steps=None):
    """The oracle's C restatement of the reference's Numba kernels on the
    host: standard_grid_jit (rows of the grid owned by threads) then
    dgrid_numba (time steps split over threads) of the sample's first
    ``t_steps`` time steps.  Returns (seconds, vis processed)."""
    import oracle as O
    t = smp["uvw"].shape[0] if t_steps is None else t_steps
    uvw, vis, wt, flag = smp["uvw"][:t], smp["vis"][:t], smp["wt"][:t], smp["flag"][:t]
    cgk = O.create_prolate_spheroidal_kernel_1D(100, 7)
    t0 = time.perf_counter()
    g, _sw = O.standard_grid(vis, uvw, wt, smp["freq"], cgk, smp["image_size"],
                             smp["pixelincr"], nthreads=nthreads, rows=True)
    O.degrid(g, uvw, smp["freq"], smp["pixelincr"], flag=flag, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return dt, uvw.shape[0] * uvw.shape[1] * len(smp["freq"])


def cpu_baseline_leg(smp, nthreads, reps=1):
    """cpu_baseline object: the N-thread rate on the whole sample (mean of
    ``reps`` runs after one untimed run) and the one-thread rate on its first
    CPU_SINGLE_T steps."""
    times = []
    for i in range(reps + 1):  # the first run warms the allocator and the caches
        dt, nv = cpu_grid_degrid(smp, nthreads)
        if i > 0:
            times.append(dt)
    dt1, nv1 = cpu_grid_degrid(smp, 1, CPU_SINGLE_T)
    t = smp["uvw"].shape[0]
    return {"value": nv / float(np.mean(times)) / 1e6, "unit": "Mvis/s", "cores": nthreads,
            "kind": "port",
            "sample": f"first {t} of {N_TIME} time steps ({nv} vis, {4 * nv} corr), Briggs 0.5 "
                      "weights: the oracle's C restatement of standard_grid_jit (grid rows "
                      "owned by threads) + dgrid_numba (time steps split over threads)",
            "single_thread": {"value": nv1 / dt1 / 1e6, "unit": "Mvis/s",
                              "sample": f"first {CPU_SINGLE_T} time steps ({nv1} vis)"},
            "host_cpus": os.cpu_count(), "threads_allowed": host_threads()}


def host_briggs_weights(uvw_all, freq, image_size, pixelincr, robust, t_sample, npol):
    """Briggs imaging weights of the first ``t_sample`` time steps with the
    density of every step (unit data weights), through the oracle: the same
    weights the GPU arm computes on the device."""
    import oracle as O
    nt, nb = uvw_all.shape[:2]
    nchan = len(freq)
    nu, nv = int(image_size[0]), int(image_size[1])
    G = np.zeros((nchan, 1, nu, nv), dtype=np.float64)
    sw = np.zeros((nchan, 1), dtype=np.float64)
    O.grid_imaging_weights_jit(G, sw, uvw_all, freq, np.arange(nchan),
                               np.ones((nt, nb, nchan, 1)), np.array([nu, nv]), pixelincr)
    bf = O.calculate_briggs_params(G, sw, {"weighting": "briggs", "robust": robust})
    iw = np.zeros((t_sample, nb, nchan, 1), dtype=np.float64)
    O.degrid_imaging_weights_jit(iw, G, bf, np.ascontiguousarray(uvw_all[:t_sample]), freq,
                                 np.arange(nchan), np.arange(1), np.ones((t_sample, nb, nchan, 1)),
                                 np.array([nu, nv]), pixelincr)
    return np.repeat(iw, npol, axis=3)


def reference_arm(args, rank, world):
    """Times the reference's CPU implementation of the path (the oracle's C
    restatement of its Numba gridder and degridder; the reference itself is
    Python+Numba, its sources do not travel) with every host thread this
    process may use, each step one grid+degrid of the first CPU_SAMPLE_T of
    the workload's 256 time steps with the workload's Briggs weights."""
    if rank != 0:
        return
    from astroviper_b200 import synthetic as S
    W = S.workload_large(n_time=N_TIME, time_slice=slice(0, CPU_SAMPLE_T))
    iw = host_briggs_weights(W["uvw_all"], W["freq"], W["image_size"], W["pixelincr"],
                             W["robust"], CPU_SAMPLE_T, W["vis"].shape[3])
    smp = cpu_sample(W["uvw"], W["vis"], iw, W["freq"], W["image_size"], W["pixelincr"])
    del W, iw
    nthreads = host_threads()
    times = []
    for i in range(args.warmup + args.steps):
        dt, nvis = cpu_grid_degrid(smp, nthreads)
        if i >= args.warmup:
            times.append(dt)
    ms = 1e3 * float(np.mean(times))
    value = nvis / (ms / 1e3) / 1e6
    dt1, nv1 = cpu_grid_degrid(smp, 1, CPU_SINGLE_T)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mvis/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": bench_config(world),
        "cpu_baseline": {
            "value": value, "unit": "Mvis/s", "cores": nthreads, "kind": "port",
            "sample": f"each step: first {CPU_SAMPLE_T} of {N_TIME} time steps ({nvis} vis, "
                      f"{4 * nvis} corr), Briggs 0.5 weights; the oracle's C restatement of "
                      "standard_grid_jit (grid rows owned by threads) + dgrid_numba (time steps "
                      "split over threads)",
            "single_thread": {"value": nv1 / dt1 / 1e6, "unit": "Mvis/s",
                              "sample": f"first {CPU_SINGLE_T} time steps ({nv1} vis)"},
            "host_cpus": os.cpu_count(), "threads_allowed": nthreads},
        "e2e": {"value": value, "unit": "Mvis/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import _lib
    from astroviper_b200 import synthetic as S
    from astroviper_b200.gridder import Gridder
    if args.degrid_lanes != "auto":
        lanes = {"tf32": _lib.AV_DEGRID_LANES_TF32, "fp32": _lib.AV_DEGRID_LANES_FP32,
                 "tc05": _lib.AV_DEGRID_LANES_TC05}[args.degrid_lanes]
        _lib.check(_lib.lib().av_tune_set(_lib.AV_TUNE_DEGRID_LANES, lanes), "av_tune_set")
    dev = torch.device("cuda", local)
    n_time = args.n_time

    # ---------------------------------------------------------------- inputs
    W = S.workload_large(n_time=n_time, device=dev)
    vis = W["vis"]
    nt, nb, nchan, npol = (int(s) for s in vis.shape)
    n_vis = nt * nb * nchan
    n_corr = n_vis * npol
    img = W["image_size"]
    cell = W["pixelincr"]
    # Briggs robust 0.5 imaging weights (unit data weights, no flags), once
    ones = torch.ones((nt, nb, nchan, npol), dtype=torch.float32, device=dev)
    dens, swd = K.weight_density(W["uvw"], W["freq"], ones, None, img, cell)
    bf = K.briggs_factors(dens, swd, W["robust"])
    iw, err = K.briggs_apply(dens, bf, W["uvw"], W["freq"], ones, None, img, cell,
                             out_dtype=torch.float32)
    assert int(err.item()) == 0
    del dens, ones
    G = Gridder(W["uvw"], W["freq"], img, cell, npol, support=7, oversampling=100)
    grid = G.new_grid()
    sumw = torch.zeros((1, npol), dtype=torch.float64, device=dev)
    values = torch.zeros((nt, nb, nchan, npol), dtype=torch.complex64, device=dev)

    def step(ev=None):
        G._gplan = None  # the binning plans are rebuilt every step (counted in the time)
        G._dplan = None
        G.plan()         # one plan for both directions
        G.clear_grid(grid)  # the cells the plan can touch (the rest stays zero)
        sumw.zero_()
        if ev is not None:
            ev[0].record()
        G.grid(vis, iw, grid=grid, sum_weight=sumw)
        if ev is not None:
            ev[1].record()
        G.degrid(grid, values=values)  # values = model (every element written once)
        if ev is not None:
            ev[2].record()

    # ------------------------------------------------------- warm-up / timing
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    # kernel-only timing of the two main kernels (plans built outside)
    G._gplan = None
    G._dplan = None
    G.grid(vis, iw, grid=grid.zero_(), sum_weight=sumw.zero_())
    G.degrid(grid, values=values)
    torch.cuda.synchronize()
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(3)]
    for a, b, c in kev:
        grid.zero_()
        a.record()
        G.grid(vis, iw, grid=grid, sum_weight=sumw)   # plan reused: the grid kernel alone
        b.record()
        G.degrid(grid, values=values)                 # plan reused: the degrid kernel alone
        c.record()
    torch.cuda.synchronize()
    t_grid_k = float(np.mean([a.elapsed_time(b) for a, b, c in kev]))
    t_degrid_k = float(np.mean([b.elapsed_time(c) for a, b, c in kev]))
    from astroviper_b200 import _lib
    # support 7: the tensor-core kernels unless the lane knobs force the others
    # (read now: later legs may tune the knobs)
    grid_kernel = ("k_grid_tiled" if _lib.lib().av_tune_get(_lib.AV_TUNE_GRID_LANES) ==
                   _lib.AV_GRID_LANES_ROWS else "k_grid_mma")
    degrid_kernel = {_lib.AV_DEGRID_LANES_FP32: "k_degrid_tiled",
                     _lib.AV_DEGRID_LANES_TC05: "k_degrid_umma"}.get(
        _lib.lib().av_tune_get(_lib.AV_TUNE_DEGRID_LANES), "k_degrid_tc")

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = _lib.lib().av_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    launches = int(_lib.lib().av_launch_count() - launches0)
    if degrid_kernel == "k_degrid_umma":  # its bounded waits must all have held
        import ctypes
        fault = ctypes.c_int(-1)
        _lib.check(_lib.lib().av_degrid_fault_read(ctypes.byref(fault), 1, K.stream_ptr()),
                   "av_degrid_fault_read")
        if fault.value:
            raise RuntimeError("k_degrid_umma: a wait for its MMAs gave up")
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
    value = n_vis * world / (ms / 1e3) / 1e6

    # ---------------------------------------------------------------- accuracy
    # FP64 references on a sample of the time steps: the plain FP64 gridder /
    # degridder (the reference's per-sample arithmetic in FP64)
    ts = max(1, nt // 8)
    uvw_s = W["uvw"][:ts]
    vis_s = vis[:ts].to(torch.complex128)
    iw_s = iw[:ts].to(torch.float64)
    Gs = Gridder(uvw_s, W["freq"], img, cell, npol, support=7, oversampling=100)
    g32, s32 = Gs.grid(vis[:ts], iw[:ts])
    torch.cuda.synchronize()
    pa = torch.cuda.Event(enable_timing=True)
    pb = torch.cuda.Event(enable_timing=True)
    pa.record()
    g64, s64 = K.grid(vis_s, iw_s, uvw_s, W["freq"], np.zeros(nchan, int), np.arange(npol),
                      G.cgk, img, cell, 7, 100, 1, npol, precision="fp64")
    pb.record()
    torch.cuda.synchronize()
    t_plain = pa.elapsed_time(pb)
    plain_mvis = ts * nb * nchan / (t_plain / 1e3) / 1e6
    err_grid = rel(g32, g64)
    mx_grid = max_elem_err(g32, g64)
    im32 = Gs.image(g32, s32)
    im64 = Gs.image(g64, s64)
    err_img = rel(im32, im64)
    mx_img = max_elem_err(im32, im64)
    # PSF: the weights gridded (do_psf) and imaged, FP32-input tiled path
    # against the FP64 plain gridder
    p32, ps32 = Gs.grid(None, iw[:ts], do_psf=True)
    p64, ps64 = K.grid(None, iw_s, uvw_s, W["freq"], np.zeros(nchan, int), np.arange(npol),
                       G.cgk, img, cell, 7, 100, 1, npol, do_psf=True, precision="fp64")
    pi32, pi64 = Gs.image(p32, ps32), Gs.image(p64, ps64)
    err_psf = rel(pi32, pi64)
    mx_psf = max_elem_err(pi32, pi64)
    del p32, p64, pi32, pi64
    v32 = Gs.degrid(g64)
    nx, ny = int(img[0]), int(img[1])
    v64 = K.degrid(g64, uvw_s, W["freq"], (-cell[0] * nx, -cell[1] * ny), (nx / 2, ny / 2),
                   (np.arange(nchan) / nchan * 1).astype(int), np.arange(npol) % npol, G.cgk, 7,
                   100, nvchan=nchan, nvpol=npol, precision="fp64")
    err_vis = rel(v32, v64)
    mx_vis = max_elem_err(v32, v64)
    del g64, v64, v32, vis_s
    torch.cuda.empty_cache()

    # ------------------------------------------------------------------- CLEAN
    clean = None
    if not (args.quick or args.no_clean) and rank == 0:
        clean = bench_clean(args, dev)

    # ------------------------------------------------------- forward model
    forward = None
    if not (args.quick or args.no_forward) and rank == 0:
        forward = bench_forward(args, dev)

    # ------------------------------------------------------ imaging loop
    imaging = None
    if not (args.quick or args.no_imager) and rank == 0:
        imaging = bench_imager(args, dev)

    mosaic = None
    if not (args.quick or args.no_mosaic) and rank == 0:
        mosaic = bench_mosaic(args, dev)

    # ------------------------------------------------------------- batched
    batched = None
    if not (args.quick or args.no_batched) and rank == 0:
        del G, grid, values
        torch.cuda.empty_cache()
        from astroviper_b200 import _lib
        knobs = {k: _lib.lib().av_tune_get(k) for k in range(5)}
        batched = bench_batched(args, dev)
        for k, v in knobs.items():  # the autotuner's choices were for that workload
            _lib.check(_lib.lib().av_tune_set(k, v), "av_tune_set")
        G = Gridder(W["uvw"], W["freq"], img, cell, npol, support=7, oversampling=100)

    # ------------------------------------------------------------ CPU baseline
    cpu = None
    if not (args.quick or args.no_cpu) and rank == 0:
        tsc = min(CPU_SAMPLE_T, nt)
        smp = cpu_sample(W["uvw"][:tsc], vis[:tsc].cpu().numpy(), iw[:tsc].cpu().numpy(),
                         W["freq"], img, cell)
        cpu = cpu_baseline_leg(smp, host_threads(), reps=2)
        del smp

    # --------------------------------------------------------------------- e2e
    e2e = None
    if not (args.quick or args.no_e2e):
        e2e = bench_e2e(W, vis, iw, G)

    peak, peak_kind = load_peaks()
    bytes_grid = n_corr * 12 + nt * nb * 24 + nx * ny * npol * 8
    bytes_degrid = n_corr * 9 + nt * nb * 24 + nx * ny * npol * 8
    dom = (grid_kernel, bytes_grid, t_grid_k) if t_grid_k >= t_degrid_k else \
        (degrid_kernel, bytes_degrid, t_degrid_k)
    achieved = dom[1] / (dom[2] / 1e3) / 1e9
    # the gridder's FP64 footprint sums against the device's FP64 tensor rate:
    # 49 taps x 2 FMA per correlation plus the 49 tap products per sample
    import ctypes
    fp64_peak = ctypes.c_double(0.0)
    fp64_tensor = None
    if _lib.lib().av_probe_fp64_mma(ctypes.byref(fp64_peak), None) == 0 and fp64_peak.value > 0:
        grid_flops = n_corr * 196 + n_vis * 49
        ach = grid_flops / (t_grid_k / 1e3) / 1e12
        fp64_tensor = {"kernel": grid_kernel, "achieved": ach, "peak": fp64_peak.value,
                       "unit": "TFLOP/s", "frac": ach / fp64_peak.value,
                       "flops": grid_flops,
                       "peak_source": "av_probe_fp64_mma (mma.sync.m16n8k4.f64) on this GPU"}
    line = {
        "metric": METRIC, "value": value, "unit": "Mvis/s", "n_gpus": world,
        "Mcorr_per_s": value * npol,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": bench_config(world, n_time),
        "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "traffic": DRAM_BYTES_PER_VIS[dom[0]] * n_vis,
                     "traffic_source": "ncu dram bytes of the 8.26M-vis case, scaled by vis",
                     "peak_kind": peak_kind, "algorithmic_bytes": dom[1],
                     "kernel_ms": dom[2]},
        "fp64_tensor": fp64_tensor,
        "kernels_ms": {"grid_tiled": t_grid_k, "degrid_tiled": t_degrid_k,
                       "plan_and_rest": ms - t_grid_k - t_degrid_k,
                       "degrid_kernel": degrid_kernel},
        "fp64_plain_gridder": {"value": plain_mvis, "unit": "Mvis/s",
                               "sample": f"{ts} of {nt} time steps"},
        "speedup_vs_fp64_plain": (n_vis / (t_grid_k / 1e3) / 1e6) / plain_mvis,
        "rel_err_vs_fp64": {"grid": err_grid, "dirty_image": err_img, "psf": err_psf,
                            "degrid_vis": err_vis, "sample": f"{ts} of {nt} time steps"},
        "max_elem_err_vs_fp64": {"grid": mx_grid, "dirty_image": mx_img, "psf": mx_psf,
                                 "degrid_vis": mx_vis,
                                 "definition": "max |x - x64| / max(|x64|, 1e-7 max |x64|)"},
        "clocks": clk,
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clean": clean,
        "batched_uneven": batched,
        "forward_model": forward,
        "imaging_loop": imaging,
        "mosaic_grid": mosaic,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def bench_batched(args, dev):
    """Batched uneven gridding: 128 channels x 2 polarisations of the array at
    496 time steps = 256 independent 1024^2 grids (cube mode, 2 arcsec
    cells), each with a flag fraction uniform in [0, 0.6) (zero weights).
    For support 7 and 9: the persistent gridder over all grids in one launch
    replayed as a CUDA graph (lane mapping and chunks per SM from the
    autotuner; only the cells the plan can touch cleared between calls), the
    same launch without the graph, the graph that also rebuilds the plan from
    each batch's weights and leaves fully flagged samples out, one launch per
    grid (plan per channel), and the plain FP64 gridder; error of the batched
    grids against the FP64 ones.  Also the support the aliasing criterion
    picks (support="auto")."""
    import torch
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import autotune
    from astroviper_b200 import synthetic as S
    from astroviper_b200.batched import BatchedGridder, PerGridGridder
    W = S.workload_batched(device=dev)
    vis, wt = W["vis"], W["weight"]
    nt, nb, nchan, npol = (int(x) for x in vis.shape)
    per_grid = wt.sum(dim=(0, 1)).flatten().cpu().numpy()
    out = {"grids": nchan * npol, "image": int(W["image_size"][0]),
           "samples": nt * nb * nchan, "corr_unflagged": int(per_grid.sum()),
           "corr_per_grid_min": int(per_grid.min()), "corr_per_grid_max": int(per_grid.max())}

    def timed(fn, reps):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    for support in (7, 9):
        r = {}
        B = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], npol,
                           support=support, graph=True, tune=True)
        B(vis, wt)  # tunes the launch knobs, captures the graph
        r["tuned"] = autotune._applied.get(B.tune_key())
        sv, sw = B.static_inputs()
        r["graph_ms"] = timed(lambda: B(sv, sw), 5)             # replay, inputs in place
        r["graph_with_input_copy_ms"] = timed(lambda: B(vis, wt), 3)
        B.graph = False
        r["launch_ms"] = timed(lambda: B(vis, wt), 3)
        r["Mvis_per_s"] = nt * nb * nchan / (r["graph_ms"] / 1e3) / 1e6
        r["Mcorr_unflagged_per_s"] = out["corr_unflagged"] / (r["graph_ms"] / 1e3) / 1e6
        gb = B.grid.clone()
        del B
        torch.cuda.empty_cache()
        # the plan rebuilt from every batch's weights, fully flagged samples left out
        Bd = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], npol,
                            support=support, graph=True, tune=True, drop_flagged=True)
        Bd(vis, wt)
        sv, sw = Bd.static_inputs()
        r["drop_flagged_graph_ms"] = timed(lambda: Bd(sv, sw), 5)
        r["drop_flagged_rel_diff"] = rel(Bd.grid, gb)
        r["drop_flagged_Mcorr_unflagged_per_s"] = (out["corr_unflagged"] /
                                                   (r["drop_flagged_graph_ms"] / 1e3) / 1e6)
        del Bd
        torch.cuda.empty_cache()
        P = PerGridGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], npol,
                           support=support)
        parts = P.split(vis, wt)
        P(parts)
        r["per_grid_ms"] = timed(lambda: P(parts), 2)
        r["per_grid_launches"] = len(parts)
        del P, parts
        torch.cuda.empty_cache()
        cgk = K.pswf_table(100, support)
        v64 = vis.to(torch.complex128)
        w64 = wt.to(torch.float64)
        t64 = {}

        def fp64():
            t64["g"], _ = K.grid(v64, w64, W["uvw"], W["freq"], np.arange(nchan), np.arange(npol),
                                 cgk, W["image_size"], W["pixelincr"], support, 100, nchan, npol,
                                 precision="fp64")
        r["fp64_plain_ms"] = timed(fp64, 1)
        r["rel_err_vs_fp64"] = rel(gb, t64["g"])
        r["speedup_vs_per_grid"] = r["per_grid_ms"] / r["graph_ms"]
        r["speedup_vs_fp64_plain"] = r["fp64_plain_ms"] / r["graph_ms"]
        del v64, w64, t64, gb
        torch.cuda.empty_cache()
        out[f"support_{support}"] = r
    Ba = BatchedGridder(W["uvw"], W["freq"], W["image_size"], W["pixelincr"], npol,
                        support="auto", graph=False)
    out["support_auto"] = {"support": Ba.support, "alias_ratio": Ba.alias,
                           "criterion": "aliasing at the edge of the inner 80 % of the field "
                                        "<= 1e-2"}
    del Ba, W, vis, wt
    torch.cuda.empty_cache()
    return out


def bench_forward(args, dev):
    """Differentiable forward model: 1024^2 FP32 image -> grid correction ->
    FFT -> degrid to 4.16M visibilities (128 antennas, 128 steps, 4 channels,
    1 pol; truth 200 Gaussian blobs plus N(0, 0.01) noise), chi-squared
    steepest descent for 200 steps with the hand-written adjoint as the
    backward."""
    import torch
    from astroviper_b200 import synthetic as S
    from astroviper_b200.forward_model import ForwardModel, chi2_solve
    F = S.workload_forward()
    n = int(F["image_size"][0])
    m = ForwardModel(F["uvw"], F["freq"], (n, n), F["cell"], npol=1, precision="fp32")
    truth = torch.as_tensor(F["truth"], device=dev)
    v_obs = m.forward_op(truth)
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    noise = torch.complex(torch.randn(v_obs.shape, generator=g, device=dev),
                          torch.randn(v_obs.shape, generator=g, device=dev))
    v_obs = (v_obs + F["noise_sigma"] * noise).contiguous()
    n_vis = int(v_obs.numel())

    def timed(fn, reps=5):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    fwd_ms = timed(lambda: m.forward_op(truth))
    adj_ms = timed(lambda: m.adjoint_op(v_obs))
    steps = 200
    chi2_solve(m, v_obs, steps=2)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x, hist = chi2_solve(m, v_obs, steps=steps)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"n_vis": n_vis, "image": n, "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
            "steps": steps, "ms_per_step": dt / steps * 1e3,
            "chi2_first": hist[0], "chi2_last": hist[-1],
            "chi2_reduction": hist[-1] / hist[0],
            "step": "forward (autograd) + adjoint backward + forward for the line search"}


def bench_clean(args, dev):
    """Hogbom CLEAN: 2048^2 FP32 dirty image of 50 sources, 4096^2 PSF of the
    small array's sampling, gain 0.1, up to clean_iters iterations or 1 mJy."""
    import torch
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import synthetic as S
    cw = S.clean_workload(nx=2048, psf_factor=2, n_src=50)
    out = {}
    for name, psf in (("psf_4096", cw["psf"]), ("psf_2048", cw["psf"][1024:3072, 1024:3072])):
        run = K.HogbomRun(torch.as_tensor(cw["dirty"]), torch.as_tensor(np.ascontiguousarray(psf)),
                          niter=args.clean_iters, gain=0.1, threshold=1e-3)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        run.run(0, args.clean_iters)
        b.record()
        torch.cuda.synchronize()
        st = run.read_state()
        ms = a.elapsed_time(b)
        out[name] = {"iterations": st["iter"], "ms": ms, "iter_per_s": st["iter"] / (ms / 1e3),
                     "stopped_by_threshold": bool(st["stopped"])}
    # CPU: the reference's own Hogbom module (built from its C++ sources), a
    # bounded number of iterations on the same-size PSF
    try:
        import glob
        import importlib.util
        so = glob.glob(os.path.join(ROOT, "oracle", "_ref", "_hogbom_ext*.so"))
        spec = importlib.util.spec_from_file_location("_hogbom_ext", so[0])
        H = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(H)
        n_cpu = 200
        psf = np.ascontiguousarray(cw["psf"][1024:3072, 1024:3072])
        t0 = time.perf_counter()
        ref = H.clean(cw["dirty"], psf, max_iter=n_cpu, gain=0.1, threshold=1e-3)
        dt = time.perf_counter() - t0
        out["cpu_reference"] = {"iter_per_s": n_cpu / dt, "cores": 1, "kind": "reference",
                                "sample": f"{n_cpu} iterations, 2048^2, same-size PSF"}
        out["speedup_psf_2048"] = out["psf_2048"]["iter_per_s"] / (n_cpu / dt)
        # the same first iterations on the GPU: components (model image) and
        # residual against the reference module
        run = K.HogbomRun(torch.as_tensor(cw["dirty"]), torch.as_tensor(psf), niter=n_cpu,
                          gain=0.1, threshold=1e-3)
        run.run(0, n_cpu)
        model = run.model.cpu().numpy()
        resid = run.resid.cpu().numpy()
        # the FP32 CLEAN model against the same iterations in FP64
        run64 = K.HogbomRun(torch.as_tensor(cw["dirty"].astype(np.float64)),
                            torch.as_tensor(psf.astype(np.float64)), niter=n_cpu, gain=0.1,
                            threshold=1e-3)
        run64.run(0, n_cpu)
        m64 = run64.model.cpu().numpy()
        out["model_fp32_vs_fp64"] = {
            "iterations": n_cpu,
            "same_component_positions": bool(np.array_equal(model != 0, m64 != 0)),
            "rel_err": float(np.linalg.norm(model - m64) / np.linalg.norm(m64)),
        }
        out["components_vs_reference"] = {
            "iterations": n_cpu,
            "model_bit_exact": bool(np.array_equal(model, ref["model_image"])),
            "residual_bit_exact": bool(np.array_equal(resid, ref["residual_image"])),
            "n_components": int(np.count_nonzero(ref["model_image"])),
            "max_flux_rel_diff": float(np.max(np.abs(model - ref["model_image"])) /
                                       max(1e-30, float(np.max(np.abs(ref["model_image"]))))),
        }
    except Exception as e:  # the compiled reference module is optional
        out["cpu_reference"] = {"unavailable": str(e)}
    return out


def bench_imager(args, dev):
    """run_imaging_loop (the major/minor-cycle imager) on the small workload
    (64 antennas, 50 x 2016 x 1 ch x 2 pol, 512^2, Hogbom niter 1000 over at
    most 5 major cycles, cyclefactor 1.5), timed end to end from the host
    arrays (copies in, every cycle, columns written back), against the
    oracle's restatement of the same loop on one host core."""
    import oracle.imager as OI
    from astroviper_b200 import synthetic as S
    from astroviper_b200.core.imaging.imager import run_imaging_loop
    from astroviper_b200.core.imaging.imaging_utils import iteration_control as IC
    from astroviper_b200.core.imaging.imaging_utils.return_dict import ReturnDict
    import torch
    node, geo = S.ms4_small()
    params = dict(geo, niter=1000, nmajor=5, cyclefactor=1.5, gain=0.1, threshold=0.0,
                  chan_mode="cube")
    vis0 = node["VISIBILITY"].data.copy()
    uvw0, w0, f0 = node.UVW.data.copy(), node.WEIGHT.data.copy(), node.FLAG.data.copy()
    freq = node.coords["frequency"].values

    def fresh():
        return S.Ms4Node(vis0.copy(), uvw0.copy(), w0.copy(), f0.copy(), freq, ["XX", "YY"])

    run_imaging_loop(fresh(), params)  # warm-up (library load, plans, FFT plans)
    times = []
    for _ in range(3):
        ms = fresh()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        model, resid, _rd, ctl = run_imaging_loop(ms, params)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t_gpu = sorted(times)[1]
    octl = IC.IterationController(niter=params["niter"], nmajor=params["nmajor"],
                                  threshold=params["threshold"], gain=params["gain"],
                                  cyclefactor=params["cyclefactor"])
    t0 = time.perf_counter()
    ref = OI.run_imaging_loop(vis0.copy(), uvw0.copy(), w0.copy(), f0.copy(), freq, params, octl,
                              IC.merge_return_dicts, ReturnDict)
    t_cpu = time.perf_counter() - t0
    return {"value": t_gpu * 1e3, "unit": "ms per run_imaging_loop call",
            "higher_is_better": False, "major_cycles": ctl.major_done,
            "clean_iterations": ctl.total_iter_done,
            "ms_per_major_cycle": t_gpu * 1e3 / max(1, ctl.major_done),
            "stop": ctl.stopdescription,
            "same_decisions_as_oracle": ctl.get_state() == octl.get_state(),
            "rel_err_vs_oracle": {"model": rel(model, ref["model"]),
                                  "residual": rel(resid, ref["residual"])},
            "cpu_baseline": {"value": t_cpu * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                             "sample": "the same loop, oracle restatement (C kernels, numpy "
                                       "FFTs), one run"},
            "speedup_vs_cpu": t_cpu / t_gpu,
            "workload": "64 ant, 50 t x 2016 bl x 1 ch x 2 pol (100800 vis), 512^2, 2 arcsec, "
                        "support 7, os 100, Hogbom niter 1000, nmajor 5, cyclefactor 1.5"}


def bench_mosaic(args, dev):
    """mosaic_grid_jit (FP64, av_mosaic_grid) on 64 antennas x 64 time steps x
    8 channels (1.0-1.5 GHz) x 2 pol = 1.03M samples into a 1024^2 grid of
    2 arcsec cells, with Airy-disk convolution functions of 12 m and 25 m
    dishes built by the helpers (oversampling 4, cut 0.025, a field 30 cells
    off the phase centre), against the oracle's C restatement on 4 of the 64
    time steps."""
    import torch

    import oracle as O
    from astroviper_b200 import _kernels as K
    from astroviper_b200 import synthetic as S
    from astroviper_b200.core.imaging import make_gridding_convolution_function as G
    from astroviper_b200.core.imaging.imaging_utils import make_pb_symmetric as PB
    nt, nchan, npol, n = 64, 8, 2, 1024
    uvw, rng = S.array_uvw(64, nt, seed=20260122)
    nb = uvw.shape[1]
    freq = np.linspace(1.0e9, 1.5e9, nchan)
    cell = np.array([-2.0, 2.0]) * np.pi / 180 / 3600
    shape = (nt, nb, nchan, npol)
    vis = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    wt = rng.uniform(0.5, 2.0, size=shape)
    ant_type = np.arange(64) % 2
    bant = np.array([[i, j] for i in range(64) for j in range(i + 1, 64)])
    cfb, pairs = G.create_cf_baseline_map(ant_type, bant, 2)
    cfc, pb_freq = G.create_cf_chan_map(freq, 0.05)
    os_, ms = np.array([4, 4]), np.array([11, 11])
    gcf = {"list_dish_diameters": np.array([12.0, 25.0]),
           "list_blockage_diameters": np.array([0.75, 0.0]), "oversampling": os_,
           "max_support": ms, "support_cut_level": 0.025, "resize_conv_size": (ms + 1) * os_,
           "phase_direction": np.array([0.0, -0.5])}
    grid_p = {"image_size": np.array([n, n]), "image_size_padded": np.array([n, n]),
              "cell_size": cell}
    gcf["ipower"] = 1
    bp = G.make_baseline_patterns(pb_freq, np.array([0]), pairs, PB.airy_disk_rorder, gcf,
                                  grid_p)
    gcf["ipower"] = 2
    bp2 = G.make_baseline_patterns(pb_freq, np.array([0]), pairs, PB.airy_disk_rorder, gcf,
                                   grid_p)
    rk, _rkc, sup = G.resize_and_calc_support(G.conv_kernels(bp), G.conv_kernels(bp2), gcf,
                                              grid_p)
    pg = G.make_phase_gradient(np.array([[30 * abs(cell[0]), -0.5]]), gcf, grid_p)
    cf = K.cf_phase_product(torch.as_tensor(rk, device=dev), torch.as_tensor(pg[0], device=dev))
    vis_d = torch.as_tensor(vis, device=dev)
    wt_d = torch.as_tensor(wt, device=dev)
    uvw_d = torch.as_tensor(uvw, device=dev)
    cm, pm, cfp = np.arange(nchan), np.arange(npol), np.zeros(npol, dtype=int)
    grid = torch.zeros((nchan, npol, n, n), dtype=torch.complex128, device=dev)
    sw = torch.zeros((nchan, npol), dtype=torch.float64, device=dev)

    def run():
        K.mosaic_grid(grid, sw, False, vis_d, wt_d, uvw_d, freq, cm, pm, cfb, cfc, cfp, cf, sup,
                      (n, n), cell, os_)

    for _ in range(3):
        run()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    reps = 10
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(reps):
        run()
    ev[1].record()
    torch.cuda.synchronize()
    ms_gpu = ev[0].elapsed_time(ev[1]) / reps
    n_vis = nt * nb * nchan
    # accuracy and the CPU baseline on a sample of the time steps
    ts = 4
    g1 = torch.zeros_like(grid)
    s1 = torch.zeros_like(sw)
    K.mosaic_grid(g1, s1, False, vis_d[:ts], wt_d[:ts], uvw_d[:ts], freq, cm, pm, cfb, cfc, cfp,
                  cf, sup, (n, n), cell, os_)
    go = np.zeros((nchan, npol, n, n), dtype=np.complex128)
    so = np.zeros((nchan, npol))
    t0 = time.perf_counter()
    O.mosaic_grid(go, so, False, vis[:ts], uvw[:ts], freq, cm, pm, cfb, cfc, cfp, wt[:ts],
                  cf.cpu().numpy(), sup, (n, n), cell, os_)
    t_cpu = time.perf_counter() - t0
    cpu_mvis = ts * nb * nchan / t_cpu / 1e6
    gpu_mvis = n_vis / (ms_gpu / 1e3) / 1e6
    return {"value": gpu_mvis, "unit": "Mvis/s", "ms_per_call": ms_gpu,
            "supports": sorted(set(int(x) for x in np.asarray(sup).ravel())),
            "n_functions": int(np.prod(np.asarray(sup).shape[:3])),
            "rel_err_vs_oracle": {"grid": rel(g1.cpu().numpy(), go),
                                  "sum_weight": rel(s1.cpu().numpy(), so),
                                  "sample": f"{ts} of {nt} time steps"},
            "cpu_baseline": {"value": cpu_mvis, "unit": "Mvis/s", "cores": 1, "kind": "port",
                             "sample": f"{ts} of {nt} time steps, the oracle's C restatement"},
            "speedup_vs_cpu": gpu_mvis / cpu_mvis,
            "workload": "64 ant, 64 t x 2016 bl x 8 ch x 2 pol (1.03M vis), 1024^2 cube, "
                        "2 arcsec, Airy functions 12 m / 25 m, oversampling 4"}


def bench_e2e(W, vis_dev, iw_dev, G):
    """Same step through the numpy drop-in API with host buffers in pinned
    memory: standard_grid_numpy_wrap_input_checked + dgrid_numba, host->device
    copies of the inputs and device->host copies of the grid and model
    visibilities inside the timed region."""
    import torch
    from astroviper_b200.core.imaging.imaging_utils import standard_degrid as SD
    from astroviper_b200.core.imaging.imaging_utils import standard_grid as SG

    def pinned_like(t):
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t)
        return h.numpy()

    vis_h = pinned_like(vis_dev)
    iw_h = pinned_like(iw_dev)
    uvw = W["uvw"]
    freq = W["freq"]
    nt, nb, nchan, npol = vis_h.shape
    nx, ny = int(W["image_size"][0]), int(W["image_size"][1])
    cgk = G.cgk.cpu().numpy()
    values_h = pinned_like(torch.zeros(vis_dev.shape, dtype=torch.complex64))
    flag_h = pinned_like(torch.zeros(vis_dev.shape, dtype=torch.bool))
    scale = np.array([-W["pixelincr"][0] * nx, -W["pixelincr"][1] * ny, 0.0])
    offset = np.array([nx / 2, ny / 2, 0.0])
    chanmap = (np.arange(nchan) / nchan * 1).astype(int)
    polmap = np.round(np.arange(npol) % npol).astype(int)

    # dgrid_numba adds the model to the caller's values, as the reference
    # does: the array is zeroed once here and accumulates over the steps
    # (clearing 1 GB of host memory is the caller's business, not the API's)
    def one():
        grid, sw = SG.standard_grid_numpy_wrap_input_checked(
            vis_h, np.array([]), np.array([]), uvw, iw_h, freq, cgk, W["image_size"],
            W["pixelincr"], 100, 7, True, False, "continuum")
        SD.dgrid_numba(uvw, np.zeros((nt, nb)), values_h, flag_h, scale, offset, grid, freq,
                       299792458.0, 7, 100, cgk, chanmap, polmap)
        return grid

    one()
    torch.cuda.synchronize()
    n = 2
    t0 = time.perf_counter()
    for _ in range(n):
        one()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / n
    gbytes = 1 * npol * nx * ny * 16
    h2d = vis_h.nbytes + iw_h.nbytes + uvw.nbytes + gbytes + values_h.nbytes + flag_h.nbytes
    d2h = gbytes + npol * 8 + values_h.nbytes
    return {"value": nt * nb * nchan / dt / 1e6, "unit": "Mvis/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": dt * 1e3,
            "api": "standard_grid_numpy_wrap_input_checked + dgrid_numba (numpy, pinned)"}


if __name__ == "__main__":
    main()
