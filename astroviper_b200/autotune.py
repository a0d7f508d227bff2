"""Launch autotuner with a JSON cache, and the accuracy-driven support choice.

The tiled gridder and degridder have two launch knobs each: how a run of
samples is summed (the lane mapping: FP64 tensor-core tiles or a footprint row
per lane for the gridder, TF32 tensor-core tiles or FP32 FMA for the
degridder's fast path) and how many record chunks per SM the persistent CTAs
hand out (balancing the CTAs' finishing times against per-chunk overhead).
The best pair depends on the GPU, the support, the grid size and the numbers
of polarisations and planes.  The tuner times one launch per pair with CUDA
events on the current stream, keeps the fastest, sets both knobs with
av_tune_set and stores the pair in a JSON cache keyed by (GPU, kernel,
support, grid size, polarisations, planes), so later processes on the same GPU
model skip the timing.  Every pair computes the same result to within
summation order (the lane mappings' accuracies are stated in include/av200.h).

choose_support picks the kernel support itself, which does change the result,
so it is a separate, explicit call: the smallest candidate support whose
gridding kernel keeps the aliased response at the edge of the imaged field
below a tolerance (BatchedGridder(support="auto") uses it).

The cache file is $AV200_TUNE_CACHE, else ~/.cache/astroviper_b200/tune.json.
"""
import itertools
import json
import os
import threading

import numpy as np

from ._lib import (AV_DEGRID_LANES_FP32, AV_DEGRID_LANES_TF32, AV_GRID_LANES_MMA,
                   AV_GRID_LANES_ROWS, AV_TUNE_DEGRID_CHUNKS_PER_SM, AV_TUNE_DEGRID_LANES,
                   AV_TUNE_GRID_CHUNKS_PER_SM, AV_TUNE_GRID_LANES, check, lib)

CANDIDATES = (4, 8, 16, 32, 64)  # record chunks per SM
# kernel -> ((knob name, knob id, candidate values), ...), timed as a product
SPACES = {
    "grid": (("lanes", AV_TUNE_GRID_LANES, (AV_GRID_LANES_MMA, AV_GRID_LANES_ROWS)),
             ("chunks_per_sm", AV_TUNE_GRID_CHUNKS_PER_SM, CANDIDATES)),
    "degrid": (("lanes", AV_TUNE_DEGRID_LANES, (AV_DEGRID_LANES_TF32, AV_DEGRID_LANES_FP32)),
               ("chunks_per_sm", AV_TUNE_DEGRID_CHUNKS_PER_SM, CANDIDATES)),
}
CACHE_VERSION = "v2"
_lock = threading.Lock()
_applied = {}


def cache_path():
    p = os.environ.get("AV200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "astroviper_b200", "tune.json")


def gpu_name():
    import torch
    if not torch.cuda.is_available():
        return "cpu"
    return torch.cuda.get_device_name(torch.cuda.current_device())


def key(kernel, support, n_u, n_v, npol, planes, gpu=None):
    if kernel not in SPACES:
        raise ValueError(f"unknown kernel {kernel!r}")
    gpu = gpu_name() if gpu is None else gpu
    return (f"{CACHE_VERSION}|{gpu}|{kernel}|S{int(support)}|{int(n_u)}x{int(n_v)}"
            f"|p{int(npol)}|c{int(planes)}")


def _kernel_of(k):
    return k.split("|")[2]


def load(path=None):
    path = path or cache_path()
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save(entries, path=None):
    path = path or cache_path()
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = path + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(entries, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _label(setting):
    return "/".join(str(int(v)) for v in setting.values())


def apply(k, setting):
    """Set the knobs of key k's kernel to setting ({knob name: value})."""
    for name, knob, _cands in SPACES[_kernel_of(k)]:
        check(lib().av_tune_set(knob, int(setting[name])), "av_tune_set")
    _applied[k] = {n: int(v) for n, v in setting.items()}


def measure(run, space, reps=3, timer=None):
    """Median time (ms) of run() for every combination of the space's knob
    values; returns {label: (setting, ms)} with label "v1/v2/...".  run()
    enqueues one launch on the current stream.  timer, if given, replaces
    the CUDA-event timing (run -> ms) for tests.  The knobs are restored."""
    if timer is None:
        import torch

        def timer(fn):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s.record()
            fn()
            e.record()
            e.synchronize()
            return s.elapsed_time(e)
    old = {knob: lib().av_tune_get(knob) for _n, knob, _c in space}
    out = {}
    try:
        for values in itertools.product(*(c for _n, _k, c in space)):
            setting = {}
            for (name, knob, _c), v in zip(space, values):
                check(lib().av_tune_set(knob, int(v)), "av_tune_set")
                setting[name] = int(v)
            run()  # warm-up at this setting
            ts = sorted(timer(run) for _ in range(reps))
            out[_label(setting)] = (setting, ts[len(ts) // 2])
    finally:
        for knob, v in old.items():
            check(lib().av_tune_set(knob, int(v)), "av_tune_set")
    return out


def ensure(k, run, reps=3, path=None, timer=None):
    """Make key k's tuned knobs current: from this process's memory, else the
    JSON cache, else by timing run() over the kernel's knob space (and caching
    the result).  Returns the setting {knob name: value}."""
    with _lock:
        if k in _applied:
            apply(k, _applied[k])
            return _applied[k]
        entries = load(path)
        hit = entries.get(k, {}).get("value")
        if isinstance(hit, dict) and set(hit) == {n for n, _k, _c in SPACES[_kernel_of(k)]}:
            apply(k, hit)
            return _applied[k]
        times = measure(run, SPACES[_kernel_of(k)], reps, timer)
        best = min(times, key=lambda lab: (times[lab][1], lab))
        entries = load(path)
        entries[k] = {"value": times[best][0],
                      "ms": {lab: round(t, 4) for lab, (_s, t) in times.items()}}
        save(entries, path)
        apply(k, times[best][0])
        return _applied[k]


# ----------------------------------------------------------------------------
# support choice (changes the result: an explicit opt-in)
def alias_ratio(support, oversampling=100, field=0.8, n=2048, table=None):
    """Aliasing of the PSWF gridding kernel of this support (the reference's
    create_prolate_spheroidal_kernel_1D, gcf_prolate_spheroidal.py:87-99), in
    the image plane at the edge of the imaged field: with C(x) the response
    of the oversampled kernel at image coordinate x (in units of the grid's
    field of view, |x| <= 1/2 inside it), the ratio
    sqrt(sum over m != 0 of |C(x + m)|^2) / |C(x)| at x = field / 2, i.e. the
    power the aliases of the images' neighbours put there against the image's
    own response, the quantity grid correction cannot undo.  At the very edge
    (field = 1) the nearest alias mirrors the image's own response, so the
    ratio is about 1 for any kernel: the default looks at the inner 80 %.
    table: the kernel's 1-D half table when already at hand (else it is made
    on the device)."""
    if table is None:
        from .core.imaging.imaging_utils.gcf_prolate_spheroidal import \
            create_prolate_spheroidal_kernel_1D
        table = create_prolate_spheroidal_kernel_1D(oversampling, support)
    half = np.asarray(table, np.float64)
    # the kernel on a line of n cells sampled every 1 / os cell, taps at
    # |i| / os for |i| < len(half), centred on sample 0
    length = n * oversampling
    line = np.zeros(length)
    m = len(half) - 1
    line[:m + 1] = half
    line[-m:] = half[:0:-1]
    resp = np.abs(np.fft.fft(line))  # C at x = k / n (k in FFT order), period os
    k_edge = int(round(field / 2 * n))
    main = resp[k_edge]
    aliases = np.array([resp[(k_edge + j * n) % length] for j in range(1, oversampling)])
    return float(np.sqrt(np.sum(aliases ** 2)) / main)


def choose_support(candidates=(7, 9), oversampling=100, alias_tol=1e-2, field=0.8,
                   tables=None):
    """The smallest candidate support whose alias_ratio at the edge of the
    imaged field is at most alias_tol (the least-aliasing candidate when none
    is); returns (support, {support: ratio}).  tables: {support: 1-D half
    table} when already at hand.

    The reference's kernel is one spheroidal function (fixed coefficients)
    stretched over support // 2 cells either side, with a grid correction
    that does not depend on the support, so a wider support is not always
    the better one: 8 and 9 alias more than 6 and 7 beyond the inner half of
    the field (at field 0.8 and oversampling 100: 0.26 against 6.8e-3)."""
    tables = tables or {}
    ratios = {int(s): alias_ratio(int(s), oversampling, field, table=tables.get(int(s)))
              for s in sorted(candidates)}
    for s, r in ratios.items():
        if r <= alias_tol:
            return s, ratios
    return min(ratios, key=lambda s: (ratios[s], s)), ratios
