"""Launch autotuner with a JSON cache.

The tiled gridder and degridder hand out work in record chunks; how many
chunks per SM balances the CTAs' finishing times against per-chunk overhead
(tile flushes, tile searches), and the best value depends on the GPU, the
support, the grid size and the number of polarisations and planes.  The tuner
times one launch per candidate with CUDA events on the current stream, keeps
the fastest, sets it with av_tune_set and stores it in a JSON cache keyed by
(GPU, kernel, support, grid size, polarisations, planes), so later processes
on the same GPU model skip the timing.

The cache file is $AV200_TUNE_CACHE, else ~/.cache/astroviper_b200/tune.json.
"""
import json
import os
import threading

from ._lib import AV_TUNE_DEGRID_CHUNKS_PER_SM, AV_TUNE_GRID_CHUNKS_PER_SM, check, lib

KNOBS = {"grid": AV_TUNE_GRID_CHUNKS_PER_SM, "degrid": AV_TUNE_DEGRID_CHUNKS_PER_SM}
CANDIDATES = (4, 8, 16, 32, 64)
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
    if kernel not in KNOBS:
        raise ValueError(f"unknown kernel {kernel!r}")
    gpu = gpu_name() if gpu is None else gpu
    return f"{gpu}|{kernel}|S{int(support)}|{int(n_u)}x{int(n_v)}|p{int(npol)}|c{int(planes)}"


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


def apply(k, value):
    """Set the knob of key k's kernel to value."""
    kernel = k.split("|")[1]
    check(lib().av_tune_set(KNOBS[kernel], int(value)), "av_tune_set")
    _applied[k] = int(value)


def measure(run, candidates=CANDIDATES, reps=3, knob=AV_TUNE_GRID_CHUNKS_PER_SM, timer=None):
    """Median time (ms) of run() for each candidate value of knob; returns
    {value: ms}.  run() enqueues one launch on the current stream.  timer, if
    given, replaces the CUDA-event timing (run -> ms) for tests."""
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
    old = lib().av_tune_get(knob)
    out = {}
    try:
        for v in candidates:
            check(lib().av_tune_set(knob, int(v)), "av_tune_set")
            run()  # warm-up at this setting
            ts = sorted(timer(run) for _ in range(reps))
            out[int(v)] = ts[len(ts) // 2]
    finally:
        check(lib().av_tune_set(knob, int(old)), "av_tune_set")
    return out


def ensure(k, run, candidates=CANDIDATES, reps=3, path=None, timer=None):
    """Make key k's tuned value current: from this process's memory, else the
    JSON cache, else by timing run() over the candidates (and caching the
    result).  Returns the value."""
    with _lock:
        if k in _applied:
            apply(k, _applied[k])
            return _applied[k]
        entries = load(path)
        if k in entries and "value" in entries[k]:
            apply(k, entries[k]["value"])
            return _applied[k]
        kernel = k.split("|")[1]
        times = measure(run, candidates, reps, KNOBS[kernel], timer)
        best = min(times, key=lambda v: (times[v], v))
        entries = load(path)
        entries[k] = {"value": best, "ms": {str(v): round(t, 4) for v, t in times.items()}}
        save(entries, path)
        apply(k, best)
        return best
