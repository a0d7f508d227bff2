"""The autotuner's choice and JSON cache, with a fake timer (no GPU): the
knob is set through the C ABI, which needs no device."""
import json
import os

import pytest

from astroviper_b200 import _lib


def _lib_or_skip():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libav200.so not built")
    return _lib.lib()


def test_tune_knobs_set_get_and_reject():
    L = _lib_or_skip()
    g = L.av_tune_get(_lib.AV_TUNE_GRID_CHUNKS_PER_SM)
    assert g >= 1 and L.av_tune_get(_lib.AV_TUNE_DEGRID_CHUNKS_PER_SM) >= 1
    assert L.av_tune_get(99) == -1
    assert L.av_tune_set(99, 4) == _lib.AV_ERR_ARG
    assert L.av_tune_set(_lib.AV_TUNE_GRID_CHUNKS_PER_SM, 0) == _lib.AV_ERR_ARG
    assert L.av_tune_set(_lib.AV_TUNE_GRID_CHUNKS_PER_SM, 5000) == _lib.AV_ERR_ARG
    assert L.av_tune_set(_lib.AV_TUNE_GRID_CHUNKS_PER_SM, 24) == _lib.AV_OK
    assert L.av_tune_get(_lib.AV_TUNE_GRID_CHUNKS_PER_SM) == 24
    assert L.av_tune_get(_lib.AV_TUNE_GRID_LANES) == _lib.AV_GRID_LANES_AUTO
    assert L.av_tune_set(_lib.AV_TUNE_GRID_LANES, 4) == _lib.AV_ERR_ARG
    assert L.av_tune_set(_lib.AV_TUNE_GRID_LANES, _lib.AV_GRID_LANES_ROWS) == _lib.AV_OK
    assert L.av_tune_get(_lib.AV_TUNE_GRID_LANES) == _lib.AV_GRID_LANES_ROWS
    assert L.av_tune_set(_lib.AV_TUNE_GRID_LANES, _lib.AV_GRID_LANES_AUTO) == _lib.AV_OK
    assert L.av_tune_get(_lib.AV_TUNE_DEGRID_LANES) == _lib.AV_DEGRID_LANES_AUTO
    assert L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, 5) == _lib.AV_ERR_ARG
    assert L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, _lib.AV_DEGRID_LANES_TC05) == _lib.AV_OK
    assert L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, _lib.AV_DEGRID_LANES_FP32) == _lib.AV_OK
    assert L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, _lib.AV_DEGRID_LANES_AUTO) == _lib.AV_OK
    assert L.av_tune_set(_lib.AV_TUNE_GRID_CHUNKS_PER_SM, g) == _lib.AV_OK
    # the Hogbom barrier timeout (microseconds): 0 is allowed, the default is 2 s
    knob = _lib.AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US
    assert L.av_tune_get(knob) == _lib.AV_HOGBOM_BARRIER_TIMEOUT_US_DEFAULT
    assert L.av_tune_set(knob, -1) == _lib.AV_ERR_ARG
    assert L.av_tune_set(knob, 600000001) == _lib.AV_ERR_ARG
    assert "AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US" in _lib.last_error()
    assert L.av_tune_set(knob, 0) == _lib.AV_OK
    assert L.av_tune_get(knob) == 0
    assert L.av_tune_set(knob, _lib.AV_HOGBOM_BARRIER_TIMEOUT_US_DEFAULT) == _lib.AV_OK


def test_autotuner_picks_fastest_and_caches(tmp_path):
    """The tuner times every (lanes, chunks per SM) pair, keeps the fastest,
    sets both knobs and caches the pair; a new process takes it from the
    cache without timing."""
    L = _lib_or_skip()
    from astroviper_b200 import autotune
    kl, kc = _lib.AV_TUNE_GRID_LANES, _lib.AV_TUNE_GRID_CHUNKS_PER_SM
    before = (L.av_tune_get(kl), L.av_tune_get(kc))
    path = str(tmp_path / "tune.json")
    cost = {4: 3.0, 8: 2.0, 16: 1.5, 32: 1.2, 64: 1.4}
    lane_cost = {_lib.AV_GRID_LANES_MMA: 1.0, _lib.AV_GRID_LANES_ROWS: 1.3}
    calls = []

    def run():
        calls.append((L.av_tune_get(kl), L.av_tune_get(kc)))

    def timer(fn):
        fn()
        return cost[L.av_tune_get(kc)] * lane_cost[L.av_tune_get(kl)]

    k = autotune.key("grid", 7, 1024, 1024, 2, 128, gpu="testgpu")
    assert k == "v2|testgpu|grid|S7|1024x1024|p2|c128"
    autotune._applied.pop(k, None)
    v = autotune.ensure(k, run, path=path, timer=timer)
    assert v == {"lanes": _lib.AV_GRID_LANES_MMA, "chunks_per_sm": 32}
    assert (L.av_tune_get(kl), L.av_tune_get(kc)) == (_lib.AV_GRID_LANES_MMA, 32)
    data = json.load(open(path))
    assert data[k]["value"] == v and len(data[k]["ms"]) == 10
    assert data[k]["ms"][f"{_lib.AV_GRID_LANES_ROWS}/4"] == 3.9
    # a new process (empty memory) takes the cached pair without timing
    autotune._applied.pop(k, None)
    L.av_tune_set(kl, before[0])
    L.av_tune_set(kc, before[1])
    n = len(calls)
    assert autotune.ensure(k, run, path=path, timer=timer) == v
    assert len(calls) == n and L.av_tune_get(kc) == 32
    # an entry of the earlier single-knob format is timed again
    data[k]["value"] = 16
    json.dump(data, open(path, "w"))
    autotune._applied.pop(k, None)
    assert autotune.ensure(k, run, path=path, timer=timer) == v and len(calls) > n
    L.av_tune_set(kl, before[0])
    L.av_tune_set(kc, before[1])
    autotune._applied.pop(k, None)


def test_support_choice_by_aliasing():
    """choose_support takes the smallest candidate whose aliasing at the edge
    of the inner 80 % of the field meets the tolerance, else the least
    aliasing one; with the reference's kernel, supports 8 and 9 alias more
    than 6 and 7 there (the oracle's tables stand in for the device's)."""
    import oracle as O
    from astroviper_b200 import autotune
    t = {s: O.create_prolate_spheroidal_kernel_1D(100, s) for s in (5, 7, 9)}
    s, r = autotune.choose_support((7, 9), 100, tables=t)
    assert s == 7 and r[7] < 1e-2 < r[9]
    assert autotune.choose_support((5, 7, 9), 100, alias_tol=0.5, tables=t)[0] == 5
    assert autotune.choose_support((5, 7, 9), 100, alias_tol=1e-2, tables=t)[0] == 7
    # none meets a tight tolerance: the least aliasing one
    r5 = autotune.alias_ratio(5, 100, table=t[5])
    least = 9 if r[9] < r5 else 5
    assert autotune.choose_support((5, 9), 100, alias_tol=1e-6, tables=t)[0] == least
    # at the very edge any kernel's nearest alias mirrors its response
    assert autotune.alias_ratio(7, 100, field=1.0, table=t[7]) > 0.5


def test_autotuner_key_and_corrupt_cache(tmp_path):
    from astroviper_b200 import autotune
    with pytest.raises(ValueError):
        autotune.key("fft", 7, 8, 8, 1, 1, gpu="x")
    p = tmp_path / "bad.json"
    p.write_text("{not json")
    assert autotune.load(str(p)) == {}
