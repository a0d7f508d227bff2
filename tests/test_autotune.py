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
    assert L.av_tune_set(_lib.AV_TUNE_DEGRID_LANES, 4) == _lib.AV_ERR_ARG
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
    L = _lib_or_skip()
    from astroviper_b200 import autotune
    knob = _lib.AV_TUNE_GRID_CHUNKS_PER_SM
    before = L.av_tune_get(knob)
    path = str(tmp_path / "tune.json")
    cost = {4: 3.0, 8: 2.0, 16: 1.5, 32: 1.2, 64: 1.4}
    calls = []

    def run():
        calls.append(L.av_tune_get(knob))

    def timer(fn):
        fn()
        return cost[L.av_tune_get(knob)]

    k = autotune.key("grid", 7, 1024, 1024, 2, 128, gpu="testgpu")
    assert k == "testgpu|grid|S7|1024x1024|p2|c128"
    autotune._applied.pop(k, None)
    v = autotune.ensure(k, run, path=path, timer=timer)
    assert v == 32 and L.av_tune_get(knob) == 32
    data = json.load(open(path))
    assert data[k]["value"] == 32 and set(data[k]["ms"]) == {"4", "8", "16", "32", "64"}
    # a new process (empty memory) takes the cached value without timing
    autotune._applied.pop(k, None)
    L.av_tune_set(knob, before)
    n = len(calls)
    assert autotune.ensure(k, run, path=path, timer=timer) == 32
    assert len(calls) == n and L.av_tune_get(knob) == 32
    L.av_tune_set(knob, before)
    autotune._applied.pop(k, None)


def test_autotuner_key_and_corrupt_cache(tmp_path):
    from astroviper_b200 import autotune
    with pytest.raises(ValueError):
        autotune.key("fft", 7, 8, 8, 1, 1, gpu="x")
    p = tmp_path / "bad.json"
    p.write_text("{not json")
    assert autotune.load(str(p)) == {}
