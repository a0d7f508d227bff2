"""The C ABI: libav200.so loads and exports every entry point declared in
include/av200.h with the argument count the Python binding uses (no compute
calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "av200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|int64_t|size_t|const char \*|unsigned long long)\s*\*?\s*(av_\w+)"
                         r"\s*\(([^)]*)\)\s*;", src):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def test_header_declares_the_entry_points():
    d = declared()
    for name in ("av_grid_plain", "av_grid_tiled", "av_grid_tiled_plan", "av_grid_tiled_execute",
                 "av_degrid_plain", "av_degrid_tiled", "av_grid_to_image", "av_fft_shifted",
                 "av_weight_density", "av_briggs_factors", "av_briggs_apply", "av_hogbom_run",
                 "av_maximg", "av_pswf_table", "av_last_error"):
        assert name in d, name


def test_library_exports_every_declared_symbol():
    from astroviper_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libav200.so not built")
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared():
        assert hasattr(L, name), f"{name} declared in av200.h but not exported"


def test_binding_signatures_match_header():
    from astroviper_b200 import _lib
    d = declared()
    for name, (_res, args) in _lib.SIGNATURES.items():
        assert name in d, f"binding for undeclared {name}"
        assert len(args) == d[name], f"{name}: {len(args)} args bound, {d[name]} declared"
    for name in d:
        assert name in _lib.SIGNATURES, f"{name} has no Python binding"


def test_library_loads_and_reports_version_without_gpu():
    from astroviper_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libav200.so not built")
    L = _lib.lib()
    assert L.av_version() >= 100
    assert isinstance(L.av_last_error(), bytes)
