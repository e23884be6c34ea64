"""The C-ABI library loads, exports every entry point of include/tsc_gpu.h and
reports errors as status codes (no compute: no GPU here)."""
import ctypes
import os
import re

import pytest

from tsc_tri_t1t2j1j2_b200 import _lib
from tsc_tri_t1t2j1j2_b200 import build as tscbuild

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "tsc_gpu.h")


def declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b(tsc_[a-z_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    if not os.path.exists(_lib.LIB_PATH):
        tscbuild.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == names


def test_errors_are_status_codes_not_aborts():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present; this checks the no-device error path")
    L = _lib.load()
    h = ctypes.c_void_p()
    cfg = _lib.ModelConfig(4, 4, 1.0, 0.0, 0.4, 0.0, 12, 0)
    rc = L.tsc_create(ctypes.byref(h), ctypes.byref(cfg))
    assert rc == -3
    assert b"cuda" in L.tsc_last_error(h).lower()
    assert L.tsc_superblock_dim(h) == -4
    # entry points that need an engine report it as a status, never crash
    d = (ctypes.c_double * 64)()
    ii = (ctypes.c_int * 64)()
    ll = ctypes.c_longlong()
    assert L.tsc_measure_correlation(h, 1, 1, d, 16) == -4
    assert L.tsc_measure_pair_correlation(h, 1, 16, 0, 1, ii, d, 8) == -4
    assert L.tsc_set_lanczos_graph(h, 1) == -4
    assert L.tsc_lanczos_graph_stats(h, ctypes.byref(ll), ctypes.byref(ll), None, 0) == -4
    assert L.tsc_set_split_view_sharing(h, 1) == -4
    assert L.tsc_set_split_finish_tolerance(h, 1.0) == -4
    assert L.tsc_set_spill_directory(h, b"/tmp", 0) == -4
    assert L.tsc_set_split_renormalization(h, 1) == -4
    assert L.tsc_density_matrix(h, 0, d, 1, None, None, None, None) == -4
    assert L.tsc_measure_correlation(None, 1, 1, d, 16) == -1
    assert L.tsc_destroy(h) == 0
    assert L.tsc_create(None, ctypes.byref(cfg)) == -1
    assert L.tsc_hpsi(None, None, None) == -1


def test_context_raises_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from tsc_tri_t1t2j1j2_b200 import Context
    with pytest.raises(_lib.TscError):
        Context(4, 4)
