"""C-ABI library: loads, exports every declared symbol, sane metadata (CPU only)."""
import ctypes
import os
import re

from conftest import ROOT

HEADERS = ["ecl_b200.h", "ecl_batch.h", "ecl_server.h"]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(ecl_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_symbols_exported(ecl):
    lib = ctypes.CDLL(ecl.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(ecl.EXPORTED) <= set(declared_functions())


def test_abi_version_and_status_strings(ecl):
    assert ecl.lib.ecl_abi_version() == 2
    for s in range(9):
        assert ecl.lib.ecl_status_string(s)
    assert ecl.lib.ecl_status_string(999) == b"unknown status"


def test_workspace_bytes(ecl):
    for code in range(6):
        assert ecl.workspace_bytes(code, 1000, 8000) >= 256
    assert ecl.workspace_bytes(ecl.CC, 0, 10) == 0
    assert ecl.workspace_bytes(99, 10, 10) == 0


def test_solver_without_device_reports_status(ecl):
    """With no CUDA device the solvers return a status code, never crash."""
    import numpy as np

    from conftest import has_gpu

    if has_gpu():
        return
    g = ecl.Graph(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    out = np.empty(2, np.int32)
    v = g.view()
    o = ecl.Opts()
    st = ecl.lib.ecl_cc(ctypes.byref(v), out.ctypes.data, ctypes.byref(o))
    assert st == ecl.ERR_NO_DEVICE


def test_bad_arguments_rejected_before_device(ecl):
    import numpy as np

    o = ecl.Opts()
    assert ecl.lib.ecl_cc(None, None, ctypes.byref(o)) != ecl.OK
    g = ecl.Graph(np.array([0], np.int32), np.array([], np.int32))  # nodes = 0
    v = g.view()
    out = np.empty(1, np.int32)
    assert ecl.lib.ecl_cc(ctypes.byref(v), out.ctypes.data, ctypes.byref(o)) == ecl.ERR_BAD_GRAPH


def test_tune_knobs_round_trip_and_range_checks(ecl):
    """ecl_set_tune keeps valid knobs process-wide and rejects out-of-range
    ones without changing anything (no device needed)."""
    old = ecl.set_tune(gc_core_ranks=1024, blocks_per_sm=4)
    try:
        t = ecl.get_tune()
        assert (t.gc_core_ranks, t.blocks_per_sm) == (1024, 4)
        bad = ecl.Tune()
        bad.gc_core_ranks = 1 << 20
        assert ecl.lib.ecl_set_tune(ctypes.byref(bad)) == ecl.ERR_INVALID_ARG
        assert ecl.get_tune().gc_core_ranks == 1024
    finally:
        ecl.set_tune(old)
    assert ecl.get_tune().as_dict() == old.as_dict()
