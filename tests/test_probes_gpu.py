"""The measurement probes behind the bench line's rooflines: the INT32
min-plus rate (APSP), the dependency-hop latency (GC's chain bound) and the
streaming-gather rate (the CSR scans' bound).  Each returns a plausible
positive figure on the device and rejects bad arguments with
ECL_ERR_INVALID_ARG before any launch."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_minplus_peak_is_positive(ecl):
    for variant in (0, 1):
        rate = ecl.minplus_peak(variant)
        assert 1e12 < rate < 1e15, (variant, rate)  # integer ops/s


def test_hop_latency_orders_shared_below_l2(ecl):
    l2 = ecl.hop_latency(0)
    smem = ecl.hop_latency(2)
    assert 10.0 < smem < l2 < 100000.0, (smem, l2)  # ns per hop


def test_gather_peak_on_graph_indices(ecl):
    import torch

    g = ecl.gen_rmat(16, 16, seed=2).to_device()
    ro = ecl.gather_peak(g.nlist, g.nodes, 0)
    at = ecl.gather_peak(g.nlist, g.nodes, 1)
    assert ro > 1e9 and at > 1e9, (ro, at)  # entries/s
    idx = torch.zeros(1024, dtype=torch.int32, device="cuda")
    assert ecl.gather_peak(idx, 1, 0) > 0


def test_probes_reject_bad_arguments(ecl):
    v = C.c_double(0.0)
    assert ecl.lib.ecl_minplus_peak(7, C.byref(v)) == ecl.ERR_INVALID_ARG
    assert ecl.lib.ecl_hop_latency(9, C.byref(v)) == ecl.ERR_INVALID_ARG
    assert ecl.lib.ecl_gather_peak(None, 16, 16, 0, C.byref(v)) == ecl.ERR_INVALID_ARG
    idx = np.zeros(4, np.int32)
    assert ecl.lib.ecl_gather_peak(idx.ctypes.data, 0, 16, 0, C.byref(v)) == ecl.ERR_INVALID_ARG
    assert ecl.lib.ecl_gather_peak(idx.ctypes.data, 4, 16, 2, C.byref(v)) == ecl.ERR_INVALID_ARG
