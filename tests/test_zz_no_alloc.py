"""ecl_cc_noalloc: the allocation-free CC entry point, for callers that cannot
allocate device memory.  Called through the C ABI and compared with ecl_cc
(the regular entry point) on the same device graphs, twice in a row so the
second call runs on scratch that still holds the first call's contents.

This file is collected last on purpose; it passes both alone in a fresh
process and after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from conftest import overlapping_rows, undirected

pytestmark = pytest.mark.gpu


def _entry(ecl):
    f = ecl.lib.ecl_cc_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def test_cc_noalloc_matches_ecl_cc_on_two_calls(ecl):
    import torch

    f = _entry(ecl)
    graphs = [
        ecl.gen_rmat(15, 16, seed=2),
        ecl.gen_rmat(12, 8, seed=9, symmetrise=False),
        ecl.gen_grid(200, 300, 0.3, seed=3),
        # hubs above the chunk threshold exercise the chunk counters
        undirected(9000, [(8999, i) for i in range(8999)] + [(i, i + 1) for i in range(0, 400, 2)]),
    ]
    stream = torch.cuda.current_stream().cuda_stream
    for g in graphs:
        dg = g.to_device()
        expected = ecl.cc(dg).cpu().numpy()  # the regular entry point
        for _ in range(2):
            out = torch.full((g.nodes,), -1, dtype=torch.int32, device="cuda")
            st = f(g.nodes, g.edges, dg.nindex.data_ptr(), dg.nlist.data_ptr(), out.data_ptr(), stream)
            assert st == ecl.OK
            assert np.array_equal(out.cpu().numpy(), expected)


def test_cc_noalloc_rejects_graphs_beyond_its_limit(ecl):
    import torch

    f = _entry(ecl)
    limit = 1 << 27
    small = torch.zeros(2, dtype=torch.int32, device="cuda")
    # rejected on the host before any device work
    st = f(1, limit + 1, small.data_ptr(), small.data_ptr(), small.data_ptr(), None)
    assert st == ecl.ERR_UNSUPPORTED
    assert b"ECL_CC_NOALLOC_MAX_EDGES" in ecl.lib.ecl_last_error()


def test_cc_noalloc_overlapping_rows_stay_inside_the_array(ecl, orc):
    """A CSR whose rows overlap asks for more long-row chunk records than the
    fixed array holds for its edge count: the call reports ECL_ERR_BAD_GRAPH
    and writes nothing past its records, and the next call is still exact."""
    import torch

    f = _entry(ecl)
    stream = torch.cuda.current_stream().cuda_stream
    g = overlapping_rows()
    dg = g.to_device()
    out = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    assert f(g.nodes, g.edges, dg.nindex.data_ptr(), dg.nlist.data_ptr(), out.data_ptr(), stream) == ecl.ERR_BAD_GRAPH
    ok = ecl.gen_rmat(13, 16, seed=2)
    dok = ok.to_device()
    out = torch.empty(ok.nodes, dtype=torch.int32, device="cuda")
    assert f(ok.nodes, ok.edges, dok.nindex.data_ptr(), dok.nlist.data_ptr(), out.data_ptr(), stream) == ecl.OK
    assert np.array_equal(out.cpu().numpy(), orc.cc(ok))
