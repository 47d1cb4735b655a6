"""Batched engine on the B200: every graph's result equals its solo solve
(and the oracle), across several super-batches, on CUDA-graph replays."""
import numpy as np
import pytest

from conftest import undirected

pytestmark = pytest.mark.gpu


def test_batch_matches_solo_and_oracle(ecl, orc):
    b = ecl.Batch()
    b.add_mix(40, n_min=50, n_max=3000, seed=5, weight_max=1 << 16)
    hub = undirected(700, [(699, i) for i in range(699)] + [(i, i + 1) for i in range(0, 100, 2)])
    hub.eweight = np.arange(1, hub.edges + 1, dtype=np.int32) % 97 + 1
    b.add(hub)
    codes = ecl.BATCH_CC | ecl.BATCH_MIS | ecl.BATCH_GC | ecl.BATCH_MST | ecl.BATCH_SCC
    b.build(codes, max_entries=30000)  # force several super-batches
    assert b.superbatches > 2
    ms0, replay0 = b.run()
    ms1, replay1 = b.run()  # CUDA-graph replay
    assert replay1, ecl.lib.ecl_last_error()
    for i in range(b.graphs):
        g = b.graph(i)
        assert np.array_equal(b.result(i, ecl.BATCH_CC), orc.cc(g)), i
        assert np.array_equal(b.result(i, ecl.BATCH_MIS), orc.mis(g)), i
        assert np.array_equal(b.result(i, ecl.BATCH_GC), orc.gc(g)), i
        assert np.array_equal(b.result(i, ecl.BATCH_SCC), orc.scc(g)), i
        inm, tot = b.result(i, ecl.BATCH_MST)
        einm, etot = orc.mst(g)
        assert tot == etot and np.array_equal(inm, einm), i
        if i % 10 == 0:  # and the solo library call agrees
            assert np.array_equal(ecl.mis(g), b.result(i, ecl.BATCH_MIS))


def test_batch_tune_keeps_results(ecl, orc):
    b = ecl.Batch()
    b.add_mix(12, n_min=500, n_max=5000, seed=9, weight_max=1 << 16)
    b.build(ecl.BATCH_CC | ecl.BATCH_MIS | ecl.BATCH_MST)
    t = b.tune(trials=1)
    assert b.tune_points > 6
    assert t.blocks_per_sm in (64, 32, 16, 8) and t.mst_light_factor in (0.75, 1.5, 3.0, 0.4)
    assert t.row_lane_max in (8, 16, 32) and t.row_chunk in (128, 256, 512, 2048)
    b.run()
    for i in range(b.graphs):
        g = b.graph(i)
        assert np.array_equal(b.result(i, ecl.BATCH_CC), orc.cc(g))
        inm, tot = b.result(i, ecl.BATCH_MST)
        assert tot == orc.mst(g)[1]
