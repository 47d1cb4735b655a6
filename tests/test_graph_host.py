"""ECLgraph file format, host validation and seeded generators (CPU only)."""
import os
import struct

import numpy as np
import pytest

from conftest import undirected


def test_roundtrip_with_and_without_weights(ecl, tmp_path):
    g = undirected(5, [(0, 1), (1, 2), (3, 4)], weights=[7, 8, 9])
    p = str(tmp_path / "w.egr")
    g.write(p)
    raw = open(p, "rb").read()
    # header + nindex + nlist + eweight, little-endian int32 (ECLgraph.h:83-90)
    assert len(raw) == 4 * (2 + 6 + 6 + 6)
    assert struct.unpack("<2i", raw[:8]) == (5, 6)
    h = ecl.read_graph(p)
    assert np.array_equal(h.nindex, g.nindex) and np.array_equal(h.nlist, g.nlist)
    assert np.array_equal(h.eweight, g.eweight)
    g.eweight = None
    p2 = str(tmp_path / "nw.egr")
    g.write(p2)
    assert os.path.getsize(p2) == 4 * (2 + 6 + 6)
    assert ecl.read_graph(p2).eweight is None


def test_read_rejects_bad_files(ecl, tmp_path):
    p = str(tmp_path / "bad.egr")
    open(p, "wb").write(struct.pack("<2i", 0, 0))  # nodes < 1 (ECLgraph.h:57)
    with pytest.raises(ecl.EclError) as e:
        ecl.read_graph(p)
    assert e.value.status == ecl.ERR_BAD_GRAPH
    open(p, "wb").write(struct.pack("<2i3i", 2, 4, 0, 2, 4))  # truncated nlist
    with pytest.raises(ecl.EclError) as e:
        ecl.read_graph(p)
    assert e.value.status == ecl.ERR_IO
    open(p, "wb").write(struct.pack("<2i3i2i1i", 2, 2, 0, 1, 2, 1, 0, 5))  # partial weights
    with pytest.raises(ecl.EclError) as e:
        ecl.read_graph(p)
    assert e.value.status == ecl.ERR_IO
    with pytest.raises(ecl.EclError):
        ecl.read_graph(str(tmp_path / "missing.egr"))


def test_validate(ecl):
    g = undirected(4, [(0, 1), (1, 2)])
    assert g.validate(symmetric=True, no_self_loops=True)
    a = ecl.Graph(np.array([0, 1, 1], np.int32), np.array([1], np.int32))
    assert a.validate() and not a.validate(symmetric=True)
    s = ecl.Graph(np.array([0, 1], np.int32), np.array([0], np.int32))
    assert s.validate() and not s.validate(no_self_loops=True)
    o = ecl.Graph(np.array([0, 1], np.int32), np.array([3], np.int32))
    assert not o.validate()
    nm = ecl.Graph(np.array([0, 2, 1], np.int32), np.array([1, 0], np.int32))
    assert not nm.validate()
    # unsorted but symmetric lists use the multiset path
    u = ecl.Graph(np.array([0, 2, 3, 4], np.int32), np.array([2, 1, 0, 0], np.int32))
    assert u.validate(symmetric=True)


def test_grid_generator(ecl):
    g = ecl.gen_grid(16, 16, 0.0, seed=1)
    assert g.nodes == 256 and g.edges == 2 * 2 * 16 * 15
    assert g.validate(symmetric=True, no_self_loops=True)
    d = ecl.gen_grid(64, 64, 0.05, seed=1)
    full = 2 * 2 * 64 * 63
    assert 0.9 * full < d.edges < full
    assert d.validate(symmetric=True, no_self_loops=True)
    d2 = ecl.gen_grid(64, 64, 0.05, seed=1)
    assert np.array_equal(d.nlist, d2.nlist)


def test_rmat_generator_deterministic_and_clean(ecl):
    g = ecl.gen_rmat(10, 8, seed=2, weight_seed=3, weight_max=1 << 20)
    h = ecl.gen_rmat(10, 8, seed=2, weight_seed=3, weight_max=1 << 20)
    assert np.array_equal(g.nindex, h.nindex) and np.array_equal(g.nlist, h.nlist)
    assert np.array_equal(g.eweight, h.eweight)
    assert g.validate(symmetric=True, no_self_loops=True)
    for v in range(g.nodes):
        row = g.nlist[g.nindex[v]:g.nindex[v + 1]]
        assert np.all(np.diff(row) > 0)
    assert g.eweight.min() >= 1 and g.eweight.max() < (1 << 20)
    # weights are symmetric per pair
    src = np.repeat(np.arange(g.nodes), np.diff(g.nindex))
    w = {(int(a), int(b)): int(c) for a, b, c in zip(src, g.nlist, g.eweight)}
    assert all(w[(b, a)] == c for (a, b), c in w.items())
    d = ecl.gen_rmat(10, 8, seed=2, symmetrise=False)
    assert not d.validate(symmetric=True)
    assert d.validate(no_self_loops=True)


def test_er_generator(ecl):
    g = ecl.gen_er(512, 0.01, seed=4, weight_seed=5, weight_min=1, weight_max=1000)
    exp = 512 * 511 * 0.01
    assert 0.8 * exp < g.edges < 1.2 * exp
    assert g.validate(no_self_loops=True)
    assert g.eweight.min() >= 1 and g.eweight.max() <= 1000
    s = ecl.gen_er(512, 0.01, seed=4, symmetrise=True)
    assert s.validate(symmetric=True, no_self_loops=True)
