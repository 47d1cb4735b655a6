"""The CPU oracle on hand-checked graphs and against the reference's own
self-checks (CPU only).  Fixture-based pins live in test_golden.py."""
import numpy as np

from conftest import from_edges, undirected


def test_cc_hand(orc):
    g = undirected(7, [(0, 3), (3, 5), (1, 2), (6, 2)])
    assert list(orc.cc(g)) == [0, 1, 1, 0, 4, 0, 1]
    assert orc.verify_cc(g, orc.cc(g)) == 0
    assert orc.verify_cc(g, np.array([0, 1, 1, 0, 4, 0, 2], np.int32)) != 0


def test_cc_asymmetric_uses_smaller_entries_only(orc):
    # 2 -> 0 is a "smaller" entry (hooked); 1 -> 3 is not (ignored), as in
    # ECL-CC-atomic.cu:132.
    g = from_edges(4, [(2, 0), (1, 3)])
    assert list(orc.cc(g)) == [0, 1, 0, 3]


def test_mis_priority_formula(orc):
    g = undirected(4, [(0, 1), (1, 2), (2, 3)])
    p = orc.mis_priority(g)
    assert all(int(x) & 1 for x in p)
    iso = undirected(3, [(0, 1)])
    assert orc.mis_priority(iso)[2] == 0xFE


def test_mis_greedy_and_verify(orc, ecl):
    g = ecl.gen_rmat(10, 8, seed=7)
    st = orc.mis(g)
    assert orc.verify_mis(g, st) == 0
    p = orc.mis_priority(g)
    # the highest (byte, id) vertex with degree > 0 is always in the set
    deg = np.diff(g.nindex)
    cand = [v for v in range(g.nodes) if deg[v] > 0]
    top = max(cand, key=lambda v: (int(p[v]), v))
    assert st[top] == 0xFE


def test_gc_greedy_and_verify(orc, ecl):
    g = ecl.gen_rmat(10, 8, seed=8)
    col = orc.gc(g)
    rc, k = orc.verify_gc(g, col)
    assert rc == 0 and k >= 2
    assert orc.verify_gc(g, np.zeros(g.nodes, np.int32))[0] != 0


def test_mst_hand(orc):
    # square with a diagonal; unique by (w, j)
    g = undirected(4, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2)], weights=[1, 1, 5, 1, 1])
    inm, tot = orc.mst(g)
    assert tot == 3 and int(inm.sum()) == 3
    # only v<n copies are flagged
    src = np.repeat(np.arange(4), np.diff(g.nindex))
    assert all(g.nlist[j] > src[j] for j in np.nonzero(inm)[0])


def test_scc_hand(orc):
    g = from_edges(6, [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 3), (5, 5)])
    assert list(orc.scc(g)) == [2, 2, 2, 4, 4, 5]


def test_apsp_hand(orc):
    INF = 0x7FFFFFFF // 2
    g = from_edges(3, [(0, 1), (1, 2), (0, 2), (0, 2)], weights=[2, 3, 9, 7])
    d = orc.apsp(g)
    assert d[0, 2] == 5 and d[0, 1] == 2 and d[1, 2] == 3
    assert d[2, 0] == INF and d[1, 1] == 0
    # a self-loop overwrites the 0 diagonal (init2, ECL-APSP-atomic.cu:79)
    s = from_edges(2, [(0, 0), (0, 1)], weights=[4, 1])
    assert orc.apsp(s)[0, 0] == 4


def _omp_graphs(ecl):
    return [
        ecl.gen_rmat(14, 16, seed=2),
        ecl.gen_rmat(13, 8, seed=9, symmetrise=False),
        ecl.gen_grid(120, 90, 0.2, seed=3),
        ecl.gen_er(3000, 0.003, seed=4, symmetrise=True),
        undirected(2100, [(2099, i) for i in range(2099)] + [(i, i + 1) for i in range(0, 300, 2)]),
    ]


def test_openmp_baselines_match_the_serial_oracle(orc, ecl):
    """The OpenMP CPU baselines (bench.py's CPU legs for CC, MIS, GC and SCC)
    return exactly the serial oracle's results."""
    assert orc.omp_threads() >= 1
    for g in _omp_graphs(ecl):
        assert np.array_equal(orc.omp_cc(g), orc.cc(g))
        assert np.array_equal(orc.omp_scc(g), orc.scc(g))
        if g.symmetric:
            assert np.array_equal(orc.omp_mis(g), orc.mis(g))
            assert np.array_equal(orc.omp_gc(g), orc.gc(g))


def test_apsp_rows_match_the_closure(orc, ecl):
    """Dijkstra rows (used at full size) equal rows of the FW restatement."""
    for g in [ecl.gen_er(300, 0.02, seed=4, weight_seed=5), ecl.gen_er(257, 0.05, seed=9, weight_seed=2)]:
        full = orc.apsp(g)
        rows = np.array([0, 7, 100, g.nodes - 1], np.int32)
        assert np.array_equal(orc.apsp_rows(g, rows), full[rows])
    # duplicates: the last entry of an arc wins, as in the matrix fill
    d = from_edges(3, [(0, 1), (0, 1), (1, 2)], weights=[9, 4, 2])
    assert np.array_equal(orc.apsp_rows(d, np.array([0])), orc.apsp(d)[[0]])


def test_oracle_generators_equal_the_library_generators(orc, ecl):
    """The reference arm of the bench builds its graphs with the oracle's
    restated generators (it must not load the product library); they give the
    same CSR and weights byte for byte as ecl_gen_rmat / _grid / _er."""

    def same(a, b):
        if not (np.array_equal(a.nindex, b.nindex) and np.array_equal(a.nlist, b.nlist)):
            return False
        if a.eweight is None or b.eweight is None:
            return a.eweight is None and b.eweight is None
        return np.array_equal(a.eweight, b.eweight)

    assert same(orc.gen_rmat(13, 16, seed=2, weight_seed=3), ecl.gen_rmat(13, 16, seed=2, weight_seed=3))
    assert same(orc.gen_rmat(12, 16, seed=2, symmetrise=False), ecl.gen_rmat(12, 16, seed=2, symmetrise=False))
    assert same(orc.gen_rmat(11, 8, 0.45, 0.15, 0.15, seed=7), ecl.gen_rmat(11, 8, 0.45, 0.15, 0.15, seed=7))
    assert same(orc.gen_grid(64, 48, 0.05, seed=1), ecl.gen_grid(64, 48, 0.05, seed=1))
    assert same(orc.gen_grid(30, 20, 0.3, seed=1, weight_seed=9, weight_max=1 << 16),
                ecl.gen_grid(30, 20, 0.3, seed=1, weight_seed=9, weight_max=1 << 16))
    assert same(orc.gen_er(2000, 0.004, seed=4, weight_seed=5), ecl.gen_er(2000, 0.004, seed=4, weight_seed=5))
    assert same(orc.gen_er(2000, 0.004, seed=4, symmetrise=True, weight_seed=5),
                ecl.gen_er(2000, 0.004, seed=4, symmetrise=True, weight_seed=5))
