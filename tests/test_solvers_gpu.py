"""MIS, GC, MST, SCC and APSP on the B200 vs the oracle (bit-exact)."""
import numpy as np
import pytest

from conftest import from_edges, overlapping_rows, undirected

pytestmark = pytest.mark.gpu


def sym_cases(ecl):
    yield "single", ecl.Graph(np.array([0, 0], np.int32), np.array([], np.int32), symmetric=True)
    yield "pair", undirected(2, [(0, 1)])
    yield "path", undirected(9, [(i, i + 1) for i in range(8)])
    yield "star", undirected(300, [(0, i) for i in range(1, 300)])
    yield "isolated", undirected(12, [(3, 7), (7, 9)])
    yield "clique", undirected(50, [(i, j) for i in range(50) for j in range(i + 1, 50)])
    yield "grid", ecl.gen_grid(48, 48, 0.05, seed=1)
    yield "rmat12", ecl.gen_rmat(12, 16, seed=2)
    yield "rmat14", ecl.gen_rmat(14, 8, seed=5)
    yield "er", ecl.gen_er(3000, 0.003, seed=4, symmetrise=True)
    yield "hub", undirected(9000, [(8999, i) for i in range(8999)] + [(i, i + 1) for i in range(0, 200, 2)])


def weighted(g, seed=3, wmax=1 << 20):
    """Attach pair-symmetric weights to a symmetric graph."""
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(g.nodes), np.diff(g.nindex))
    lo = np.minimum(src, g.nlist).astype(np.int64)
    hi = np.maximum(src, g.nlist).astype(np.int64)
    key = lo * (g.nodes + 1) + hi
    uniq, inv = np.unique(key, return_inverse=True)
    w = rng.integers(1, wmax, size=uniq.shape[0]).astype(np.int32)
    g.eweight = w[inv]
    return g


# ------------------------------------------------------------------------- MIS


def test_mis_matches_oracle(ecl, orc):
    for name, g in sym_cases(ecl):
        got = ecl.mis(g)
        assert np.array_equal(got, orc.mis(g)), name
        assert orc.verify_mis(g, got) == 0, name


def test_mis_device_resident(ecl, orc):
    g = ecl.gen_rmat(14, 16, seed=2)
    out = ecl.mis(g.to_device())
    assert np.array_equal(out.cpu().numpy(), orc.mis(g))


def test_mis_self_loop_is_rejected(ecl):
    """The reference spins forever on a self-loop (v never beats itself);
    here the device scan reports ECL_ERR_BAD_GRAPH, and host validation
    rejects it before any launch."""
    g = from_edges(3, [(0, 0), (0, 1), (1, 0)])
    with pytest.raises(ecl.EclError) as e:
        ecl.mis(g, max_rounds=50)
    assert e.value.status == ecl.ERR_BAD_GRAPH
    with pytest.raises(ecl.EclError) as e:
        ecl.mis(g, validate=True)
    assert e.value.status == ecl.ERR_BAD_GRAPH


# -------------------------------------------------------------------------- GC


def test_gc_matches_greedy_oracle(ecl, orc):
    for name, g in sym_cases(ecl):
        got = ecl.gc(g)
        exp = orc.gc(g)
        assert orc.verify_gc(g, got)[0] == 0, name
        assert np.array_equal(got, exp), name


def test_gc_large_colour_windows(ecl, orc):
    # a 150-clique forces colours far beyond one 64-colour window
    g = undirected(160, [(i, j) for i in range(150) for j in range(i + 1, 150)] + [(150 + k, k) for k in range(10)])
    got = ecl.gc(g)
    assert np.array_equal(got, orc.gc(g))
    assert got.max() == 149


# ------------------------------------------------------------------------- MST


@pytest.mark.parametrize("core", [1, 7, 64, 0])
@pytest.mark.parametrize("ctas", [0, 1, 4])
def test_gc_core_size_does_not_change_colours(ecl, orc, core, ctas):
    """The leading ranks are coloured in shared memory -- by a cluster of CTAs
    (two by default, one or four here) with a copy of the colours in each --
    and the rest by the grid-wide pull; where the boundary lies (1, 7, 64
    ranks, or the default of 8192) and how many CTAs colour the core change no
    colour.  A 2100-clique
    (every vertex a long row inside the default core) forces colours past the
    first 2048-colour window there."""
    old = ecl.set_tune(gc_core_ranks=core, gc_core_ctas=ctas)
    try:
        cases = list(sym_cases(ecl)) + [("rmat16", ecl.gen_rmat(16, 16, seed=3))]
        if core == 0:
            cases.append(("clique2100", undirected(2100, [(i, j) for i in range(2100) for j in range(i + 1, 2100)])))
        for name, g in cases:
            assert np.array_equal(ecl.gc(g), orc.gc(g)), (core, ctas, name)
    finally:
        ecl.set_tune(old)


def test_gc_short_row_ignores_colours_above_its_range(ecl, orc):
    """A row of <= 32 entries (one lane) whose higher neighbour is a hub with
    colour 64 or more: that colour cannot be its smallest free one and must
    not stand for a low colour (64 would alias 0 in a 64-bit mask).  A
    70-clique with one pendant vertex on every member: the members keep equal
    degrees, so their colours run 0..69, and every pendant of a member
    coloured 1..69 takes colour 0."""
    n = 70
    edges = [(i, j) for i in range(n) for j in range(i + 1, n)] + [(i, n + i) for i in range(n)]
    g = undirected(2 * n, edges)
    got = ecl.gc(g)
    exp = orc.gc(g)
    assert np.array_equal(got, exp)
    assert sorted(got[:n]) == list(range(n))
    for i in range(n):
        if got[i] >= 64:
            assert got[n + i] == 0


def test_mst_matches_kruskal(ecl, orc):
    for name, g in sym_cases(ecl):
        g = weighted(g)
        inm, tot = ecl.mst(g)
        einm, etot = orc.mst(g)
        assert tot == etot, name
        assert np.array_equal(inm, einm), name


def test_mst_ties_broken_by_edge_index(ecl, orc):
    g = ecl.gen_grid(40, 40, 0.0, seed=1)
    g.eweight = np.ones(g.edges, np.int32)  # all weights equal: (w, j) order decides
    inm, tot = ecl.mst(g)
    einm, etot = orc.mst(g)
    assert tot == etot == g.nodes - 1
    assert np.array_equal(inm, einm)


def test_mst_generated_weights_and_filter(ecl, orc):
    # avg degree >= 4 takes the light/heavy path
    g = ecl.gen_rmat(14, 16, seed=2, weight_seed=3, weight_max=1 << 20)
    for sym in (False, True):
        g.symmetric = sym
        inm, tot = ecl.mst(g)
        einm, etot = orc.mst(g)
        assert tot == etot and np.array_equal(inm, einm)


# ------------------------------------------------------------------------- SCC


def dir_cases(ecl):
    yield "cycle", from_edges(5, [(0, 1), (1, 2), (2, 0), (3, 4)])
    yield "two_cycles", from_edges(8, [(0, 1), (1, 0), (1, 2), (2, 3), (3, 4), (4, 2), (5, 6), (6, 7), (7, 5), (4, 5)])
    yield "self", from_edges(3, [(0, 0), (1, 2), (2, 1), (2, 2)])
    yield "dag", from_edges(6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (0, 5)])
    yield "rmat12d", ecl.gen_rmat(12, 16, seed=2, symmetrise=False)
    yield "rmat15d", ecl.gen_rmat(15, 8, seed=7, symmetrise=False)
    yield "er_d", ecl.gen_er(4000, 0.0008, seed=4)
    yield "sym", ecl.gen_rmat(11, 8, seed=3)


def test_scc_matches_tarjan(ecl, orc):
    for name, g in dir_cases(ecl):
        got = ecl.scc(g)
        assert np.array_equal(got, orc.scc(g)), name


# ------------------------------------------------------------------------ APSP


def apsp_cases(ecl):
    yield "tiny", from_edges(3, [(0, 1), (1, 2), (0, 2), (0, 2)], weights=[2, 3, 9, 7])
    yield "selfloop", from_edges(2, [(0, 0), (0, 1)], weights=[4, 1])
    yield "er200", ecl.gen_er(200, 0.02, seed=4, weight_seed=5)
    yield "er300", ecl.gen_er(300, 0.01, seed=9, weight_seed=6)
    yield "er512", ecl.gen_er(512, 0.004, seed=4, weight_seed=4)


def test_apsp_matches_fw(ecl, orc):
    for name, g in apsp_cases(ecl):
        got = ecl.apsp(g)
        assert np.array_equal(got, orc.apsp(g)), name


def test_apsp_leading_dimension_and_device(ecl, orc):
    import torch

    g = ecl.gen_er(256, 0.01, seed=11, weight_seed=12)
    exp = orc.apsp(g)
    out = np.full((256, 300), -7, np.int32)
    ecl.apsp(g, out=out, ld=300)
    assert np.array_equal(out[:, :256], exp) and np.all(out[:, 256:] == -7)
    d = ecl.apsp(g.to_device())  # n % 128 == 0, ld == n: computed in place
    assert np.array_equal(d.cpu().numpy(), exp)


def test_apsp_reference_padded_layout(ecl, orc):
    import ctypes as C

    g = ecl.gen_er(100, 0.03, seed=13, weight_seed=14)
    upper = 128
    out = np.zeros((upper, upper), np.int32)
    st = ecl.lib.ecl_compute_apsp(g.nodes, g.edges, g.nindex.ctypes.data_as(C.POINTER(C.c_int32)),
                                  g.nlist.ctypes.data_as(C.POINTER(C.c_int32)),
                                  g.eweight.ctypes.data_as(C.POINTER(C.c_int32)), out.ctypes.data_as(C.POINTER(C.c_int32)))
    assert st == 0
    assert np.array_equal(out[:100, :100], orc.apsp(g))
    assert np.all(out[100:, :] == ecl.APSP_INF) and np.all(out[:, 100:] == ecl.APSP_INF)


# ---------------------------------------------------------- malformed input and wait limits


@pytest.mark.parametrize("code", ["cc", "mis", "gc", "mst", "scc"])
def test_overlapping_rows_are_rejected_on_the_device(ecl, orc, code):
    """Without host validation the kernels see the overlapping rows: each code
    reports ECL_ERR_BAD_GRAPH (chunk records beyond the buffer are counted,
    not written), and the next solve on the same device is correct."""
    g = overlapping_rows()
    with pytest.raises(ecl.EclError) as e:
        getattr(ecl, code)(g.to_device(), validate=False)
    assert e.value.status == ecl.ERR_BAD_GRAPH
    ok = ecl.gen_rmat(12, 8, seed=2, weight_seed=3)
    assert np.array_equal(ecl.cc(ok), orc.cc(ok))


def test_mis_wait_limit_reports_no_convergence_then_recovers(ecl, orc):
    """A 100k-vertex path needs many dependent sweeps; capped at max_rounds = 1
    the persistent launch gives up with ECL_ERR_NO_CONVERGENCE instead of
    sweeping on, and the next solve on the same stream is bit-exact."""
    import torch

    n = 100000
    g = undirected(n, [(i, i + 1) for i in range(n - 1)])
    dg = g.to_device()
    with pytest.raises(ecl.EclError) as e:
        ecl.mis(dg, max_rounds=1)
    assert e.value.status == ecl.ERR_NO_CONVERGENCE
    torch.cuda.synchronize()
    assert np.array_equal(ecl.mis(dg).cpu().numpy(), orc.mis(g))


def test_scc_round_limit_reports_no_convergence_then_recovers(ecl, orc):
    """A chain of 2-cycles c0 -> c1 -> ... needs one trimming round per cycle
    (only the last cycle's maximum reaches back); max_rounds = 1 stops after
    the first round with ECL_ERR_NO_CONVERGENCE, and the next solve on the
    same stream equals the oracle."""
    k = 64
    edges = []
    for c in range(k):
        a, b = 2 * c, 2 * c + 1
        edges += [(a, b), (b, a)]
        if c + 1 < k:
            edges.append((b, 2 * c + 2))
    g = from_edges(2 * k, sorted(edges))
    dg = g.to_device()
    with pytest.raises(ecl.EclError) as e:
        ecl.scc(dg, max_rounds=1)
    assert e.value.status == ecl.ERR_NO_CONVERGENCE
    assert np.array_equal(ecl.scc(dg).cpu().numpy(), orc.scc(g))


def test_cc_validate_checks_the_symmetric_flag(ecl):
    """CC's sampling path uses each entry in both directions, so with
    validation on, an asymmetric graph flagged symmetric is rejected on the
    host before any launch."""
    g = from_edges(4, [(0, 1), (2, 3), (3, 2)], symmetric=True)
    with pytest.raises(ecl.EclError) as e:
        ecl.cc(g, validate=True)
    assert e.value.status == ecl.ERR_BAD_GRAPH


@pytest.mark.parametrize("knobs", [dict(row_lane_max=1, row_chunk=128), dict(row_lane_max=8, row_chunk=512),
                                   dict(row_lane_max=32, row_chunk=8192, blocks_per_sm=2),
                                   dict(mst_light_factor=0.4, gc_core_ranks=5, gc_pull_blocks=4, gc_core_ctas=4),
                                   dict(gc_poll_ns=2048, row_vec=1, scc_sweep_batch=4, gc_pull_blocks=1, gc_core_ctas=2)])
def test_launch_knobs_never_change_results(ecl, orc, knobs):
    """Every code under non-default degree bins, grid sizes, MST split and GC
    core size gives the oracle's result (hub rows cross every chunk size)."""
    old = ecl.set_tune(**knobs)
    try:
        g = weighted(ecl.gen_rmat(15, 16, seed=2))
        hub = undirected(9000, [(8999, i) for i in range(8999)] + [(i, i + 1) for i in range(0, 200, 2)])
        for h in (g, hub):
            assert np.array_equal(ecl.cc(h), orc.cc(h)), knobs
            assert np.array_equal(ecl.mis(h), orc.mis(h)), knobs
            assert np.array_equal(ecl.gc(h), orc.gc(h)), knobs
        inm, tot = ecl.mst(g)
        einm, etot = orc.mst(g)
        assert tot == etot and np.array_equal(inm, einm), knobs
        d = ecl.gen_rmat(14, 16, seed=2, symmetrise=False)
        assert np.array_equal(ecl.scc(d), orc.scc(d)), knobs
    finally:
        ecl.set_tune(old)


def test_mst_on_arrays_that_are_not_16_byte_aligned(ecl, orc):
    """Device CSR arrays that start 4 bytes past an allocation: the scans see
    that 16-byte row loads would be misaligned and keep to 4-byte loads; the
    forest is the same."""
    import torch

    g = ecl.gen_rmat(14, 16, seed=2, weight_seed=3)
    nl = torch.empty(g.edges + 1, dtype=torch.int32, device="cuda")
    ew = torch.empty(g.edges + 1, dtype=torch.int32, device="cuda")
    nl[1:] = torch.from_numpy(g.nlist).cuda()
    ew[1:] = torch.from_numpy(g.eweight).cuda()
    dg = ecl.DeviceGraph(torch.from_numpy(g.nindex).cuda(), nl[1:], ew[1:], True)
    assert dg.nlist.data_ptr() % 16 == 4
    inm, tot = ecl.mst(dg)
    einm, etot = orc.mst(g)
    assert tot == etot and np.array_equal(inm.cpu().numpy(), einm)
