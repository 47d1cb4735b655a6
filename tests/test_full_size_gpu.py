"""Parity at the benchmark configs' full sizes (one B200).

- Grid: CC on the 1024x1024 grid with 5 % of edges deleted, equal to the
  oracle.
- R-MAT-22 suite: CC, MIS, GC and MST on symmetrised R-MAT-22 and SCC on the
  directed R-MAT-22, each equal to the oracle.  The oracles take about 30 s of
  host time here, MST's Kruskal most of it.
- APSP: ER n=8192.  An O(n^3) host closure would take hours, so
  32 random rows are checked exactly against Dijkstra from those sources.
- Batch: the 4096-graph mix, 16 sampled graphs against the oracle.

The same configs are also compared with the reference's OWN race-free CUDA
build (oracle/_ref, the reference's .cu files compiled unchanged) on the same
graphs: CC, MIS, GC and SCC labels against its kernels, the MST edge set and
weight against its cpuMST, and the APSP distances against FW_gpu_64.
"""
import numpy as np
import pytest

import refbuild

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not refbuild.available(), reason="oracle/_ref not built (make -C oracle ref)")


@pytest.fixture(scope="module")
def rmat22(ecl):
    sym = ecl.gen_rmat(22, 16, seed=2, symmetrise=True, weight_seed=3)
    dirg = ecl.gen_rmat(22, 16, seed=2, symmetrise=False)
    return sym, dirg, sym.to_device("cuda"), dirg.to_device("cuda")


def test_grid_cc_full_size(ecl, orc):
    g = ecl.gen_grid(1024, 1024, 0.05, seed=1)
    assert np.array_equal(ecl.cc(g.to_device("cuda")).cpu().numpy(), orc.cc(g))


def test_rmat22_cc_mis_scc_full_size(ecl, orc, rmat22):
    sym, dirg, dsym, ddir = rmat22
    assert np.array_equal(ecl.cc(dsym).cpu().numpy(), orc.cc(sym))
    assert np.array_equal(ecl.mis(dsym).cpu().numpy(), orc.omp_mis(sym))
    assert np.array_equal(ecl.scc(ddir).cpu().numpy(), orc.scc(dirg))


def test_rmat22_gc_full_size(ecl, orc, rmat22):
    sym, _, dsym, _ = rmat22
    got = ecl.gc(dsym).cpu().numpy()
    assert np.array_equal(got, orc.omp_gc(sym))
    rc, ncolors = orc.verify_gc(sym, got)
    assert rc == 0 and ncolors == int(got.max()) + 1


def test_rmat22_mst_full_size(ecl, orc, rmat22):
    sym, _, dsym, _ = rmat22
    in_mst, total = ecl.mst(dsym)
    ref_in, ref_total = orc.mst(sym)
    assert total == ref_total
    assert np.array_equal(in_mst.cpu().numpy(), ref_in)


def test_apsp_er8192_sampled_rows(ecl, orc):
    g = ecl.gen_er(8192, 0.001, seed=4, weight_seed=5, weight_min=1, weight_max=1000)
    src = np.repeat(np.arange(g.nodes), np.diff(g.nindex))
    assert not np.any(src == g.nlist), "the row oracle assumes no self-loops"
    dist = ecl.apsp(g.to_device("cuda")).cpu().numpy()
    rows = np.random.default_rng(7).choice(g.nodes, 32, replace=False).astype(np.int32)
    assert np.array_equal(dist[rows], orc.apsp_rows(g, rows))
    assert np.all(np.diag(dist) == 0)


def test_batch4096_sampled_graphs(ecl, orc):
    """The 4096-graph mix (about 1.4 G CSR entries in 3
    super-batches), CC+MIS+MST on a CUDA-graph replay; 16 sampled graphs are
    checked against the oracle."""
    b = ecl.Batch()
    b.add_mix(4096, n_min=1000, n_max=200000, seed=5, weight_max=1 << 16)
    b.build(ecl.BATCH_CC | ecl.BATCH_MIS | ecl.BATCH_MST)
    b.run()
    _, replay = b.run()
    assert replay
    for i in np.random.default_rng(3).choice(b.graphs, 16, replace=False):
        g = b.graph(int(i))
        assert np.array_equal(b.result(int(i), ecl.BATCH_CC), orc.cc(g)), i
        assert np.array_equal(b.result(int(i), ecl.BATCH_MIS), orc.mis(g)), i
        inm, tot = b.result(int(i), ecl.BATCH_MST)
        einm, etot = orc.mst(g)
        assert tot == etot and np.array_equal(inm, einm), i


# ------------------------------------------------ against the reference's own build


@needs_ref
def test_grid_cc_equals_reference_kernel(ecl):
    g = ecl.gen_grid(1024, 1024, 0.05, seed=1)
    assert np.array_equal(ecl.cc(g.to_device("cuda")).cpu().numpy(), refbuild.cc(g))


@needs_ref
def test_rmat22_cc_mis_scc_equal_reference_kernels(ecl, rmat22):
    sym, dirg, dsym, ddir = rmat22
    assert np.array_equal(ecl.cc(dsym).cpu().numpy(), refbuild.cc(sym))
    assert np.array_equal(ecl.mis(dsym).cpu().numpy(), refbuild.mis(sym))
    assert np.array_equal(ecl.scc(ddir).cpu().numpy(), refbuild.scc(dirg))


@needs_ref
def test_rmat22_gc_equals_reference_kernels(ecl, rmat22):
    """Bit-identical colours, hence the same colour count (the north-star bar
    is "no more colours than the reference")."""
    sym, _, dsym, _ = rmat22
    got = ecl.gc(dsym).cpu().numpy()
    ref = refbuild.gc(sym)
    assert int(got.max()) <= int(ref.max())
    assert np.array_equal(got, ref)


@needs_ref
def test_rmat22_mst_equals_reference_cpumst(ecl, rmat22):
    sym, _, dsym, _ = rmat22
    in_mst, total = ecl.mst(dsym)
    ref_in, ref_total = refbuild.mst_cpu(sym)
    assert total == ref_total
    assert np.array_equal(in_mst.cpu().numpy(), ref_in)


@needs_ref
def test_apsp_er8192_equals_reference_fw_gpu_64(ecl):
    g = ecl.gen_er(8192, 0.001, seed=4, weight_seed=5, weight_min=1, weight_max=1000)
    dist = ecl.apsp(g.to_device("cuda")).cpu().numpy()
    ref = refbuild.apsp_gpu(g)
    assert np.array_equal(dist, ref[: g.nodes, : g.nodes])
