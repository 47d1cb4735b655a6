"""Generates tests/golden/*.npz from the REFERENCE implementation itself.

Each fixture holds a small seeded input graph and the output that the
reference produced on it:
  cc / mis / gc / scc : the reference's race-free GPU kernels
                        (oracle/_ref/libeclref.so, compiled unchanged from the
                        ECL-Suite sources by `make -C oracle ref`), run on a B200;
  mst                 : the reference's CPU routine cpuMST (ECL-MST_10-atomic.cu:112);
  apsp                : the reference's CPU routine FW_cpu (ECL-APSP-atomic.cu:533).

Usage (on a machine with a B200 and the built oracle/_ref library):
    python tests/golden/make_golden.py OUTDIR [NAME ...]
The fixtures in tests/golden/ were made this way and then copied there.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "ecl-suite_b200"), os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import ecl_b200 as ecl  # noqa: E402  (generators only)
from conftest import from_edges, undirected  # noqa: E402

import refbuild  # noqa: E402  (the reference's own build, oracle/_ref)

ref_cc, ref_mis, ref_gc, ref_scc, ref_mst, ref_apsp = (refbuild.cc, refbuild.mis, refbuild.gc, refbuild.scc,
                                                       refbuild.mst_cpu, refbuild.apsp_cpu)


def pair_weights(g, seed):
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(g.nodes), np.diff(g.nindex))
    key = np.minimum(src, g.nlist).astype(np.int64) * (g.nodes + 1) + np.maximum(src, g.nlist)
    uniq, inv = np.unique(key, return_inverse=True)
    g.eweight = rng.integers(1, 1 << 20, size=uniq.shape[0]).astype(np.int32)[inv]
    return g


def cases():
    sym = {
        "path": undirected(17, [(i, i + 1) for i in range(16)]),
        "star": undirected(100, [(0, i) for i in range(1, 100)]),
        "grid32": ecl.gen_grid(32, 32, 0.05, seed=1),
        "rmat11": ecl.gen_rmat(11, 16, seed=2),
        "er1500": ecl.gen_er(1500, 0.004, seed=4, symmetrise=True),
    }
    for name, g in sym.items():
        yield f"cc_{name}", "cc", g
        yield f"mis_{name}", "mis", g
        yield f"gc_{name}", "gc", g
        yield f"mst_{name}", "mst", pair_weights(ecl.Graph(g.nindex, g.nlist, None, True), 3)
    yield "cc_asym", "cc", from_edges(8, [(2, 0), (1, 3), (5, 4), (4, 1), (7, 6), (6, 5)])
    yield "cc_rmat10_directed", "cc", ecl.gen_rmat(10, 8, seed=9, symmetrise=False)
    yield "mst_ties", "mst", ecl.Graph(ecl.gen_grid(16, 16, 0.0).nindex, ecl.gen_grid(16, 16, 0.0).nlist,
                                       np.ones(ecl.gen_grid(16, 16, 0.0).edges, np.int32), True)
    yield "scc_cycles", "scc", from_edges(8, [(0, 1), (1, 0), (1, 2), (2, 3), (3, 4), (4, 2), (5, 6), (6, 7), (7, 5), (4, 5)])
    yield "scc_rmat11", "scc", ecl.gen_rmat(11, 16, seed=2, symmetrise=False)
    yield "scc_er2000", "scc", ecl.gen_er(2000, 0.0012, seed=4)
    yield "apsp_dups", "apsp", from_edges(4, [(0, 1), (0, 1), (1, 2), (2, 3), (0, 0), (3, 0)], weights=[9, 5, 2, 7, 3, 1])
    yield "apsp_er130", "apsp", ecl.gen_er(130, 0.03, seed=4, weight_seed=5)
    yield "apsp_er200", "apsp", ecl.gen_er(200, 0.02, seed=6, weight_seed=7)
    # more than 64 colours: the reference's runLarge keeps the candidate
    # colours of rows with 32 or more higher-priority entries in posscol2
    # bitmaps (ECL-GC-atomic.cu:144, 148-251), a path no smaller case reaches
    yield "gc_clique150", "gc", undirected(150, [(i, j) for i in range(150) for j in range(i + 1, 150)])
    yield "gc_rmat13_ef64", "gc", ecl.gen_rmat(13, 64, seed=2)


def main(outdir, only=()):
    os.makedirs(outdir, exist_ok=True)
    fn = {"cc": ref_cc, "mis": ref_mis, "gc": ref_gc, "scc": ref_scc, "mst": ref_mst, "apsp": ref_apsp}
    for name, code, g in cases():
        if only and name not in only:
            continue
        res = fn[code](g)
        arrs = dict(nindex=g.nindex, nlist=g.nlist, code=np.array(code))
        if g.eweight is not None:
            arrs["eweight"] = g.eweight
        if code == "mst":
            arrs["in_mst"], arrs["total"] = res[0], np.array(res[1], np.int64)
        else:
            arrs["expected"] = res
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **arrs)
        print(name, code, g.nodes, g.edges)


if __name__ == "__main__":
    # make_golden.py [OUTDIR [NAME ...]]: every fixture, or only the named ones
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)), tuple(sys.argv[2:]))
