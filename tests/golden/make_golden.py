"""Generates tests/golden/*.npz from the REFERENCE implementation itself.

Each fixture holds a small seeded input graph and the output that the
reference produced on it:
  cc / mis / gc / scc : the reference's race-free GPU kernels
                        (oracle/_ref/libeclref.so, compiled unchanged from the
                        ECL-Suite sources by `make -C oracle ref`), run on a B200;
  mst                 : the reference's CPU routine cpuMST (ECL-MST_10-atomic.cu:112);
  apsp                : the reference's CPU routine FW_cpu (ECL-APSP-atomic.cu:533).

Usage (on a machine with a B200 and the built oracle/_ref library):
    python tests/golden/make_golden.py OUTDIR
The fixtures in tests/golden/ were made this way and then copied there.
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "ecl-suite_b200"), os.path.join(ROOT, "tests")]

import ecl_b200 as ecl  # noqa: E402  (generators only)
from conftest import from_edges, undirected  # noqa: E402

REF = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libeclref.so"))
REF.eclref_cc_device.restype = C.c_float
REF.eclref_mis_device.restype = C.c_float
REF.eclref_gc_device.restype = C.c_float
REF.eclref_gc_scratch_bytes.restype = C.c_size_t
REF.eclref_scc_device.restype = C.c_float
REF.eclref_scc_scratch_bytes.restype = C.c_size_t
REF.eclref_mst_cpu.restype = C.c_double
REF.eclref_apsp_cpu.restype = C.c_double


def P(a):
    return C.c_void_p(a.ctypes.data if hasattr(a, "ctypes") else a.data_ptr())


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ref_cc(g):
    import torch

    ni, nl = dev(g.nindex), dev(g.nlist if g.edges else np.zeros(1, np.int32))
    st = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    wl = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    REF.eclref_cc_device(g.nodes, C.c_void_p(ni.data_ptr()), C.c_void_p(nl.data_ptr()), C.c_void_p(st.data_ptr()),
                         C.c_void_p(wl.data_ptr()))
    return st.cpu().numpy()


def ref_mis(g):
    import torch

    ni, nl = dev(g.nindex), dev(g.nlist if g.edges else np.zeros(1, np.int32))
    st = torch.empty((g.nodes + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    REF.eclref_mis_device(g.nodes, g.edges, C.c_void_p(ni.data_ptr()), C.c_void_p(nl.data_ptr()),
                          C.c_void_p(st.data_ptr()))
    return st.cpu().numpy()[: g.nodes]


def ref_gc(g):
    import torch

    ni, nl = dev(g.nindex), dev(g.nlist if g.edges else np.zeros(1, np.int32))
    col = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    scr = torch.empty(REF.eclref_gc_scratch_bytes(g.nodes, g.edges) // 4 + 1, dtype=torch.int32, device="cuda")
    REF.eclref_gc_device(g.nodes, g.edges, C.c_void_p(ni.data_ptr()), C.c_void_p(nl.data_ptr()),
                         C.c_void_p(col.data_ptr()), C.c_void_p(scr.data_ptr()))
    return col.cpu().numpy()


def ref_scc(g):
    import torch

    ni, nl = dev(g.nindex), dev(g.nlist if g.edges else np.zeros(1, np.int32))
    scr = torch.empty(REF.eclref_scc_scratch_bytes(g.nodes, g.edges) // 8 + 2, dtype=torch.int64, device="cuda")
    lab = np.empty(g.nodes, np.int32)
    REF.eclref_scc_device(g.nodes, g.edges, C.c_void_p(ni.data_ptr()), C.c_void_p(nl.data_ptr()), P(lab),
                          C.c_void_p(scr.data_ptr()))
    return lab


def ref_mst(g):
    out = np.zeros(max(g.edges, 1), np.uint8)
    REF.eclref_mst_cpu(g.nodes, g.edges, P(g.nindex), P(g.nlist), P(g.eweight), P(out))
    out = out[: g.edges]
    src = np.repeat(np.arange(g.nodes), np.diff(g.nindex))
    return out, int(g.eweight[out.astype(bool)].astype(np.int64).sum()) if g.edges else 0


def ref_apsp(g):
    out = np.zeros((g.nodes, g.nodes), np.int32)
    REF.eclref_apsp_cpu(g.nodes, g.edges, P(g.nindex), P(g.nlist), P(g.eweight), P(out))
    return out


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


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    fn = {"cc": ref_cc, "mis": ref_mis, "gc": ref_gc, "scc": ref_scc, "mst": ref_mst, "apsp": ref_apsp}
    for name, code, g in cases():
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
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
