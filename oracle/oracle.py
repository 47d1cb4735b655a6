"""ctypes wrapper of the CPU oracle (oracle.c) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module.  It is the checker, never the thing measured or
shipped; the product library has no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
if not os.path.exists(LIB_PATH):
    raise ImportError(f"oracle not built at {LIB_PATH}; run `make -C oracle`")
_lib = C.CDLL(LIB_PATH)

_P = C.c_void_p
for name, res, args in [
    ("orc_cc", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("orc_verify_cc", C.c_int, [C.c_int, C.c_int, _P, _P, _P]),
    ("orc_mis_priority", None, [C.c_int, C.c_int, _P, _P]),
    ("orc_mis", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("orc_verify_mis", C.c_int, [C.c_int, C.c_int, _P, _P, _P]),
    ("orc_gc", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("orc_verify_gc", C.c_int, [C.c_int, C.c_int, _P, _P, _P, C.POINTER(C.c_int)]),
    ("orc_mst", C.c_uint64, [C.c_int, C.c_int, _P, _P, _P, _P]),
    ("orc_scc", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("orc_apsp", None, [C.c_int, C.c_int, _P, _P, _P, _P, C.c_long]),
    ("orc_apsp_rows", None, [C.c_int, C.c_int, _P, _P, _P, _P, C.c_int, _P]),
    ("omp_cc", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("omp_mis", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("omp_gc", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("omp_scc", None, [C.c_int, C.c_int, _P, _P, _P]),
    ("omp_threads", C.c_int, []),
]:
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args


def _arrs(g):
    nindex = np.ascontiguousarray(g.nindex, dtype=np.int32)
    nlist = np.ascontiguousarray(g.nlist, dtype=np.int32)
    if nlist.size == 0:
        nlist = np.zeros(1, np.int32)
    return int(nindex.shape[0] - 1), int(g.nlist.shape[0]), nindex, nlist


def cc(g) -> np.ndarray:
    n, m, ni, nl = _arrs(g)
    out = np.empty(n, np.int32)
    _lib.orc_cc(n, m, ni.ctypes.data, nl.ctypes.data, out.ctypes.data)
    return out


def verify_cc(g, label) -> int:
    n, m, ni, nl = _arrs(g)
    lab = np.ascontiguousarray(label, dtype=np.int32)
    return _lib.orc_verify_cc(n, m, ni.ctypes.data, nl.ctypes.data, lab.ctypes.data)


def mis_priority(g) -> np.ndarray:
    n, m, ni, _ = _arrs(g)
    out = np.empty(n, np.uint8)
    _lib.orc_mis_priority(n, m, ni.ctypes.data, out.ctypes.data)
    return out


def mis(g) -> np.ndarray:
    n, m, ni, nl = _arrs(g)
    out = np.empty(n, np.uint8)
    _lib.orc_mis(n, m, ni.ctypes.data, nl.ctypes.data, out.ctypes.data)
    return out


def verify_mis(g, status) -> int:
    n, m, ni, nl = _arrs(g)
    st = np.ascontiguousarray(status, dtype=np.uint8)
    return _lib.orc_verify_mis(n, m, ni.ctypes.data, nl.ctypes.data, st.ctypes.data)


def gc(g) -> np.ndarray:
    n, m, ni, nl = _arrs(g)
    out = np.empty(n, np.int32)
    _lib.orc_gc(n, m, ni.ctypes.data, nl.ctypes.data, out.ctypes.data)
    return out


def verify_gc(g, color):
    """Returns (rc, number of colours)."""
    n, m, ni, nl = _arrs(g)
    col = np.ascontiguousarray(color, dtype=np.int32)
    k = C.c_int(0)
    rc = _lib.orc_verify_gc(n, m, ni.ctypes.data, nl.ctypes.data, col.ctypes.data, C.byref(k))
    return rc, k.value


def mst(g):
    """Returns (in_mst bytes, total weight)."""
    n, m, ni, nl = _arrs(g)
    w = np.ascontiguousarray(g.eweight, dtype=np.int32) if m else np.zeros(1, np.int32)
    out = np.zeros(max(m, 1), np.uint8)
    total = _lib.orc_mst(n, m, ni.ctypes.data, nl.ctypes.data, w.ctypes.data, out.ctypes.data)
    return out[:m], int(total)


def scc(g) -> np.ndarray:
    n, m, ni, nl = _arrs(g)
    out = np.empty(n, np.int32)
    _lib.orc_scc(n, m, ni.ctypes.data, nl.ctypes.data, out.ctypes.data)
    return out


def apsp_rows(g, rows) -> np.ndarray:
    """Rows of the APSP closure by Dijkstra (no self-loops; last duplicate wins)."""
    n, m, ni, nl = _arrs(g)
    w = np.ascontiguousarray(g.eweight, dtype=np.int32) if m else np.zeros(1, np.int32)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.empty((r.size, n), np.int32)
    _lib.orc_apsp_rows(n, m, ni.ctypes.data, nl.ctypes.data, w.ctypes.data, r.ctypes.data, int(r.size), out.ctypes.data)
    return out


def apsp(g) -> np.ndarray:
    n, m, ni, nl = _arrs(g)
    w = np.ascontiguousarray(g.eweight, dtype=np.int32) if m else np.zeros(1, np.int32)
    out = np.empty((n, n), np.int32)
    _lib.orc_apsp(n, m, ni.ctypes.data, nl.ctypes.data, w.ctypes.data, out.ctypes.data, n)
    return out


# ---- OpenMP CPU baselines (omp_baseline.c): same results, all host threads ----


def omp_threads() -> int:
    return int(_lib.omp_threads())


def _omp(name, g, dtype):
    n, m, ni, nl = _arrs(g)
    out = np.empty(n, dtype)
    getattr(_lib, name)(n, m, ni.ctypes.data, nl.ctypes.data, out.ctypes.data)
    return out


def omp_cc(g) -> np.ndarray:
    return _omp("omp_cc", g, np.int32)


def omp_mis(g) -> np.ndarray:
    return _omp("omp_mis", g, np.uint8)


def omp_gc(g) -> np.ndarray:
    return _omp("omp_gc", g, np.int32)


def omp_scc(g) -> np.ndarray:
    return _omp("omp_scc", g, np.int32)


# ---- seeded generators (gen.c): the benchmark graphs without the product library ----


class _GenGraph(C.Structure):
    _fields_ = [("nodes", C.c_int32), ("edges", C.c_int32), ("nindex", C.POINTER(C.c_int32)),
                ("nlist", C.POINTER(C.c_int32)), ("eweight", C.POINTER(C.c_int32))]


class Graph:
    """CSR arrays with the attribute names the oracle functions read."""

    def __init__(self, nindex, nlist, eweight=None, symmetric=False):
        self.nindex = np.ascontiguousarray(nindex, dtype=np.int32)
        self.nlist = np.ascontiguousarray(nlist, dtype=np.int32)
        self.eweight = None if eweight is None else np.ascontiguousarray(eweight, dtype=np.int32)
        self.symmetric = symmetric

    @property
    def nodes(self) -> int:
        return int(self.nindex.shape[0] - 1)

    @property
    def edges(self) -> int:
        return int(self.nlist.shape[0])


_lib.gen_rmat.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int32,
                          C.c_uint64, C.c_int32, C.POINTER(_GenGraph)]
_lib.gen_grid.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_uint64, C.c_uint64, C.c_int32, C.POINTER(_GenGraph)]
_lib.gen_er.argtypes = [C.c_int32, C.c_double, C.c_uint64, C.c_int32, C.c_uint64, C.c_int32, C.c_int32,
                        C.POINTER(_GenGraph)]
_lib.gen_free.argtypes = [C.POINTER(_GenGraph)]
for _f in (_lib.gen_rmat, _lib.gen_grid, _lib.gen_er):
    _f.restype = C.c_int
_lib.gen_free.restype = None


def _gen_take(rc, g, symmetric, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")
    try:
        n, m = g.nodes, g.edges
        nindex = np.ctypeslib.as_array(g.nindex, shape=(n + 1,)).copy()
        nlist = np.ctypeslib.as_array(g.nlist, shape=(m,)).copy() if m else np.zeros(0, np.int32)
        ew = np.ctypeslib.as_array(g.eweight, shape=(m,)).copy() if (g.eweight and m) else None
    finally:
        _lib.gen_free(C.byref(g))
    return Graph(nindex, nlist, ew, symmetric)


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=2, symmetrise=True, weight_seed=0,
             weight_max=1 << 20) -> Graph:
    g = _GenGraph()
    rc = _lib.gen_rmat(scale, edge_factor, a, b, c, seed, int(symmetrise), weight_seed, weight_max, C.byref(g))
    return _gen_take(rc, g, symmetrise, "gen_rmat")


def gen_grid(rows, cols, delete_frac=0.05, seed=1, weight_seed=0, weight_max=1 << 20) -> Graph:
    g = _GenGraph()
    rc = _lib.gen_grid(rows, cols, delete_frac, seed, weight_seed, weight_max, C.byref(g))
    return _gen_take(rc, g, True, "gen_grid")


def gen_er(n, p, seed=4, symmetrise=False, weight_seed=0, weight_min=1, weight_max=1000) -> Graph:
    g = _GenGraph()
    rc = _lib.gen_er(n, p, seed, int(symmetrise), weight_seed, weight_min, weight_max, C.byref(g))
    return _gen_take(rc, g, symmetrise, "gen_er")
