"""Python host binding of libeclb200.so (the B200-native race-free graph codes).

The library is C++/CUDA behind a C ABI (include/ecl_b200.h); this module only
marshals arguments through ctypes.  There is no Python or CPU compute path:
if the shared library is missing the import fails, and every solver runs the
sm_100a kernels.

Operators mirror the reference's per-code contracts (ECL-Suite,
src/racefree/...): ``cc`` returns nstat labels, ``mis`` the 0xfe/0 status
bytes, ``gc`` colours, ``mst`` the in_mst edge flags, ``scc`` max-id labels,
``apsp`` the distance matrix.  Arguments are either an :class:`Graph` of host
numpy arrays (the call copies to the device and back) or a
:class:`DeviceGraph` of torch CUDA tensors (nothing crosses PCIe).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libeclb200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libeclb200.so not built at {LIB_PATH}; run `make -C ecl-suite_b200` or __graft_entry__.build()")

lib = C.CDLL(LIB_PATH)

# ---- status / enums --------------------------------------------------------------

OK, ERR_INVALID_ARG, ERR_BAD_GRAPH, ERR_OOM, ERR_NO_CONVERGENCE, ERR_CUDA, ERR_IO, ERR_UNSUPPORTED, ERR_NO_DEVICE = range(9)
HOST, DEVICE = 0, 1
GRAPH_SYMMETRIC = 0x1
CC, MIS, GC, MST, SCC, APSP = range(6)
MIS_IN, MIS_OUT = 0xFE, 0x00
APSP_INF = 0x7FFFFFFF // 2


class EclError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib.ecl_status_string(status).decode()
        last = lib.ecl_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}){' - ' + last if last else ''}")
        self.status = status


class GraphView(C.Structure):
    _fields_ = [
        ("nodes", C.c_int32),
        ("edges", C.c_int32),
        ("nindex", C.c_void_p),
        ("nlist", C.c_void_p),
        ("eweight", C.c_void_p),
        ("location", C.c_int32),
        ("flags", C.c_int32),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("stream", C.c_void_p),
        ("workspace", C.c_void_p),
        ("workspace_bytes", C.c_size_t),
        ("validate", C.c_int32),
        ("max_rounds", C.c_int32),
        ("elapsed_ms", C.c_float),
        ("rounds", C.c_int32),
        ("detail", C.c_int32),
        ("nphases", C.c_int32),
        ("phase_ms", C.c_float * 8),
    ]


class CGraph(C.Structure):
    _fields_ = [
        ("nodes", C.c_int32),
        ("edges", C.c_int32),
        ("nindex", C.POINTER(C.c_int32)),
        ("nlist", C.POINTER(C.c_int32)),
        ("eweight", C.POINTER(C.c_int32)),
    ]


_VP, _I32, _U64, _F64 = C.c_void_p, C.c_int32, C.c_uint64, C.c_double
_PV, _PO, _PG = C.POINTER(GraphView), C.POINTER(Opts), C.POINTER(CGraph)


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_sig("ecl_abi_version", C.c_int32, [])
_sig("ecl_status_string", C.c_char_p, [C.c_int])
_sig("ecl_last_error", C.c_char_p, [])
_sig("ecl_workspace_bytes", C.c_size_t, [C.c_int, _I32, _I32])
_sig("ecl_kernel_launches", C.c_uint64, [])
_sig("ecl_minplus_peak", C.c_int, [C.c_int32, C.POINTER(C.c_double)])
_sig("ecl_hop_latency", C.c_int, [C.c_int32, C.POINTER(C.c_double)])
_sig("ecl_gather_peak", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)])
_sig("ecl_gc_critical_path", C.c_int, [_PV, C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_double)])
_sig("ecl_cc", C.c_int, [_PV, _VP, _PO])
_sig("ecl_mis", C.c_int, [_PV, _VP, _PO])
_sig("ecl_gc", C.c_int, [_PV, _VP, _PO])
_sig("ecl_mst", C.c_int, [_PV, _VP, C.POINTER(C.c_uint64), _PO])
_sig("ecl_scc", C.c_int, [_PV, _VP, _PO])
_sig("ecl_apsp", C.c_int, [_PV, _VP, C.c_int64, _PO])
_sig("ecl_graph_read", C.c_int, [C.c_char_p, _PG])
_sig("ecl_graph_write", C.c_int, [C.c_char_p, _PG])
_sig("ecl_graph_free", None, [_PG])
_sig("ecl_graph_validate", C.c_int, [_PV, _I32, _I32])
_sig("ecl_gen_rmat", C.c_int, [_I32, _I32, _F64, _F64, _F64, _U64, _I32, _U64, _I32, _PG])
_sig("ecl_gen_grid", C.c_int, [_I32, _I32, _F64, _U64, _U64, _I32, _PG])
_sig("ecl_gen_er", C.c_int, [_I32, _F64, _U64, _I32, _U64, _I32, _I32, _PG])

# Every symbol that include/ecl_b200.h declares (checked by the CPU tests).
EXPORTED = [
    "ecl_abi_version", "ecl_status_string", "ecl_last_error", "ecl_workspace_bytes", "ecl_kernel_launches",
    "ecl_minplus_peak", "ecl_hop_latency", "ecl_gather_peak", "ecl_gc_critical_path", "ecl_set_tune", "ecl_get_tune",
    "ecl_cc", "ecl_mis", "ecl_gc", "ecl_mst", "ecl_scc", "ecl_apsp",
    "ecl_compute_cc", "ecl_compute_mis", "ecl_compute_gc", "ecl_compute_mst", "ecl_compute_scc", "ecl_compute_apsp",
    "ecl_graph_read", "ecl_graph_write", "ecl_graph_free", "ecl_graph_validate",
    "ecl_gen_rmat", "ecl_gen_grid", "ecl_gen_er",
]


def _check(st: int, where: str) -> None:
    if st != OK:
        raise EclError(st, where)


# ---- graphs ----------------------------------------------------------------------


@dataclass
class Graph:
    """ECLgraph CSR in host memory (library/ECLgraph.h:41-47)."""

    nindex: np.ndarray
    nlist: np.ndarray
    eweight: Optional[np.ndarray] = None
    symmetric: bool = False

    def __post_init__(self):
        self.nindex = np.ascontiguousarray(self.nindex, dtype=np.int32)
        self.nlist = np.ascontiguousarray(self.nlist, dtype=np.int32)
        if self.eweight is not None:
            self.eweight = np.ascontiguousarray(self.eweight, dtype=np.int32)

    @property
    def nodes(self) -> int:
        return int(self.nindex.shape[0] - 1)

    @property
    def edges(self) -> int:
        return int(self.nlist.shape[0])

    def view(self) -> GraphView:
        v = GraphView()
        v.nodes, v.edges = self.nodes, self.edges
        v.nindex = self.nindex.ctypes.data
        v.nlist = self.nlist.ctypes.data if self.edges else None
        v.eweight = self.eweight.ctypes.data if self.eweight is not None else None
        v.location = HOST
        v.flags = GRAPH_SYMMETRIC if self.symmetric else 0
        return v

    def validate(self, symmetric: bool = False, no_self_loops: bool = False) -> bool:
        v = self.view()
        return lib.ecl_graph_validate(C.byref(v), int(symmetric), int(no_self_loops)) == OK

    def write(self, path: str) -> None:
        cg = CGraph(self.nodes, self.edges,
                    self.nindex.ctypes.data_as(C.POINTER(C.c_int32)),
                    self.nlist.ctypes.data_as(C.POINTER(C.c_int32)),
                    self.eweight.ctypes.data_as(C.POINTER(C.c_int32)) if self.eweight is not None else None)
        _check(lib.ecl_graph_write(path.encode(), C.byref(cg)), "ecl_graph_write")

    def to_device(self, device: str = "cuda"):
        import torch

        return DeviceGraph(
            torch.from_numpy(self.nindex).to(device),
            torch.from_numpy(self.nlist).to(device) if self.edges else torch.zeros(1, dtype=torch.int32, device=device),
            torch.from_numpy(self.eweight).to(device) if self.eweight is not None else None,
            self.symmetric,
            self.edges,
        )


def _take(cg: CGraph, symmetric: bool) -> Graph:
    """Copies a library-allocated ecl_graph into numpy arrays and frees it."""
    n, m = cg.nodes, cg.edges
    try:
        nindex = np.ctypeslib.as_array(cg.nindex, shape=(n + 1,)).copy()
        nlist = np.ctypeslib.as_array(cg.nlist, shape=(m,)).copy() if m else np.zeros(0, np.int32)
        ew = np.ctypeslib.as_array(cg.eweight, shape=(m,)).copy() if (cg.eweight and m) else None
        if cg.eweight and m == 0:
            ew = np.zeros(0, np.int32)
    finally:
        lib.ecl_graph_free(C.byref(cg))
    return Graph(nindex, nlist, ew, symmetric)


def read_graph(path: str) -> Graph:
    """readECLgraph (library/ECLgraph.h:49-76), returning status instead of exiting."""
    cg = CGraph()
    _check(lib.ecl_graph_read(path.encode(), C.byref(cg)), f"ecl_graph_read({path})")
    return _take(cg, False)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 2, symmetrise: bool = True, weight_seed: int = 0, weight_max: int = 1 << 20) -> Graph:
    cg = CGraph()
    _check(lib.ecl_gen_rmat(scale, edge_factor, a, b, c, seed, int(symmetrise), weight_seed, weight_max, C.byref(cg)),
           "ecl_gen_rmat")
    return _take(cg, symmetrise)


def gen_grid(rows: int, cols: int, delete_frac: float = 0.05, seed: int = 1, weight_seed: int = 0,
             weight_max: int = 1 << 20) -> Graph:
    cg = CGraph()
    _check(lib.ecl_gen_grid(rows, cols, delete_frac, seed, weight_seed, weight_max, C.byref(cg)), "ecl_gen_grid")
    return _take(cg, True)


def gen_er(n: int, p: float, seed: int = 4, symmetrise: bool = False, weight_seed: int = 0,
           weight_min: int = 1, weight_max: int = 1000) -> Graph:
    cg = CGraph()
    _check(lib.ecl_gen_er(n, p, seed, int(symmetrise), weight_seed, weight_min, weight_max, C.byref(cg)), "ecl_gen_er")
    return _take(cg, symmetrise)


@dataclass
class DeviceGraph:
    """CSR held in torch CUDA int32 tensors (torch is only the allocator here)."""

    nindex: "object"
    nlist: "object"
    eweight: "object" = None
    symmetric: bool = False
    edges_: int = -1

    @property
    def nodes(self) -> int:
        return int(self.nindex.shape[0] - 1)

    @property
    def edges(self) -> int:
        return int(self.nlist.shape[0]) if self.edges_ < 0 else self.edges_

    def view(self) -> GraphView:
        v = GraphView()
        v.nodes, v.edges = self.nodes, self.edges
        v.nindex = self.nindex.data_ptr()
        v.nlist = self.nlist.data_ptr()
        v.eweight = self.eweight.data_ptr() if self.eweight is not None else None
        v.location = DEVICE
        v.flags = GRAPH_SYMMETRIC if self.symmetric else 0
        return v


# ---- solvers ---------------------------------------------------------------------


def _opts(stream=None, workspace=None, validate=False, max_rounds=0, detail=False) -> Opts:
    o = Opts()
    o.stream = stream
    o.detail = int(detail)
    if workspace is not None:
        o.workspace = workspace.data_ptr()
        o.workspace_bytes = workspace.numel() * workspace.element_size()
    o.validate = int(validate)
    o.max_rounds = max_rounds
    return o


def workspace_bytes(code: int, nodes: int, edges: int) -> int:
    return int(lib.ecl_workspace_bytes(code, nodes, edges))


def _out(g, n, dtype, torch_dtype):
    if isinstance(g, DeviceGraph):
        import torch

        return torch.empty(n, dtype=torch_dtype, device=g.nindex.device)
    return np.empty(n, dtype=dtype)


def _ptr(a) -> int:
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


def _run(fn, name, g, out, *extra, opts: Optional[Opts] = None, **kw):
    o = opts if opts is not None else _opts(**kw)
    v = g.view()
    _check(fn(C.byref(v), _ptr(out), *extra, C.byref(o)), name)
    return o


def cc(g, out=None, **kw):
    """label[v] = smallest id in v's component (ECL-CC-atomic.cu:275 computeCC contract)."""
    out = _out(g, g.nodes, np.int32, _torch_dtype("int32")) if out is None else out
    _run(lib.ecl_cc, "ecl_cc", g, out, **kw)
    return out


def mis(g, out=None, **kw):
    """status[v] in {0xfe, 0} (ECL-MIS-atomic.cu:147 computeMIS contract)."""
    out = _out(g, g.nodes, np.uint8, _torch_dtype("uint8")) if out is None else out
    _run(lib.ecl_mis, "ecl_mis", g, out, **kw)
    return out


def gc(g, out=None, **kw):
    """color[v] >= 0, first-fit greedy in (degree, hash, id) priority (ECL-GC-atomic.cu:333-373)."""
    out = _out(g, g.nodes, np.int32, _torch_dtype("int32")) if out is None else out
    _run(lib.ecl_gc, "ecl_gc", g, out, **kw)
    return out


def mst(g, out=None, **kw):
    """(in_mst[m] bytes, total weight) (ECL-MST_10-atomic.cu:285 gpuMST contract)."""
    out = _out(g, max(g.edges, 1), np.uint8, _torch_dtype("uint8")) if out is None else out
    total = C.c_uint64(0)
    o = _opts(**kw) if "opts" not in kw else kw.pop("opts")
    v = g.view()
    _check(lib.ecl_mst(C.byref(v), _ptr(out), C.byref(total), C.byref(o)), "ecl_mst")
    return out[: g.edges], int(total.value)


def scc(g, out=None, **kw):
    """label[v] = largest id in v's SCC (ECL-SCC_10-atomic.cu:318 readFirst(iomax[v]))."""
    out = _out(g, g.nodes, np.int32, _torch_dtype("int32")) if out is None else out
    _run(lib.ecl_scc, "ecl_scc", g, out, **kw)
    return out


def apsp(g, out=None, ld: Optional[int] = None, **kw):
    """n x ld int32 distances (ECL-APSP-atomic.cu:460 FW_gpu_64 contract, unpadded)."""
    n = g.nodes
    ld = n if ld is None else ld
    if out is None:
        if isinstance(g, DeviceGraph):
            import torch

            out = torch.empty((n, ld), dtype=torch.int32, device=g.nindex.device)
        else:
            out = np.empty((n, ld), dtype=np.int32)
    o = _opts(**kw) if "opts" not in kw else kw.pop("opts")
    v = g.view()
    _check(lib.ecl_apsp(C.byref(v), _ptr(out), ld, C.byref(o)), "ecl_apsp")
    return out


def _torch_dtype(name):
    try:
        import torch

        return getattr(torch, name)
    except ImportError:  # host-only use
        return None


def kernel_launches() -> int:
    return int(lib.ecl_kernel_launches())


def minplus_peak(variant: int = 0) -> float:
    """Measured INT32 min-plus rate of the current device, integer ops/s
    (variant 0: DPX add-min, the APSP instruction; 1: separate add and min)."""
    v = C.c_double(0.0)
    _check(lib.ecl_minplus_peak(variant, C.byref(v)), "ecl_minplus_peak")
    return float(v.value)


def hop_latency(variant: int = 0) -> float:
    """Measured ns of one dependency hop (0: L2 with GC's back-off polling,
    1: L2 with a bare spin, 2: shared memory between two warps of a CTA)."""
    v = C.c_double(0.0)
    _check(lib.ecl_hop_latency(variant, C.byref(v)), "ecl_hop_latency")
    return float(v.value)


def gather_peak(index, n: int, variant: int = 0) -> float:
    """Measured streaming-gather rate, entries/s: each of the device indices
    `index` (a CUDA int32 tensor, values in [0, n)) loads one 8-byte word of
    an L2-resident n-word table (0: read-only loads, 1: relaxed atomic loads)
    -- the roofline of a CSR scan over a graph with those column indices."""
    v = C.c_double(0.0)
    _check(lib.ecl_gather_peak(_ptr(index), int(index.numel()), n, variant, C.byref(v)), "ecl_gather_peak")
    return float(v.value)


def gc_critical_path(g: "Graph", core_ranks: int = 0, hop_core_ns: float = 0.0, hop_rest_ns: float = 0.0):
    """GC's longest dependency chain of a host graph: (hops, hops inside the
    shared-memory core, the chain's time with the given hop costs in ns)."""
    v = g.view()
    h, hc, t = C.c_int32(0), C.c_int32(0), C.c_double(0.0)
    _check(lib.ecl_gc_critical_path(C.byref(v), core_ranks, hop_core_ns, hop_rest_ns, C.byref(h), C.byref(hc),
                                    C.byref(t)), "ecl_gc_critical_path")
    return int(h.value), int(hc.value), float(t.value)


# ---- batched engine (include/ecl_batch.h) ------------------------------------------

BATCH_CC, BATCH_MIS, BATCH_GC, BATCH_MST, BATCH_SCC = 0x1, 0x2, 0x4, 0x8, 0x10


class Tune(C.Structure):
    """ecl_tune: launch knobs (0 = built-in default); they never change results."""

    _fields_ = [("blocks_per_sm", C.c_int32), ("mst_light_factor", C.c_float), ("gc_core_ranks", C.c_int32),
                ("row_lane_max", C.c_int32), ("row_chunk", C.c_int32), ("scc_sweep_batch", C.c_int32),
                ("gc_poll_ns", C.c_int32), ("row_vec", C.c_int32),
                ("gc_pull_blocks", C.c_int32), ("gc_core_ctas", C.c_int32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_sig("ecl_set_tune", C.c_int, [C.POINTER(Tune)])
_sig("ecl_get_tune", C.c_int, [C.POINTER(Tune)])


def get_tune() -> Tune:
    t = Tune()
    _check(lib.ecl_get_tune(C.byref(t)), "ecl_get_tune")
    return t


def set_tune(t: Optional[Tune] = None, **knobs) -> Tune:
    """Sets the process-wide knobs of the single-graph solvers (unnamed knobs
    keep their current values); returns the previous setting."""
    old = get_tune()
    new = Tune()
    C.memmove(C.byref(new), C.byref(t if t is not None else old), C.sizeof(Tune))
    for k, v in knobs.items():
        setattr(new, k, v)
    _check(lib.ecl_set_tune(C.byref(new)), "ecl_set_tune")
    return old


_PB = C.c_void_p
_sig("ecl_batch_create", C.c_int, [C.POINTER(C.c_void_p)])
_sig("ecl_batch_destroy", None, [_PB])
_sig("ecl_batch_add", C.c_int, [_PB, _PV])
_sig("ecl_batch_add_mix", C.c_int, [_PB, _I32, _I32, _I32, _U64, _I32])
_sig("ecl_batch_build", C.c_int, [_PB, C.c_uint32, C.c_int64, _VP])
_sig("ecl_batch_run", C.c_int, [_PB, _PO])
_sig("ecl_batch_tune", C.c_int, [_PB, _I32, C.POINTER(Tune)])
_sig("ecl_batch_set_tune", C.c_int, [_PB, C.POINTER(Tune)])
_sig("ecl_batch_tune_points", C.c_int32, [_PB])
_sig("ecl_batch_graphs", C.c_int32, [_PB])
_sig("ecl_batch_superbatches", C.c_int32, [_PB])
_sig("ecl_batch_graph_size", C.c_int, [_PB, _I32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)])
_sig("ecl_batch_graph_csr", C.c_int, [_PB, _I32, _VP, _VP, _VP])
_sig("ecl_batch_result", C.c_int, [_PB, _I32, C.c_uint32, _VP, C.POINTER(C.c_uint64)])
EXPORTED += ["ecl_batch_create", "ecl_batch_destroy", "ecl_batch_add", "ecl_batch_add_mix", "ecl_batch_build",
             "ecl_batch_run", "ecl_batch_tune", "ecl_batch_set_tune", "ecl_batch_tune_points", "ecl_batch_graphs",
             "ecl_batch_superbatches",
             "ecl_batch_graph_size", "ecl_batch_graph_csr", "ecl_batch_result"]


class Batch:
    """Many graphs solved by one set of launches (one CUDA graph replay)."""

    def __init__(self):
        h = C.c_void_p()
        _check(lib.ecl_batch_create(C.byref(h)), "ecl_batch_create")
        self.h = h

    def close(self):
        """Releases the engine's device memory now (also done on garbage collection)."""
        if getattr(self, "h", None):
            lib.ecl_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def add(self, g: Graph):
        v = g.view()
        _check(lib.ecl_batch_add(self.h, C.byref(v)), "ecl_batch_add")

    def add_mix(self, count, n_min=1000, n_max=200000, seed=5, weight_max=1 << 16):
        _check(lib.ecl_batch_add_mix(self.h, count, n_min, n_max, seed, weight_max), "ecl_batch_add_mix")

    def build(self, codes, max_entries=0, stream=None):
        _check(lib.ecl_batch_build(self.h, codes, max_entries, stream), "ecl_batch_build")

    def run(self):
        o = Opts()
        _check(lib.ecl_batch_run(self.h, C.byref(o)), "ecl_batch_run")
        return o.elapsed_ms, bool(o.rounds)

    def tune(self, trials=2) -> Tune:
        t = Tune()
        _check(lib.ecl_batch_tune(self.h, trials, C.byref(t)), "ecl_batch_tune")
        return t

    @property
    def tune_points(self) -> int:
        """Knob settings the last tune() timed."""
        return int(lib.ecl_batch_tune_points(self.h))

    @property
    def graphs(self) -> int:
        return int(lib.ecl_batch_graphs(self.h))

    @property
    def superbatches(self) -> int:
        return int(lib.ecl_batch_superbatches(self.h))

    def graph(self, i) -> Graph:
        n, m = C.c_int32(), C.c_int32()
        _check(lib.ecl_batch_graph_size(self.h, i, C.byref(n), C.byref(m)), "ecl_batch_graph_size")
        ni = np.empty(n.value + 1, np.int32)
        nl = np.empty(max(m.value, 1), np.int32)
        ew = np.empty(max(m.value, 1), np.int32)
        _check(lib.ecl_batch_graph_csr(self.h, i, ni.ctypes.data, nl.ctypes.data, ew.ctypes.data), "ecl_batch_graph_csr")
        return Graph(ni, nl[: m.value], ew[: m.value], True)

    def result(self, i, code):
        n, m = C.c_int32(), C.c_int32()
        _check(lib.ecl_batch_graph_size(self.h, i, C.byref(n), C.byref(m)), "ecl_batch_graph_size")
        if code in (BATCH_CC, BATCH_SCC, BATCH_GC):
            out = np.empty(n.value, np.int32)
        elif code == BATCH_MIS:
            out = np.empty(n.value, np.uint8)
        else:
            out = np.empty(max(m.value, 1), np.uint8)
        tot = C.c_uint64(0)
        _check(lib.ecl_batch_result(self.h, i, code, out.ctypes.data, C.byref(tot)), "ecl_batch_result")
        if code == BATCH_MST:
            return out[: m.value], int(tot.value)
        return out


# ---- server (include/ecl_server.h) ---------------------------------------------------


class ServerCfg(C.Structure):
    _fields_ = [("slots", C.c_int32), ("hbm_budget_bytes", C.c_uint64)]


class Request(C.Structure):
    _fields_ = [
        ("code", C.c_int32),
        ("graph", C.c_int32),
        ("arrival_s", C.c_double),
        ("out", C.c_void_p),
        ("total_weight", C.c_uint64),
        ("latency_s", C.c_double),
        ("queue_s", C.c_double),
        ("status", C.c_int32),
        ("slot", C.c_int32),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_int32),
        ("failed", C.c_int32),
        ("makespan_s", C.c_double),
        ("graphs_per_s", C.c_double),
        ("p50_s", C.c_double),
        ("p99_s", C.c_double),
        ("mean_s", C.c_double),
        ("max_in_flight", C.c_int32),
        ("peak_bytes", C.c_uint64),
    ]


_sig("ecl_server_create", C.c_int, [C.POINTER(ServerCfg), C.POINTER(C.c_void_p)])
_sig("ecl_server_destroy", None, [C.c_void_p])
_sig("ecl_server_add_graph", C.c_int, [C.c_void_p, _PV, C.POINTER(C.c_int32)])
_sig("ecl_server_run", C.c_int, [C.c_void_p, C.POINTER(Request), C.c_int32, C.POINTER(ServerStats)])
EXPORTED += ["ecl_server_create", "ecl_server_destroy", "ecl_server_add_graph", "ecl_server_run"]


class Server:
    """Continuous-batching server over resident graphs (see ecl_server.h).
    Result buffers should be pinned host memory so copies stay asynchronous."""

    def __init__(self, slots=8, hbm_budget_bytes=0):
        cfg = ServerCfg(slots, hbm_budget_bytes)
        h = C.c_void_p()
        _check(lib.ecl_server_create(C.byref(cfg), C.byref(h)), "ecl_server_create")
        self.h = h

    def close(self):
        """Releases the resident graphs and the server's streams now (also on garbage collection)."""
        if getattr(self, "h", None):
            lib.ecl_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def add_graph(self, g: Graph) -> int:
        gid = C.c_int32()
        v = g.view()
        _check(lib.ecl_server_add_graph(self.h, C.byref(v), C.byref(gid)), "ecl_server_add_graph")
        return int(gid.value)

    def run(self, reqs):
        """reqs: list of (code, graph_id, arrival_s, out_ptr_or_None)."""
        arr = (Request * len(reqs))()
        for k, (code, gid, t, out) in enumerate(reqs):
            arr[k].code, arr[k].graph, arr[k].arrival_s, arr[k].out = code, gid, t, out
        st = ServerStats()
        rc = lib.ecl_server_run(self.h, arr, len(reqs), C.byref(st))
        return rc, arr, st
