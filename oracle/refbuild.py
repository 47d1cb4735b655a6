"""The reference's own build (oracle/_ref/libeclref.so) -- TEST INFRASTRUCTURE ONLY.

`make -C oracle ref` compiles the reference's race-free .cu files unchanged
(each included by an oracle/ref_*.cu harness) into one library.  This module
calls it on host CSR arrays: the reference GPU kernels of CC, MIS, GC and SCC
and the APSP FW_gpu_64 driver (they need a CUDA device; torch only provides
device memory here), and the reference CPU routines cpuMST and FW_cpu.

Only tests/, tests/golden/make_golden.py and bench.py's reference and CPU
baseline legs use it: it is the checker, never the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libeclref.so")


def available() -> bool:
    return os.path.exists(LIB_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        r = C.CDLL(LIB_PATH)
        for name, res in [("eclref_mst_cpu", C.c_double), ("eclref_mst_gpu", C.c_double),
                          ("eclref_apsp_gpu", C.c_double), ("eclref_apsp_cpu", C.c_double),
                          ("eclref_cc_device", C.c_float), ("eclref_mis_device", C.c_float),
                          ("eclref_gc_device", C.c_float), ("eclref_gc_scratch_bytes", C.c_size_t),
                          ("eclref_scc_device", C.c_float), ("eclref_scc_scratch_bytes", C.c_size_t)]:
            getattr(r, name).restype = res
        _lib = r
    return _lib


def _host(a):
    return C.c_void_p(np.ascontiguousarray(a).ctypes.data)


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _dp(t):
    return C.c_void_p(t.data_ptr())


def _nlist(g):
    return g.nlist if g.edges else np.zeros(1, np.int32)


def cc(g) -> np.ndarray:
    """nstat of the reference CC kernels (ECL-CC-atomic.cu computeCC's timed region)."""
    import torch

    ni, nl = _dev(g.nindex), _dev(_nlist(g))
    st = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    wl = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    lib().eclref_cc_device(g.nodes, _dp(ni), _dp(nl), _dp(st), _dp(wl))
    return st.cpu().numpy()


def mis(g) -> np.ndarray:
    """Status bytes of the reference MIS kernels (0xfe in, 0 out)."""
    import torch

    ni, nl = _dev(g.nindex), _dev(_nlist(g))
    st = torch.empty((g.nodes + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    lib().eclref_mis_device(g.nodes, g.edges, _dp(ni), _dp(nl), _dp(st))
    return st.cpu().numpy()[: g.nodes]


def gc(g) -> np.ndarray:
    """Colours of the reference GC kernels (init, runLarge, runSmall)."""
    import torch

    ni, nl = _dev(g.nindex), _dev(_nlist(g))
    col = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    scr = torch.empty(lib().eclref_gc_scratch_bytes(g.nodes, g.edges) // 4 + 1, dtype=torch.int32, device="cuda")
    lib().eclref_gc_device(g.nodes, g.edges, _dp(ni), _dp(nl), _dp(col), _dp(scr))
    return col.cpu().numpy()


def scc(g) -> np.ndarray:
    """Labels of the reference SCC kernels (readFirst of iomax, the largest id of the SCC)."""
    import torch

    ni, nl = _dev(g.nindex), _dev(_nlist(g))
    scr = torch.empty(lib().eclref_scc_scratch_bytes(g.nodes, g.edges) // 8 + 2, dtype=torch.int64, device="cuda")
    lab = np.empty(g.nodes, np.int32)
    lib().eclref_scc_device(g.nodes, g.edges, _dp(ni), _dp(nl), C.c_void_p(lab.ctypes.data), _dp(scr))
    return lab


def mst_cpu(g):
    """(in_mst bytes, total weight) of the reference's serial cpuMST (ECL-MST_10-atomic.cu:112)."""
    out = np.zeros(max(g.edges, 1), np.uint8)
    lib().eclref_mst_cpu(g.nodes, g.edges, _host(g.nindex), _host(g.nlist), _host(g.eweight),
                         C.c_void_p(out.ctypes.data))
    out = out[: g.edges]
    return out, int(g.eweight[out.astype(bool)].astype(np.int64).sum()) if g.edges else 0


def apsp_gpu(g) -> np.ndarray:
    """The padded upper x upper matrix (upper = ceil(n/64)*64) of the reference FW_gpu_64."""
    upper = (g.nodes + 63) // 64 * 64
    out = np.zeros((upper, upper), np.int32)
    lib().eclref_apsp_gpu(g.nodes, g.edges, _host(g.nindex), _host(g.nlist), _host(g.eweight),
                          C.c_void_p(out.ctypes.data))
    return out


def apsp_cpu(g) -> np.ndarray:
    """The n x n closure of the reference's serial FW_cpu (ECL-APSP-atomic.cu:533)."""
    out = np.zeros((g.nodes, g.nodes), np.int32)
    lib().eclref_apsp_cpu(g.nodes, g.edges, _host(g.nindex), _host(g.nlist), _host(g.eweight),
                          C.c_void_p(out.ctypes.data))
    return out
