import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "ecl-suite_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ecl():
    import ecl_b200

    return ecl_b200


@pytest.fixture(scope="session")
def orc():
    import oracle

    return oracle


@pytest.fixture(scope="session", autouse=True)
def _gpu_guard(request):
    yield


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this container")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def from_edges(n, edges, weights=None, symmetric=False):
    """CSR from an explicit (u, v) list, keeping the given entry order per row."""
    import ecl_b200

    rows = [[] for _ in range(n)]
    wrows = [[] for _ in range(n)]
    for k, (u, v) in enumerate(edges):
        rows[u].append(v)
        wrows[u].append(weights[k] if weights is not None else 0)
    nindex = np.zeros(n + 1, np.int32)
    for v in range(n):
        nindex[v + 1] = nindex[v] + len(rows[v])
    nlist = np.array([x for r in rows for x in r], dtype=np.int32)
    ew = np.array([x for r in wrows for x in r], dtype=np.int32) if weights is not None else None
    return ecl_b200.Graph(nindex, nlist, ew, symmetric)


def undirected(n, pairs, weights=None):
    """Symmetric CSR; weights given per pair are mirrored."""
    e, w = [], []
    for k, (u, v) in enumerate(pairs):
        e.append((u, v))
        e.append((v, u))
        if weights is not None:
            w += [weights[k], weights[k]]
    order = sorted(range(len(e)), key=lambda i: e[i])
    e = [e[i] for i in order]
    w = [w[i] for i in order] if weights is not None else None
    return from_edges(n, e, w, symmetric=True)


def overlapping_rows(n=63, m=4096, seed=7):
    """A CSR whose rows overlap: every even row is [0, m) and every odd row is
    [m, 0).  The odd rows are malformed (end < beg); the even rows together ask
    for far more long-row chunk records than a CSR of m entries can need.  Every
    entry is a valid vertex id, so nothing reads outside the arrays."""
    import ecl_b200

    rng = np.random.default_rng(seed)
    nindex = np.array([0 if v % 2 == 0 else m for v in range(n + 1)], np.int32)
    nlist = rng.integers(0, n, size=m).astype(np.int32)
    w = rng.integers(1, 1000, size=m).astype(np.int32)
    return ecl_b200.Graph(nindex, nlist, w, symmetric=True)
