"""Continuous-batching server on the B200: concurrent requests over resident
graphs give exactly the result of the same solve run alone; admission
respects the HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graphs(ecl):
    gs = [
        ecl.gen_rmat(12, 16, seed=2, weight_seed=3, weight_max=1 << 20),
        ecl.gen_rmat(14, 8, seed=7, weight_seed=4, weight_max=1 << 20),
        ecl.gen_grid(60, 70, 0.05, seed=1, weight_seed=5, weight_max=1 << 20),
        ecl.gen_er(5000, 0.002, seed=4, symmetrise=True, weight_seed=6, weight_min=1, weight_max=1 << 19),
    ]
    for g in gs:
        g.symmetric = True
    return gs


def _alone(ecl, code, g):
    if code == ecl.CC:
        return ecl.cc(g)
    if code == ecl.MIS:
        return ecl.mis(g)
    if code == ecl.GC:
        return ecl.gc(g)
    if code == ecl.SCC:
        return ecl.scc(g)
    return ecl.mst(g)


def _pinned(torch, n, dtype):
    t = torch.empty(max(n, 1), dtype=dtype).pin_memory()
    return t, t.numpy()


def test_server_results_equal_alone(ecl, orc):
    import torch

    gs = _graphs(ecl)
    srv = ecl.Server(slots=6)
    ids = [srv.add_graph(g) for g in gs]
    rng = np.random.default_rng(6)
    reqs, outs, keep = [], [], []
    t = 0.0
    for k in range(60):
        code = int(rng.integers(0, 5))
        code = [ecl.CC, ecl.MIS, ecl.GC, ecl.MST, ecl.SCC][code]
        gi = int(rng.integers(0, len(gs)))
        g = gs[gi]
        n = g.edges if code == ecl.MST else g.nodes
        tt, arr = _pinned(torch, n, torch.uint8 if code in (ecl.MIS, ecl.MST) else torch.int32)
        keep.append(tt)
        t += rng.exponential(1.0 / 5000.0)  # Poisson, 5k req/s: many requests overlap
        reqs.append((code, ids[gi], t, arr.ctypes.data))
        outs.append((code, gi, arr))
    rc, arr, st = srv.run(reqs)
    assert rc == ecl.OK and st.completed == 60 and st.failed == 0
    assert st.max_in_flight > 1  # work overlapped on the device
    assert st.p99_s >= st.p50_s > 0
    for k, (code, gi, out) in enumerate(outs):
        g = gs[gi]
        assert arr[k].status == ecl.OK
        alone = _alone(ecl, code, g)
        if code == ecl.MST:
            assert np.array_equal(out[: g.edges], alone[0]) and arr[k].total_weight == alone[1], k
            assert arr[k].total_weight == orc.mst(g)[1]
        else:
            assert np.array_equal(out[: g.nodes], alone), k


def test_server_budget_admission(ecl):
    import torch

    gs = _graphs(ecl)[:2]
    big = max(ecl.workspace_bytes(c, g.nodes, g.edges) for g in gs for c in (ecl.CC, ecl.MIS, ecl.MST))
    resident = sum(4 * (g.nodes + 1) + 8 * g.edges for g in gs)
    # room for about one request at a time next to the resident graphs
    srv = ecl.Server(slots=4, hbm_budget_bytes=resident + int(1.5 * big) + (1 << 20))
    ids = [srv.add_graph(g) for g in gs]
    reqs = [(c, ids[i % 2], 0.0, None) for i, c in enumerate([ecl.CC, ecl.MIS, ecl.MST, ecl.CC, ecl.MIS, ecl.MST])]
    rc, arr, st = srv.run(reqs)
    assert rc == ecl.OK and st.completed == 6
    assert st.peak_bytes <= resident + int(1.5 * big) + (1 << 20)
    # a request that cannot fit even alone is refused, the rest still run
    tiny = ecl.Server(slots=2, hbm_budget_bytes=resident + (1 << 16))
    ids = [tiny.add_graph(g) for g in gs]
    rc, arr, st = tiny.run([(ecl.MST, ids[0], 0.0, None), (ecl.CC, ids[1], 0.0, None)])
    assert arr[0].status == ecl.ERR_OOM
