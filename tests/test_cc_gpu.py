"""CC on the B200 vs the oracle: bit-exact labels (ECL-CC-atomic.cu contract)."""
import numpy as np
import pytest

from conftest import from_edges, undirected

pytestmark = pytest.mark.gpu


def cases(ecl):
    yield "single", ecl.Graph(np.array([0, 0], np.int32), np.array([], np.int32))
    yield "pair", undirected(2, [(0, 1)])
    yield "path", undirected(6, [(i, i + 1) for i in range(5)])
    yield "star", undirected(200, [(0, i) for i in range(1, 200)])
    yield "isolated", undirected(10, [(3, 7)])
    yield "clique", undirected(40, [(i, j) for i in range(40) for j in range(i + 1, 40)])
    yield "asymmetric", from_edges(6, [(2, 0), (1, 3), (5, 4), (4, 1)])
    yield "selfloop", from_edges(3, [(0, 0), (1, 0), (0, 1), (2, 2)])
    yield "grid", ecl.gen_grid(64, 64, 0.05, seed=1)
    yield "grid_sparse", ecl.gen_grid(48, 80, 0.45, seed=3)
    yield "rmat12", ecl.gen_rmat(12, 16, seed=2)
    yield "rmat14", ecl.gen_rmat(14, 8, seed=5)
    # hub with > 2048 entries exercises the chunk path
    yield "hub", undirected(6000, [(5999, i) for i in range(5999)] + [(i, i + 1) for i in range(0, 100, 2)])
    yield "directed_rmat", ecl.gen_rmat(12, 8, seed=9, symmetrise=False)


def test_cc_matches_oracle_host(ecl, orc):
    for name, g in cases(ecl):
        got = ecl.cc(g)
        exp = orc.cc(g)
        assert np.array_equal(got, exp), name


def test_cc_device_resident_and_workspace(ecl, orc):
    import torch

    g = ecl.gen_rmat(13, 16, seed=2)
    dg = g.to_device()
    ws = torch.empty(ecl.workspace_bytes(ecl.CC, g.nodes, g.edges), dtype=torch.uint8, device="cuda")
    for _ in range(2):  # workspace reuse across calls
        out = ecl.cc(dg, workspace=ws)
        assert np.array_equal(out.cpu().numpy(), orc.cc(g))


def test_cc_full_grid_config(ecl, orc):
    """Config: 1024x1024 grid, 5% deleted (seed 1): labels bit-exact, self-check passes."""
    g = ecl.gen_grid(1024, 1024, 0.05, seed=1)
    got = ecl.cc(g)
    assert np.array_equal(got, orc.cc(g))
    assert orc.verify_cc(g, got) == 0


def test_cc_validate_rejects_bad_graph(ecl):
    g = ecl.Graph(np.array([0, 1, 1], np.int32), np.array([7], np.int32))
    with pytest.raises(ecl.EclError) as e:
        ecl.cc(g, validate=True)
    assert e.value.status == ecl.ERR_BAD_GRAPH
