"""Golden fixtures made by the reference itself (tests/golden/make_golden.py):
the oracle must reproduce every one (CPU), and so must the B200 library (GPU)."""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load(path):
    import ecl_b200 as ecl

    z = np.load(path)
    g = ecl.Graph(z["nindex"], z["nlist"], z["eweight"] if "eweight" in z else None, False)
    return str(z["code"]), g, z


def test_fixtures_present():
    codes = {str(np.load(p)["code"]) for p in FIXTURES}
    assert codes == {"cc", "mis", "gc", "mst", "scc", "apsp"}, codes


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_reference_fixture(path, orc):
    code, g, z = load(path)
    if code == "mst":
        inm, tot = orc.mst(g)
        assert np.array_equal(inm, z["in_mst"]) and tot == int(z["total"])
    else:
        assert np.array_equal(getattr(orc, code)(g), z["expected"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_library_matches_reference_fixture(path, ecl):
    code, g, z = load(path)
    if code == "mst":
        inm, tot = ecl.mst(g)
        assert np.array_equal(inm, z["in_mst"]) and tot == int(z["total"])
    else:
        assert np.array_equal(getattr(ecl, code)(g), z["expected"])
