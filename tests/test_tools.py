"""Host tooling: the MatrixMarket converter (against the reference's own
converter, compiled from its source, when it is built) and the .egr
generator CLI (CPU only)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

BIN = os.path.join(ROOT, "ecl-suite_b200", "bin")
REF_MM = os.path.join(ROOT, "oracle", "_ref", "mm2ecl")

MM_FILES = {
    "pattern_general.mtx": "%%MatrixMarket matrix coordinate pattern general\n% c\n5 5 6\n1 2\n2 1\n5 3\n3 5\n1 4\n4 1\n",
    "int_symmetric.mtx": "%%MatrixMarket matrix coordinate integer symmetric\n4 4 3\n2 1 7\n3 1 9\n4 4 2\n",
    "real_gaps.mtx": "%%MatrixMarket matrix coordinate real general\n%% x\n6 6 4\n6 1 0.25\n1 6 1.5\n1 2 3.999\n3 1 -2.5\n",
}


def _write(tmp_path):
    paths = {}
    for name, text in MM_FILES.items():
        p = tmp_path / name
        p.write_text(text)
        paths[name] = str(p)
    return paths


def test_mm_reader_semantics(ecl, tmp_path):
    paths = _write(tmp_path)
    out = str(tmp_path / "o.egr")
    subprocess.run([os.path.join(BIN, "mm2egr"), paths["real_gaps.mtx"], out], check=True, capture_output=True)
    g = ecl.read_graph(out)
    assert g.nodes == 6 and g.edges == 4
    assert list(g.nindex) == [0, 2, 2, 3, 3, 3, 4]  # empty rows keep the running offset
    assert list(g.nlist) == [1, 5, 0, 0]
    assert list(g.eweight) == [399, 150, -250, 25]  # (int)(w * 100)
    # a "symmetric" file is not mirrored unless asked
    subprocess.run([os.path.join(BIN, "mm2egr"), paths["int_symmetric.mtx"], out], check=True, capture_output=True)
    assert ecl.read_graph(out).edges == 3
    subprocess.run([os.path.join(BIN, "mm2egr"), paths["int_symmetric.mtx"], out, "--symmetrise"], check=True,
                   capture_output=True)
    s = ecl.read_graph(out)
    assert s.edges == 5 and s.validate(symmetric=True)


@pytest.mark.skipif(not os.path.exists(REF_MM), reason="reference converter not built (make -C oracle ref)")
def test_mm_converter_byte_identical_to_reference(tmp_path):
    paths = _write(tmp_path)
    for name, p in paths.items():
        ours, ref = str(tmp_path / (name + ".ours.egr")), str(tmp_path / (name + ".ref.egr"))
        subprocess.run([os.path.join(BIN, "mm2egr"), p, ours], check=True, capture_output=True)
        subprocess.run([REF_MM, p, ref], check=True, capture_output=True)
        assert open(ours, "rb").read() == open(ref, "rb").read(), name


def test_egr_gen_cli_matches_library(ecl, tmp_path):
    out = str(tmp_path / "r.egr")
    subprocess.run([os.path.join(BIN, "egr-gen"), "rmat", "10", "8", "2", "1", "3", out], check=True,
                   capture_output=True)
    g = ecl.read_graph(out)
    h = ecl.gen_rmat(10, 8, seed=2, weight_seed=3, weight_max=1 << 20)
    assert np.array_equal(g.nlist, h.nlist) and np.array_equal(g.eweight, h.eweight)
