"""CLI drop-ins on the B200: they take the reference executables' argument
(one .egr file) and print the reference's stdout key lines, which the
reference harness parses with `time: +(\\d+\\.\\d+) s`."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "ecl-suite_b200", "bin")
TIME_RE = re.compile(r"time: +(\d+\.\d+) s")


def _run(tool, path):
    r = subprocess.run([os.path.join(BIN, tool), path], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_cli_tools(ecl, orc, tmp_path):
    g = ecl.gen_rmat(12, 16, seed=2, weight_seed=3)
    p = str(tmp_path / "g.egr")
    g.write(p)
    out = _run("ecl-cc", p)
    assert TIME_RE.search(out) and "verification passed" in out
    ncc = len(set(orc.cc(g).tolist()))
    assert f"number of connected components: {ncc}" in out
    out = _run("ecl-mis", p)
    assert TIME_RE.search(out) and "elements in set:" in out
    out = _run("ecl-gc", p)
    assert "runtime:" in out and "result verification passed" in out
    assert f"colors used: {int(orc.gc(g).max()) + 1}" in out
    out = _run("ecl-mst", p)
    assert re.search(r"Dev[-+]: +\d+\.\d+ s", out) and "all good" in out
    assert f"MST weight: {orc.mst(g)[1]}" in out
    d = ecl.gen_rmat(11, 8, seed=5, symmetrise=False)
    pd = str(tmp_path / "d.egr")
    d.write(pd)
    out = _run("ecl-scc", pd)
    assert TIME_RE.search(out) and f"number of SCCs: {len(set(orc.scc(d).tolist()))}" in out
    e = ecl.gen_er(300, 0.01, seed=4, weight_seed=5)
    pe = str(tmp_path / "e.egr")
    e.write(pe)
    out = _run("ecl-apsp", pe)
    assert "FW_64 gpu comp time:" in out
