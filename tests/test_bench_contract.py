"""bench.py's reference arm runs on host cores only, so its JSON contract is
checked here on the CPU: one line with impl, metric, value, unit, the CPU
baseline description and an e2e block with zero transfer bytes."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out
    return json.loads(lines[0])


def test_reference_arm_grid_line():
    d = _run("--impl", "reference", "--workload", "grid", "--steps", "1", "--warmup", "0")
    assert d["impl"] == "reference"
    assert d["unit"] == "edges/s" and d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("port", "reference") and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("grid1024")


def test_phase_tables_cover_every_phase():
    sys.path.insert(0, ROOT)
    import bench

    for code, names in bench.PHASE_NAMES.items():
        for i in range(len(names)):
            b = bench.phase_bytes(code, i, 1 << 20, 16 << 20)
            assert b is None or b > 0, (code, i)


def test_reference_arm_suite_never_loads_the_product_library():
    """The reference arm builds the R-MAT graphs with the oracle's restated
    generators and times only oracle/ code (the reference's cpuMST, the C
    restatements): the product library is neither imported nor mapped.  A
    step is one code round robin; value = one pass's edges / the sum of the
    codes' mean times."""
    code = (
        "import json, sys, argparse\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import bench\n"
        "args = bench.parse(['--impl', 'reference', '--scale', '13', '--steps', '5', '--warmup', '0',\n"
        "                    '--no-other-configs'])\n"
        "bench.run_reference(args, 0, 1)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'ecl_b200' : 'ecl_b200' in sys.modules, 'mapped': 'libeclb200' in maps}))\n"
    )
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         check=True).stdout
    lines = [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]
    line, probe = lines[0], lines[1]
    assert probe == {"ecl_b200": False, "mapped": False}
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "edges/s"
    assert line["config"]["workload"].startswith("rmat13-suite")
    cb = line["cpu_baseline"]
    assert set(cb["per_code_kind"]) == {"cc", "mis", "gc", "mst", "scc"}
    assert cb["kind"] in ("reference", "port", "mixed")
    assert cb["value"] == line["value"]
