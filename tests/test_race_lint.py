"""Race-freedom lint of the kernels (CPU only).

The reference removes data races by routing every access to state that other
threads may write concurrently through atomic loads and stores
(library/ECLatomic.h:45-55).  The library keeps that rule with explicit
cuda::atomic_ref operations (csrc/common.cuh: ld, st, cas, fetch_*, and the
block-scope bref of GC's shared-memory core).  This test reads every kernel
source and flags each access to a solver-state array -- the arrays that
threads of one launch share -- that is neither such an atomic operation nor
an address taken for one, unless a `race-free:` comment on the line (or just
above it) says why the plain access cannot race: a thread-owned write with no
reader in that launch, or a read of an array no thread of that launch
writes.
"""
import os
import re

from conftest import ROOT

CSRC = os.path.join(ROOT, "ecl-suite_b200", "csrc")

# solver-state arrays per source file
SHARED = {
    "cc.cu": ["parent"],
    "mis.cu": ["st4"],
    "gc.cu": ["color", "hc", "col_s"],
    "mst.cu": ["parent", "minv", "mcur", "mprev", "in_mst"],
    "scc.cu": ["io", "flags", "label"],
    "batch.cu": ["in_mst"],
}

# an access inside one of these is atomic (or only takes the address)
ATOMIC = re.compile(
    r"(\b(ld|st|cas|fetch_add|fetch_min|fetch_max|fetch_or|fetch_and|ld_acquire|st_release|io_raise<(true|false)>)"
    r"\(\s*(reinterpret_cast<[^>]*>\()?\s*&\s*$)|(\bbref\(\*?(const_cast<[^>]*>\()?&?\s*$)|(&\s*$)"
)


def code_lines(text):
    """Source lines with comments blanked (line numbers kept)."""
    text = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), text, flags=re.S)
    return [re.sub(r"//.*", "", ln) for ln in text.split("\n")]


def plain_accesses(path, names):
    raw = open(path).read().split("\n")
    code = code_lines(open(path).read())
    found = []
    for i, ln in enumerate(code):
        for name in names:
            for m in re.finditer(r"(?<![\w.>])" + re.escape(name) + r"\s*\[", ln):
                if ATOMIC.search(ln[: m.start()]):
                    continue
                context = "\n".join(raw[max(0, i - 3): i + 1])
                if "race-free:" in context:
                    continue
                found.append(f"{os.path.basename(path)}:{i + 1}: {raw[i].strip()}")
    return found


def test_every_shared_state_access_is_atomic_or_justified():
    bad = []
    for fname, names in SHARED.items():
        bad += plain_accesses(os.path.join(CSRC, fname), names)
    assert not bad, "plain accesses to shared solver state:\n" + "\n".join(bad)


def test_the_lint_catches_a_plain_access(tmp_path):
    """A plain read-modify-write of shared state without a justification is
    reported; the same access through the atomic wrapper is not."""
    src = tmp_path / "k.cu"
    src.write_text(
        "__global__ void k(int* parent, int v) {\n"
        "  parent[v] = parent[v] + 1;\n"
        "  st(&parent[v], ld(&parent[v]) + 1);\n"
        "}\n"
    )
    bad = plain_accesses(str(src), ["parent"])
    assert len(bad) == 2 and all(":2:" in b for b in bad)
