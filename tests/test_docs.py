"""Documentation kept in step with the code (no GPU): every environment variable the library reads
is listed in INTEGRATION.md's table, and every entry point the C header declares is named in
INTEGRATION.md or DESIGN.md."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "nndex_b200", "csrc")


def _read(*parts):
    with open(os.path.join(ROOT, *parts), encoding="utf-8") as f:
        return f.read()


def test_every_environment_variable_is_documented():
    used = set()
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".h")):
            used |= set(re.findall(r'(?:getenv|env_u32)\("(NNDEX_[A-Z0-9_]+)"\)', _read("nndex_b200", "csrc", name)))
    assert used, "no environment variables found (the pattern is stale)"
    doc = _read("INTEGRATION.md")
    missing = sorted(v for v in used if v not in doc)
    assert not missing, f"not in INTEGRATION.md: {missing}"


def test_every_declared_entry_point_is_documented():
    header = _read("include", "nndex_cuda.h")
    declared = set(re.findall(r"NNDEX_API\s+[\w\s\*]+?\b(nndex_cuda_\w+)\s*\(", header))
    assert declared
    docs = _read("INTEGRATION.md") + _read("DESIGN.md") + header
    # each declaration carries its own comment in the header; the integration notes or the design
    # must name every function a wrapper would bind, except the diagnostics the header marks as such
    missing = sorted(f for f in declared if docs.count(f) < 2)
    assert not missing, f"named only once (the declaration): {missing}"
