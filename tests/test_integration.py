"""The SORT-side adapter in INTEGRATION.md compiles against SORT's own headers.

Skipped where SORT's sources are absent (they are not shipped with this
repository). The adapter is compiled, not run: SORT's scene loader needs
libraries this repository does not have.
"""
import os
import re
import subprocess

import pytest

from conftest import ROOT

REF_SRC = "/root/reference/src"


def adapter_source():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    src = [b for b in blocks if "class Gbvh" in b]
    assert len(src) == 1
    return src[0]


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="SORT sources not present")
def test_adapter_compiles_against_sort_headers(tmp_path):
    f = tmp_path / "gbvh_check.cpp"
    f.write_text(adapter_source() + "\nint main() { Gbvh g; (void)g; return 0; }\n")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", "-msse4.1", "-DSIMD_4WAY_ENABLED", "-DSORT_RELEASE",
           "-I" + os.path.join(ROOT, "oracle", "ref", "tsl_stub"), "-I" + REF_SRC,
           "-I" + os.path.join(ROOT, "include"), str(f)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_adapter_uses_only_declared_entry_points():
    from test_abi import declared_functions
    used = set(re.findall(r"\b(sg_[a-z_0-9]+)\s*\(", adapter_source()))
    assert used and used <= set(declared_functions())
