"""The SORT-side adapter (sort_b200/integration/gbvh.h) against SORT's headers.

The adapter is compiled into oracle/_ref/libsortref_gbvh.so with SORT's own
sources by oracle/Makefile, and tests/test_gpu_sort_adapter.py runs it inside
SORT's code on the GPU. Here (no GPU): the header compiles against SORT's
headers on its own, and it calls only entry points include/sortgpu.h declares.
Where SORT's sources were found is recorded by that build (oracle/_ref/ref_src);
the compile check is skipped where it did not run.
"""
import os
import re
import subprocess

import pytest

from conftest import ROOT

ADAPTER = os.path.join(ROOT, "sort_b200", "integration", "gbvh.h")
REF_SRC_RECORD = os.path.join(ROOT, "oracle", "_ref", "ref_src")


def _ref_src():
    if not os.path.exists(REF_SRC_RECORD):
        return None
    path = open(REF_SRC_RECORD).read().strip()
    return path if os.path.isdir(path) else None


@pytest.mark.skipif(_ref_src() is None, reason="SORT sources not recorded by an oracle build")
def test_adapter_compiles_against_sort_headers(tmp_path):
    f = tmp_path / "gbvh_check.cpp"
    # SORT keeps the shape fields the adapter reads protected or private; a SORT
    # build grants access with friend declarations, this check by opening them.
    f.write_text("#define private public\n#define protected public\n#include \"core/scene.h\"\n"
                 "#include \"shape/line.h\"\n#include \"shape/quad.h\"\n#include \"shape/disk.h\"\n"
                 "#undef private\n#undef protected\n#include \"gbvh.h\"\n"
                 "int main() { Gbvh g(8, 16, 8); (void)g; return 0; }\n")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", "-msse4.1", "-mavx", "-DSIMD_4WAY_ENABLED",
           "-DSIMD_8WAY_ENABLED", "-DSORT_RELEASE", "-I" + os.path.join(ROOT, "oracle", "ref", "tsl_stub"),
           "-I" + os.path.join(ROOT, "oracle", "_ref", "generated_src"), "-I" + _ref_src(),
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.dirname(ADAPTER), str(f)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_adapter_uses_only_declared_entry_points():
    from test_abi import declared_functions
    used = set(re.findall(r"\b(sg_[a-z_0-9]+)\s*\(", open(ADAPTER).read()))
    assert used and used <= set(declared_functions())
