"""The ABI structs as a C compiler lays them out (include/icflow_b200.h) against
the ctypes mirrors the tests use (icflow_b200/_lib.py) and the C# mirrors a
maintainer adds: every field's offset and every struct's size.

gcc compiles a probe that prints sizeof/offsetof for each field; the C# structs
are read from INTEGRATION.md and must list the same fields, in the same order,
with the same types (LayoutKind.Sequential then gives the C offsets on x64)."""
from __future__ import annotations

import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from icflow_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
STRUCTS = {"icf_params": _lib.icf_params, "icf_counts": _lib.icf_counts,
           "icf_device_buffers": _lib.icf_device_buffers, "icf_kernel_times": _lib.icf_kernel_times,
           "icf_tune_report": _lib.icf_tune_report}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    d = tmp_path_factory.mktemp("abi")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "icflow_b200.h"', "int main(void) {"]
    for sname, cls in STRUCTS.items():
        lines.append(f'  printf("{sname} sizeof %zu\\n", sizeof({sname}));')
        for f in cls._fields_:
            lines.append(f'  printf("{sname} {f[0]} %zu\\n", offsetof({sname}, {f[0]}));')
    lines.append("  return 0; }")
    (d / "probe.c").write_text("\n".join(lines))
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(d / "probe.c"), "-o", str(d / "probe")], check=True)
    out = subprocess.run([str(d / "probe")], check=True, capture_output=True, text=True).stdout
    res = {}
    for ln in out.splitlines():
        s, f, v = ln.split()
        res[(s, f)] = int(v)
    return res


@pytest.mark.parametrize("sname", list(STRUCTS))
def test_ctypes_mirror_matches_c(c_layout, sname):
    cls = STRUCTS[sname]
    assert C.sizeof(cls) == c_layout[(sname, "sizeof")], sname
    for f in cls._fields_:
        assert getattr(cls, f[0]).offset == c_layout[(sname, f[0])], (sname, f[0])


def _csharp_fields(struct: str):
    text = (ROOT / "INTEGRATION.md").read_text()
    m = re.search(r"struct " + struct + r"\s*\{(.*?)\n\}", text, re.S)
    assert m, struct
    fields = []
    for ln in m.group(1).splitlines():
        ln = ln.split("//")[0].strip()
        if not ln.startswith(("public", "[MarshalAs")):
            continue
        size = re.search(r"SizeConst = (\d+)", ln)
        decl = re.search(r"public (\w+)(\[\])? (.*);", ln)
        typ = decl.group(1)
        for name in decl.group(3).split(","):
            fields.append((name.strip(), typ, int(size.group(1)) if size else 1))
    return fields


@pytest.mark.parametrize("struct,cls", [("IcfParams", _lib.icf_params), ("IcfCounts", _lib.icf_counts)])
def test_csharp_mirror_lists_the_c_fields(struct, cls):
    cs = _csharp_fields(struct)
    want = []
    for name, ct in cls._fields_:
        n = getattr(ct, "_length_", 1)
        base = ct._type_ if hasattr(ct, "_length_") else ct
        typ = "double" if base is C.c_double else "int"
        want.append((name, typ, n))
    assert cs == want
