"""The C ABI (include/fsi_b200.h): the built library loads without a GPU,
exports every declared entry point, and the ctypes mirrors of the structs
match the C layout (checked by compiling the header with gcc)."""

import ctypes
import os
import re
import subprocess

import pytest

from mpm_lbm_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fsi_b200.h")


def declared_functions():
    text = open(HEADER, encoding="utf-8").read()
    return sorted(set(re.findall(r"^(?:int|uint64_t)\s+(fsi_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported_and_bound(lib):
    names = declared_functions()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name
    assert lib.fsi_abi_version() == _lib.ABI_VERSION == 2
    # no kernel has run in this process without a GPU
    assert _lib.launch_count() == 0


def test_struct_layouts_match_c(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fsi_b200.h"', "int main(void){"]
    for sname, cls in _lib.STRUCTS.items():
        lines.append(f'printf("{sname} size %zu\\n", sizeof({sname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{sname} {fname} %zu\\n", offsetof({sname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        parts = line.split()
        sname, what, value = parts[0], parts[1], int(parts[2])
        cls = _lib.STRUCTS[sname]
        if what == "size":
            assert ctypes.sizeof(cls) == value, line
        else:
            assert getattr(cls, what).offset == value, line


def test_invalid_arguments_fail_loudly(lib):
    # a null state is rejected with a message, without touching a device
    rc = lib.fsi_lbm_substep(None, None, None, None)
    assert rc == -1
    assert "null" in _lib.last_error()


def test_header_constants_match_binding():
    text = open(HEADER, encoding="utf-8").read()

    def define(name):
        return int(re.search(rf"#define {name} (\d+)", text).group(1))

    assert define("FSI_ABI_VERSION") == _lib.ABI_VERSION
    assert define("FSI_BIN_CHUNK") == _lib.FSI_BIN_CHUNK
    assert define("FSI_BIN_EDGE") == _lib.FSI_BIN_EDGE
    assert define("FSI_CAMPAIGN_REGIONS") == _lib.FSI_CAMPAIGN_REGIONS
