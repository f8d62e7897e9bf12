"""The C ABI: the shared library loads, exports every declared symbol, and the
ctypes structures have the layout the header gives them (checked against a
C compiler). No compute call is made, so this runs without a GPU."""

import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT
from pyrite_b200 import _lib as L

HEADER = ROOT / "include" / "pyrite_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*\**\s*(pb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_functions()
    assert set(names) == set(L.EXPORTS)
    for name in names:
        assert hasattr(lib, name), name
    assert lib.pb_abi_version() == L.ABI_VERSION == 3


STRUCTS = {
    "pb_layers": L.PbLayers, "pb_lut": L.PbLut, "pb_beam": L.PbBeam, "pb_rows": L.PbRows,
    "pb_segments": L.PbSegments, "pb_tallies": L.PbTallies, "pb_transport_args": L.PbTransportArgs,
    "pb_cxr_tables": L.PbCxrTables, "pb_cxr_args": L.PbCxrArgs, "pb_brem_args": L.PbBremArgs,
    "pb_coherent_args": L.PbCoherentArgs,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_layout_matches_header(tmp_path: Path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for name, cls in STRUCTS.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for field, _t in cls._fields_:
            lines.append(f'printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    for name, cls in STRUCTS.items():
        assert int(got[name]) == C.sizeof(cls), name
        for field, _t in cls._fields_:
            assert int(got[f"{name}.{field}"]) == getattr(cls, field).offset, f"{name}.{field}"


def test_errors_are_reported_without_a_device():
    lib = L.load()
    a = L.PbTransportArgs()
    a.n = -1
    assert lib.pb_transport(C.byref(a), None) == 1
    assert b"n = -1" in lib.pb_last_error()
    c = L.PbCxrArgs()
    c.n_dir = 0
    assert lib.pb_cxr_score(C.byref(c), None) == 1
