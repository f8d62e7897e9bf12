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
    assert lib.pb_abi_version() == L.ABI_VERSION == 6


STRUCTS = {
    "pb_layers": L.PbLayers, "pb_lut": L.PbLut, "pb_beam": L.PbBeam, "pb_rows": L.PbRows,
    "pb_segments": L.PbSegments, "pb_tallies": L.PbTallies, "pb_transport_args": L.PbTransportArgs,
    "pb_cxr_tables": L.PbCxrTables, "pb_cxr_args": L.PbCxrArgs, "pb_brem_args": L.PbBremArgs,
    "pb_coherent_args": L.PbCoherentArgs, "pb_coherent_records_args": L.PbCoherentRecordsArgs,
    "pb_decoherence_args": L.PbDecoherenceArgs, "pb_elsepa": L.PbElsepa, "pb_stopping": L.PbStopping,
    "pb_transport_score_args": L.PbTransportScoreArgs, "pb_coherent_stream_args": L.PbCoherentStreamArgs, "pb_coherent_blend_args": L.PbCoherentBlendArgs,
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


def _filled_cxr_args():
    """A bin-mean pb_cxr_args whose pointers are all set (to addresses that are
    never dereferenced: every call below fails in its host checks)."""
    c = L.PbCxrArgs()
    c.n_seg, c.n_dir, c.n_E = 16, 1, 8
    c.precision, c.quadrature = L.PB_MIXED, L.PB_QUAD_BINMEAN
    fake = 0x1000
    for f in ("n_hat", "r_mid", "v_hat", "L", "E_keV", "elec_id", "edges", "spec", "E_grid"):
        setattr(c, f, fake)
    t = c.tables
    t.n_g, t.n_tab, t.n_mu = 4, 8, 1
    for f in ("G", "ES", "EP", "WM", "row_table", "E_tab", "chi_re", "chi_im", "u_re", "u_im", "log_mu", "delta"):
        setattr(t, f, fake)
    c.tables = t
    return c


@pytest.mark.parametrize("entry", ["pb_cxr_score", "pb_cxr_score_noalloc"])
def test_cxr_entry_points_share_their_argument_checks(entry):
    """Both scorer entry points refuse, before any launch, a line buffer
    without its count (the kernel would add to a NULL counter) and a layered
    absorber without its tables, with the same code and a message naming
    the entry point."""
    lib = L.load()
    fn = getattr(lib, entry)
    c = _filled_cxr_args()
    c.line_E = 0x2000  # line_count left NULL
    assert fn(C.byref(c), None) == L.PB_ERR_INVALID
    msg = lib.pb_last_error()
    assert entry.encode() in msg and b"line buffer" in msg
    c = _filled_cxr_args()
    c.n_layer = 2  # no bounds, no mu tables
    assert fn(C.byref(c), None) == L.PB_ERR_INVALID
    assert b"layered" in lib.pb_last_error()
    c = _filled_cxr_args()
    c.n_layer = 5
    assert fn(C.byref(c), None) == L.PB_ERR_UNSUPPORTED
    c = _filled_cxr_args()
    c.precision = 7
    assert fn(C.byref(c), None) == L.PB_ERR_INVALID


def test_noalloc_far_field_capacity_is_checked_before_any_cuda_call():
    lib = L.load()
    c = _filled_cxr_args()
    c.exact_widths, c.far_pad = 64.0, 10
    c.n_dir, c.n_E = 64, 4096  # 64 * (4096 + 20) * 3 moments > 262144
    assert lib.pb_cxr_score_noalloc(C.byref(c), None) == L.PB_ERR_CAPACITY
    assert b"262144" in lib.pb_last_error()


def test_coherent_work_size_at_the_largest_accepted_sizes():
    """The field kernel's grid stays within 2^31 - 1 x-blocks for every size
    the entry points accept (items <= n_row + 1776)."""
    lib = L.load()
    nb = C.c_uint64()
    assert lib.pb_coherent_work_size(1 << 24, 1 << 40, 1 << 24, C.byref(nb)) == 0
    assert lib.pb_coherent_work_size(1 << 24, 1 << 40, 1, C.byref(nb)) == 0
    assert lib.pb_coherent_work_size((1 << 24) + 1, 10, 10, C.byref(nb)) == L.PB_ERR_INVALID


def test_blend_and_decoherence_checks_without_a_device():
    """The blend needs its electron ids and row factors, the decoherence
    factor its population; both refuse before any CUDA call."""
    lib = L.load()
    nb = C.c_uint64()
    assert lib.pb_coherent_blend_work_size(4, 1000, 64, C.byref(nb)) == 0
    plain = C.c_uint64()
    assert lib.pb_coherent_work_size(4, 1000, 64, C.byref(plain)) == 0
    assert nb.value > plain.value
    b = L.PbCoherentBlendArgs()
    a = b.base
    a.n_row, a.n_E, a.n_line = 4, 64, 1000
    fake = 0x1000
    for f in ("row_off", "row_weight", "E", "delta_omega", "spec") + tuple(
            n for n, _ in L.PbCoherentArgs._fields_[7:20]):
        setattr(a, f, fake)
    a.work, a.work_bytes = 0x100000, nb.value
    b.base = a
    assert lib.pb_coherent_blend(C.byref(b), None) == L.PB_ERR_INVALID
    assert b"elec_id and F_row" in lib.pb_last_error()
    a.work_bytes = plain.value
    b.base = a
    b.elec_id, b.F_row = fake, fake
    assert lib.pb_coherent_blend(C.byref(b), None) == L.PB_ERR_CAPACITY
    d = L.PbDecoherenceArgs()
    d.n_row, d.n_pop, d.n_E = 3, 0, 16
    assert lib.pb_decoherence_factor(C.byref(d), None) == L.PB_ERR_INVALID
    d.n_pop = 8
    assert lib.pb_decoherence_factor(C.byref(d), None) == L.PB_ERR_INVALID
    assert b"must be set" in lib.pb_last_error()


def _filled_brem_args(precision=None):
    """A single-slab pb_brem_args with every pointer set (never dereferenced:
    the calls below stop in the host checks)."""
    b = L.PbBremArgs()
    b.precision = L.PB_MIXED if precision is None else precision
    b.n_dir, b.n_seg, b.n_el, b.n_E, b.Ne = 16, 1000, 1, 2048, 1 << 20
    b.thickness = 5e6
    fake = 0x1000
    for f in ("n_hat", "r_mid", "v_hat", "L", "E_keV", "elec_id", "Z", "n_ang3", "E_grid", "mu", "spec"):
        setattr(b, f, fake)
    return b


def test_brem_work_size_and_workspace_checks_without_a_device():
    lib = L.load()
    nb = C.c_int64(-1)
    b = _filled_brem_args()
    assert lib.pb_brem_work_size(C.byref(b), C.byref(nb)) == 0
    need = nb.value
    assert need > 0  # mixed, single slab, one element: the depth-node form applies
    # the workspace grows with the segment capacity (the left-out list)
    b.n_seg = 100_000
    nb2 = C.c_int64(0)
    assert lib.pb_brem_work_size(C.byref(b), C.byref(nb2)) == 0 and nb2.value > need
    for prec, layers, n_el in ((L.PB_FP64, 0, 1), (L.PB_MIXED, 2, 1), (L.PB_MIXED, 0, 3)):
        c = _filled_brem_args(prec)
        c.n_layer, c.n_el = layers, n_el
        z = C.c_int64(-1)
        assert lib.pb_brem_work_size(C.byref(c), C.byref(z)) == 0
        assert z.value == 0, (prec, layers, n_el)  # the form does not apply: no workspace
    # a workspace below the size, or misaligned, is refused before any launch
    b = _filled_brem_args()
    b.work, b.work_bytes = 0x2000, need - 8
    assert lib.pb_brem_score(C.byref(b), None) == 1
    assert b"work_bytes" in lib.pb_last_error()
    b.work, b.work_bytes = 0x2008, need
    assert lib.pb_brem_score(C.byref(b), None) == 1
    assert b"aligned" in lib.pb_last_error()


def test_copy_segments_checks_without_a_device():
    lib = L.load()
    assert lib.pb_copy_segments(-1, None, None) == 1
    assert lib.pb_copy_segments(3, None, None) == 1
    assert lib.pb_copy_segments(0, None, None) == 0  # nothing to copy: no launch
