"""CPU-only checks of the C ABI library: it loads without a GPU, exports every
function include/*.h declares, parses BoundaryConditions.txt like the
reference, builds the reference's boundary wiring, and rejects bad cases with
status codes (no device call needed)."""
import ctypes as C
import glob
import json
import os
import re

import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import ACP_ERR_INVALID, ACP_ERR_UNSUPPORTED, ACP_OK, CaseDesc, default_case
from acpulse_vclbm_b200.config import read_case_file, write_case_file

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(acp_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_function():
    lib = engine.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.acp_abi_version() == 1


def test_struct_size_matches_library():
    # the library fills the whole struct: a size mismatch would corrupt the sentinel
    buf = (C.c_ubyte * (C.sizeof(CaseDesc) + 16))()
    for i in range(len(buf)):
        buf[i] = 0xAB
    engine.lib().acp_default_case(C.cast(buf, C.POINTER(CaseDesc)))
    assert all(b == 0xAB for b in bytes(buf)[C.sizeof(CaseDesc):])
    d = C.cast(buf, C.POINTER(CaseDesc)).contents
    ref = default_case()
    assert (d.nx, d.ny, d.nz, d.op, d.eq_order) == (ref.nx, ref.ny, ref.nz, ref.op, ref.eq_order)


GOLD = json.load(open(os.path.join(HERE, "golden", "single_level.json")))


@pytest.mark.parametrize("c", GOLD["cases"][:12], ids=[c["name"] for c in GOLD["cases"][:12]])
def test_c_parser_matches_python_parser(c, tmp_path):
    p = tmp_path / "bc.txt"
    p.write_text(c["case_file"])
    a = engine.parse_case_file(str(p))
    b = read_case_file(str(p))
    assert bytes(a) == bytes(b)


def test_parser_reference_rules(tmp_path):
    d = default_case()
    p = tmp_path / "bc.txt"
    write_case_file(d, str(p))
    text = p.read_text()
    # trailing ';' and comments after the value are ignored; commented keys never match
    text = text.replace("Density 1.17621", "Density 1.17621; //!air") + "//Collision-Model SRT\n"
    p.write_text(text)
    a = engine.parse_case_file(str(p))
    assert a.density == 1.17621 and a.op == default_case().op
    # a missing mandatory keyword is an error naming the keyword
    p.write_text("\n".join(l for l in text.splitlines() if not l.startswith("SpeedOfSound")))
    with pytest.raises(engine.AcpError, match="SpeedOfSound"):
        engine.parse_case_file(str(p))
    # node counts: ceil(size / spacing + 1e-8) (Control.cpp:43-45)
    d2 = read_case_file(str(tmp_path / "bc.txt")) if False else None
    write_case_file(default_case(), str(p))
    a = engine.parse_case_file(str(p))
    assert (a.nx, a.ny, a.nz) == (151, 151, 21)


@pytest.mark.parametrize("dims", [(7, 6, 5), (9, 5, 6)])
def test_boundary_wiring_matches_reference(dims):
    from tests.golden.make_golden import small_case
    L = engine.lib()
    L.acp_boundary_wiring.argtypes = [C.POINTER(CaseDesc), C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong)]
    d = small_case(*dims)
    cnt = C.c_longlong()
    assert L.acp_boundary_wiring(C.byref(d), None, 0, C.byref(cnt)) == ACP_OK
    rows = np.zeros((cnt.value, 12), dtype=np.int64)
    assert L.acp_boundary_wiring(C.byref(d), rows.ctypes.data, cnt.value, C.byref(cnt)) == ACP_OK
    gold = np.loadtxt(os.path.join(HERE, "golden", "topo_%dx%dx%d.txt" % dims), dtype=np.int64)
    gold = gold[np.argsort(gold[:, 0] + dims[0] * (gold[:, 1] + dims[1] * gold[:, 2]))]
    np.testing.assert_array_equal(rows, gold)


def test_invalid_cases_rejected_before_device_use():
    L = engine.lib()
    bad = default_case()
    bad.eq_order = 5
    h = C.c_void_p()
    assert L.acp_create(C.byref(bad), -1, C.byref(h)) == ACP_ERR_INVALID
    assert b"order" in L.acp_last_error(h)
    L.acp_destroy(h)
    small = default_case()
    small.nz = 3  # LODI axis with 3 nodes
    h = C.c_void_p()
    assert L.acp_create(C.byref(small), -1, C.byref(h)) == ACP_ERR_UNSUPPORTED
    L.acp_destroy(h)
    size = C.c_size_t()
    assert L.acp_estimate_bytes(C.byref(default_case()), C.byref(size)) == ACP_OK
    n = 151 * 151 * 21
    assert size.value >= n * 2 * 19 * 8


def test_coupling_needs_matching_overlap():
    """STD couples with one coarse cell of overlap, DC1/DC2 with none
    (BoundaryConditions.txt: Overlap 0 for the direct coupling)."""
    from acpulse_vclbm_b200.capi import COUPLING, LAYOUT_BOX, lattice_units_case
    L = engine.lib()
    for coupling, overlap in [("STD", 0), ("DC1", 1), ("DC2", 1)]:
        d = lattice_units_case(32, 16, 3, op="HRR", periodic=(False, True, True))
        d.max_level, d.layout = 1, LAYOUT_BOX
        d.box_lo[:] = [16, 0, 0]
        d.box_hi[:] = [31, 15, 2]
        d.coupling, d.overlap = COUPLING[coupling], overlap
        h = C.c_void_p()
        assert L.acp_create(C.byref(d), -1, C.byref(h)) == ACP_ERR_INVALID
        assert b"Overlap" in L.acp_last_error(h)
        L.acp_destroy(h)
