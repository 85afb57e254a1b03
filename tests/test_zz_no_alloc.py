"""acp_read_populations_window: reading populations without device allocation.

Some callers of this library cannot allocate device memory: a serving process
that has handed its whole HBM budget to resident lattices, and applications
whose own allocator owns all device memory.  acp_read_populations makes a
temporary FP64 copy of a whole level on the device; the window variant goes
through a fixed array built into the library instead, at most
ACP_WINDOW_MAX_NODES nodes per call.  This test reads two windows in a row
through the C ABI and checks each against the same nodes of
acp_read_populations.  It lives in a file of its own that pytest collects
last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import ACP_ERR_INVALID, ACP_OK, lattice_units_case

pytestmark = pytest.mark.gpu

WINDOW_MAX = 32768  # ACP_WINDOW_MAX_NODES in include/acp.h


def _bind():
    lib = engine.lib()
    lib.acp_read_populations_window.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p]
    return lib


def _two_level(storage):
    from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX
    d = lattice_units_case(32, 12, 3, op="HRR", nu_lu=1e-3, order=3, periodic=(False, True, True), eps=1e-3, b=3.0,
                           center=(14.0, 6.0, 1.0), storage=storage)
    d.hybrid_sigma = 0.98
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [16, 0, 0]
    d.box_hi[:] = [31, 11, 2]
    d.f2c_filter = F2C_FILTER["LAG"]
    return d


@pytest.mark.parametrize("storage,level", [("FP32-DEV", 0), ("FP64", 0), ("FP16-DEV", 0),
                                           ("FP32-DEV", 1), ("FP16-DEV", 1)])
def test_window_read_matches_full_read_twice(storage, level):
    lib = _bind()
    if level == 0:
        d = lattice_units_case(40, 24, 3, op="HRR", nu_lu=1e-3, order=3, eps=1e-3, b=4.0, center=(14.0, 12.0, 1.0),
                               storage=storage)
    else:  # the fine level of a two-level case, whose state sits in its first array between coarse steps
        d = _two_level(storage)
    L = engine.Lattice(d).init()
    L.step(7)
    L.sync()
    full = L.populations(level).reshape(19, -1)
    n = full.shape[1]
    windows = [(5, 1000), (n - 777, 777)]  # two calls in a row, the second at the end of the level
    for begin, count in windows:
        out = np.full((19, count), np.nan)
        s = lib.acp_read_populations_window(L._h, level, begin, count, out.ctypes.data)
        assert s == ACP_OK, lib.acp_last_error(L._h)
        np.testing.assert_allclose(out, full[:, begin:begin + count], rtol=0, atol=1e-14)
    L.close()


def test_window_limits_are_enforced():
    lib = _bind()
    d = lattice_units_case(40, 24, 3, op="SRT", nu_lu=1e-3, order=3)
    L = engine.Lattice(d).init()
    out = np.zeros((19, 4))
    assert lib.acp_read_populations_window(L._h, 0, 0, WINDOW_MAX + 1, out.ctypes.data) == ACP_ERR_INVALID
    assert b"ACP_WINDOW_MAX_NODES" in lib.acp_last_error(L._h)
    assert lib.acp_read_populations_window(L._h, 0, 40 * 24 * 3 - 2, 4, out.ctypes.data) == ACP_ERR_INVALID
    # a begin near the largest 64-bit value is refused, not wrapped around
    assert lib.acp_read_populations_window(L._h, 0, (1 << 63) - 2, 4, out.ctypes.data) == ACP_ERR_INVALID
    assert lib.acp_read_populations_window(L._h, 0, -1, 4, out.ctypes.data) == ACP_ERR_INVALID
    L.close()
