"""The x-slab decomposition (acpulse_vclbm_b200/slabs.py) through the engine on
one GPU: every slab its own case, halos refreshed with acp_copy_columns and,
for the rank path, acp_get_columns / acp_put_columns.  The owned columns of
all slabs equal the undivided lattice's state bit for bit -- each node runs
the same kernels on the same inputs -- for HRR (y-marching collide), RR with
cubic-Mach on a 3-D box with transverse LODI (x-y tiled collide), a periodic
x axis, and the FP32 deviation form."""
import numpy as np
import pytest

from acpulse_vclbm_b200 import engine, slabs
from acpulse_vclbm_b200.capi import lattice_units_case

pytestmark = pytest.mark.gpu


def _cases():
    a = lattice_units_case(96, 20, 3, op="HRR", nu_lu=1e-3, periodic=(False, True, True), eps=1e-2, b=4.0,
                           center=(40.0, 10.0, 1.0))
    a.hybrid_sigma = 0.98
    b = lattice_units_case(48, 12, 10, op="RR", nu_lu=1e-3, periodic=(False, False, False), eps=1e-2, b=3.0,
                           center=(23.5, 5.5, 4.5), ic_dims=3)
    b.transverse, b.cubic_mach = 1, 1
    c = lattice_units_case(64, 10, 4, op="SRT", nu_lu=1e-3, periodic=(True, True, True), eps=1e-2, b=3.0,
                           center=(3.0, 5.0, 2.0), ic_dims=3)
    d = lattice_units_case(96, 20, 3, op="HRR", nu_lu=1e-3, periodic=(False, True, True), eps=1e-2, b=4.0,
                           center=(40.0, 10.0, 1.0), storage="FP32-DEV")
    return [("hrr-quasi2d", a, 3, 8), ("rr-cubic-3d", b, 3, 6), ("srt-periodic-x", c, 2, 6), ("hrr-fp32", d, 4, 8)]


@pytest.mark.parametrize("name,desc,nslabs,halo", _cases(), ids=[c[0] for c in _cases()])
def test_slabs_equal_the_whole_lattice(name, desc, nslabs, halo):
    steps = 3 * slabs.interval(halo) + 1
    S = slabs.SlabLattice(desc, nslabs, halo=halo).init()
    S.step(steps)
    S.sync()
    got = S.populations()
    S.close()
    L = engine.Lattice(desc).init()
    L.step(steps)
    L.sync()
    want = L.populations()
    L.close()
    np.testing.assert_array_equal(got, want)


def test_get_put_columns_round_trip():
    """acp_get_columns / acp_put_columns move raw storage values: a column
    block read from one case and written into another makes those columns of
    the two cases equal, and nothing else changes"""
    import ctypes as C
    d = lattice_units_case(40, 8, 3, op="SRT", nu_lu=1e-3, periodic=(False, True, True), eps=1e-2, b=3.0,
                           center=(12.0, 4.0, 1.0), storage="FP32-DEV")
    A = engine.Lattice(d).init()
    A.step(5)
    B = engine.Lattice(d).init()
    before = B.populations()
    buf = np.empty((19, 3, 8, 6), dtype=np.float32)
    lib = engine.lib()
    assert lib.acp_get_columns(A._h, 10, 6, buf.ctypes.data) == 0
    assert lib.acp_put_columns(B._h, 20, 6, buf.ctypes.data) == 0
    fa, fb = A.populations(), B.populations()
    np.testing.assert_array_equal(fb[..., 20:26], fa[..., 10:16])
    np.testing.assert_array_equal(np.delete(fb, range(20, 26), axis=3), np.delete(before, range(20, 26), axis=3))
    assert lib.acp_get_columns(A._h, 38, 6, buf.ctypes.data) != 0  # past the last column
    A.close()
    B.close()
