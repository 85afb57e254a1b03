"""Checkpoint / restart of a case's device state through the C ABI
(acp_checkpoint_save / acp_checkpoint_load).  The reference has no restart
(main.cpp:37-121 builds every run from its case file).

A run that is saved after k coarse steps and continued must equal, bit for
bit, a fresh handle of the same case restored from that file and stepped as
far: both ping-pong arrays, the partner-strain records and the parity are
part of the file.  An odd k checks the parity; the two-level STD/HRR case
checks the partner-strain records; DC1, FP64 and FP16 storage cover the other
state shapes.  A file of another level shape is refused.
"""
import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import (C2F_REPLACE, COUPLING, F2C_FILTER, F2C_REPLACE, LAYOUT_BOX,
                                     lattice_units_case)

pytestmark = pytest.mark.gpu


def two_level(op, storage, coupling="STD", nx=48, ny=20):
    d = lattice_units_case(nx, ny, 3, op=op, nu_lu=1e-3, order=3, periodic=(False, True, True), eps=1e-3, b=4.0,
                           center=(nx / 4.0, ny / 2.0, 1.0), storage=storage)
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 1
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [nx // 2, 0, 0]
    d.box_hi[:] = [nx - 1, ny - 1, 2]
    d.f2c_filter = F2C_FILTER["LAG"]
    if coupling != "STD":
        d.coupling = COUPLING[coupling]
        d.overlap = 0
        d.c2f_replace = C2F_REPLACE["Mf"]
        d.f2c_replace = F2C_REPLACE["Mc"]
    return d


def single_level(op, storage):
    d = lattice_units_case(40, 24, 16, op=op, nu_lu=1e-3, order=3, periodic=(False, False, False), eps=1e-3, b=4.0,
                           center=(20.0, 12.0, 8.0), storage=storage, ic_dims=3)
    d.transverse = 1
    return d


def state(L, levels):
    return [L.populations(l) for l in range(levels)]


@pytest.mark.parametrize("make,levels", [
    (lambda: two_level("HRR", "FP32-DEV"), 2),
    (lambda: two_level("HRR", "FP64", coupling="DC1"), 2),
    (lambda: single_level("RR", "FP16-DEV"), 1),
    (lambda: single_level("HRR", "FP64"), 1),
])
def test_restart_continues_bit_for_bit(tmp_path, make, levels):
    path = str(tmp_path / "case.ckpt")
    a = engine.Lattice(make()).init()
    a.step(7)
    a.save_checkpoint(path)
    a.step(6)
    a.sync()
    want = state(a, levels)
    assert a.steps_done() == 13
    a.close()

    b = engine.Lattice(make()).init()
    b.step(2)  # state and parity of the fresh handle are overwritten by the file
    b.load_checkpoint(path)
    assert b.steps_done() == 7
    b.step(6)
    b.sync()
    got = state(b, levels)
    b.close()
    for w, g in zip(want, got):
        assert np.array_equal(w, g)


def test_restart_refuses_another_level_shape(tmp_path):
    path = str(tmp_path / "case.ckpt")
    a = engine.Lattice(two_level("HRR", "FP32-DEV")).init()
    a.step(1)
    a.save_checkpoint(path)
    a.close()
    b = engine.Lattice(two_level("HRR", "FP32-DEV", nx=56)).init()
    with pytest.raises(engine.AcpError) as e:
        b.load_checkpoint(path)
    assert e.value.status == -1
    c = engine.Lattice(two_level("HRR", "FP64")).init()
    with pytest.raises(engine.AcpError):
        c.load_checkpoint(path)
    with pytest.raises(engine.AcpError):
        c.load_checkpoint(str(tmp_path / "missing.ckpt"))
    b.close()
    c.close()


def test_restart_refuses_another_case_and_a_truncated_file(tmp_path):
    """A file of another operator, or a cut-off file, is refused before the
    device state is touched: the handle keeps stepping as before."""
    path = str(tmp_path / "case.ckpt")
    a = engine.Lattice(two_level("HRR", "FP32-DEV")).init()
    a.step(3)
    a.save_checkpoint(path)
    a.close()
    b = engine.Lattice(two_level("RR", "FP32-DEV")).init()  # same shapes, another operator
    b.step(2)
    b.sync()
    before = b.populations(0)
    with pytest.raises(engine.AcpError) as e:
        b.load_checkpoint(path)
    assert e.value.status == -1
    cut = str(tmp_path / "cut.ckpt")
    with open(path, "rb") as src, open(cut, "wb") as dst:
        data = src.read()
        dst.write(data[:len(data) - 100])
    c = engine.Lattice(two_level("HRR", "FP32-DEV")).init()
    c.step(2)
    c.sync()
    keep = c.populations(1)
    with pytest.raises(engine.AcpError):
        c.load_checkpoint(cut)
    assert np.array_equal(c.populations(1), keep) and c.steps_done() == 2
    assert np.array_equal(b.populations(0), before)
    b.close()
    c.close()


def test_probe_series_restart_after_load(tmp_path):
    """Probe series restart empty after a load; the step count continues."""
    path = str(tmp_path / "case.ckpt")
    d = two_level("SRT", "FP64")
    a = engine.Lattice(d).init()
    a.set_probes([(0, 8, 10, 1)])
    a.step(5)
    a.save_checkpoint(path)
    a.step(4)
    a.sync()
    ref = a.probes()
    a.close()
    b = engine.Lattice(d).init()
    b.set_probes([(0, 8, 10, 1)])
    b.step(1)
    b.load_checkpoint(path)
    b.step(4)
    b.sync()
    got = b.probes()
    assert b.steps_done() == 9
    b.close()
    assert got.shape == (4, 1)
    assert np.array_equal(got, ref[5:9])
