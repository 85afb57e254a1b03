"""The batched form: many cases of uneven sizes, operators, storage forms and
refinement layouts advanced together (acp_batch_*), against the same cases
advanced alone through acp_step, under every schedule the autotuner can
choose.  The batched kernels run the same per-node device code on the same
inputs, inlined into other kernels, where the compiler may contract a
multiply-add differently; the stated tolerance is therefore rounding-level
for each storage form: FP64 populations within 1e-12 rho0, FP32 deviations
within 1e-6 of the pulse amplitude eps rho0, FP16 deviations within 1e-3 of it
(FP16 storage rounds a last-bit FP32 difference to a half-precision step)."""
import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import (ACP_ERR_STATE, C2F_REPLACE, COUPLING, F2C_FILTER, F2C_REPLACE, LAYOUT_BOX,
                                     lattice_units_case)

pytestmark = pytest.mark.gpu


def two_level(d, coupling="STD", filt="LAG"):
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [d.nx // 2, 0, 0]
    d.box_hi[:] = [d.nx - 1, d.ny - 1, d.nz - 1]
    d.f2c_filter = F2C_FILTER[filt]
    d.coupling = COUPLING[coupling]
    d.overlap = 1 if coupling == "STD" else 0
    if coupling != "STD":
        d.c2f_replace, d.f2c_replace = C2F_REPLACE["Mf"], F2C_REPLACE["Mc"]
    return d


def mix():
    """eight cases: five operators, single and two levels, STD / DC1 / DC2,
    FP64 / FP32 / FP16 storage, quasi-2D and 3-D, one with probes"""
    cs = []
    q2 = dict(periodic=(False, True, True), eps=1e-3)
    cs.append(lattice_units_case(64, 20, 3, op="SRT", nu_lu=1e-3, b=4.0, center=(20, 10, 1), **q2))
    cs.append(two_level(lattice_units_case(96, 32, 3, op="HRR", nu_lu=1e-4, b=5.0, center=(30, 16, 1),
                                           storage="FP32-DEV", **q2)))
    cs.append(two_level(lattice_units_case(48, 24, 3, op="RR", nu_lu=1e-3, b=4.0, center=(12, 12, 1), **q2),
                        coupling="DC1", filt="TOU"))
    d = lattice_units_case(40, 16, 3, op="MRT-GS", nu_lu=1e-3, b=4.0, center=(12, 8, 1), storage="FP32-DEV", **q2)
    d.mrt_writeback = 1
    cs.append(d)
    d = two_level(lattice_units_case(48, 20, 3, op="MRT-RM", nu_lu=1e-3, b=4.0, center=(12, 10, 1), **q2),
                  coupling="DC2", filt="NOFI")
    d.mrt_writeback = 1
    cs.append(d)
    d = lattice_units_case(20, 18, 16, op="RR", nu_lu=1e-3, b=3.0, center=(10, 9, 8), periodic=(False, False, False),
                           eps=1e-3, ic_dims=3)
    d.cubic_mach = 1
    cs.append(d)
    cs.append(lattice_units_case(64, 24, 3, op="HRR", nu_lu=1e-3, b=4.0, center=(20, 12, 1), storage="FP16-DEV", **q2))
    cs.append(two_level(lattice_units_case(96, 32, 3, op="HRR", nu_lu=1e-4, b=5.0, center=(30, 16, 1),
                                           storage="FP32-DEV", **q2)))  # same group as case 1
    return cs


def make(descs):
    Ls = [engine.Lattice(d).init() for d in descs]
    Ls[1].set_probes([(0, 40, 16, 1), (1, 120, 32, 2)][:1])
    return Ls


def states(L):
    return [L.populations(l) for l in range(L.desc.max_level + 1)]


TOL = {0: 1e-12, 1: 1e-6, 2: 1e-3}  # storage -> tolerance (FP64 absolute in rho0; others of eps rho0)


def tolerance(d):
    return TOL[d.storage] * (d.density if d.storage == 0 else d.ic_eps * d.density)


def check_equal(batched, alone):
    for k, (Lb, La) in enumerate(zip(batched, alone)):
        assert Lb.steps_done() == La.steps_done()
        for l, (fb, fa) in enumerate(zip(states(Lb), states(La))):
            assert np.abs(fb - fa).max() <= tolerance(Lb.desc), (k, l, float(np.abs(fb - fa).max()))


def test_batch_matches_alone():
    descs = mix()
    Lb, La = make(descs), make(descs)
    B = engine.Batch(Lb)
    info = B.info()
    assert info["groups"] == 7  # the two FP32 HRR two-level cases share one group
    B.step(25)
    B.sync()
    for L in La:
        L.step(25)
        L.sync()
    check_equal(Lb, La)
    cs2 = descs[1].speed_of_sound ** 2
    assert np.abs(Lb[1].probes() - La[1].probes()).max() <= tolerance(descs[1]) * cs2
    with pytest.raises(engine.AcpError) as e:
        Lb[0].step(1)
    assert e.value.status == ACP_ERR_STATE
    B.close()
    Lb[0].step(1)  # released
    for L in Lb + La:
        L.close()


@pytest.mark.parametrize("persist,largest", [(0, False), (1, True), (2, False), (4, True)])
def test_batch_schedules(persist, largest):
    descs = mix()
    Lb, La = make(descs), make(descs)
    B = engine.Batch(Lb)
    B.configure(persist=persist, largest_first=largest, chunk_scale=2)
    B.step(13)
    B.sync()
    for L in La:
        L.step(13)
        L.sync()
    check_equal(Lb, La)
    B.close()
    for L in Lb + La:
        L.close()


def test_autotuner_keeps_results():
    descs = mix()
    Lb, La = make(descs), make(descs)
    B = engine.Batch(Lb)
    report = B.tune(trial_steps=2)
    assert "chosen:" in report
    B.step(3)
    B.sync()
    n = Lb[0].steps_done()
    for L in La:
        L.step(n)
        L.sync()
    check_equal(Lb, La)
    B.close()
    for L in Lb + La:
        L.close()
