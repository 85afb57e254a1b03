"""Probe series and the reflection coefficient at the refinement interface.

The reference writes ASCII VTK only and has no probes or reflection
coefficient (Lattice.cpp:2212-4352).  The pulse configurations measure the
wave reflected by the 2:1 interface: a quasi-2D Gaussian pulse travels in +x
towards the refined right half; a probe `offset` coarse cells upstream of the
interface records the incident pulse and, later, the wave the interface
reflects.  The reflected signal is isolated by subtracting the same pulse
solved on the uniform coarse lattice (no interface):

    R = max_t |p_refined(t) - p_uniform(t)| / max_t |p_uniform(t) - p0|

over the window before waves reflected by the far x faces reach the probe.
"""
import numpy as np

from .capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case


def interface_case(nx=128, ny=64, nz=3, op="SRT", nu=1e-3, eps=1e-3, b=6.0, center=(32.0, 32.0, 1.0),
                   storage="FP64", refined=True, filt="LAG", coupling="STD"):
    """The reference-sized pulse case: nx x ny x nz coarse nodes, periodic y
    and z, LODI x faces, the right half refined 2:1 (or uniform)."""
    d = lattice_units_case(nx, ny, nz, op=op, nu_lu=nu, order=3, periodic=(False, True, True), eps=eps, b=b,
                           center=center, storage=storage)
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 1
    if refined:
        from .capi import C2F_REPLACE, COUPLING, F2C_REPLACE
        d.max_level = 1
        d.layout = LAYOUT_BOX
        d.box_lo[:] = [nx // 2, 0, 0]
        d.box_hi[:] = [nx - 1, ny - 1, nz - 1]
        d.f2c_filter = F2C_FILTER[filt]
        d.coupling = COUPLING[coupling]
        d.overlap = 1 if coupling == "STD" else 0
        if coupling != "STD":
            d.c2f_replace, d.f2c_replace = C2F_REPLACE["Mf"], F2C_REPLACE["Mc"]
    return d


def interface_probes(d, offset=10):
    """(level, i, j, k) of the probes `offset` coarse cells either side of the
    interface on the pulse axis: upstream on the coarse level, downstream on
    the fine level (coarse level when uniform)."""
    x0 = d.nx // 2
    j, k = int(round(d.ic_center[1])), d.nz // 2
    up = (0, x0 - offset, j, k)
    down = (1, 2 * (x0 + offset), 2 * j, 2 * k) if d.max_level == 1 else (0, x0 + offset, j, k)
    return [up, down]


def window_steps(d, offset=10):
    """coarse steps before the wave reflected by the far x face -- the one
    face that differs between the refined and the uniform run -- can reach
    the upstream probe (sound speed 1/sqrt(3) coarse cells per coarse step),
    with a 10 % margin"""
    xp = d.nx // 2 - offset
    xc = d.ic_center[0]
    far = (d.nx - 1 - xc) + (d.nx - 1 - xp)
    return int(0.9 * far * np.sqrt(3.0))


def reflection_coefficient(p_refined, p_uniform, p0, window):
    """R from the upstream probe series of the refined and uniform runs."""
    a = np.asarray(p_refined)[:window]
    u = np.asarray(p_uniform)[:window]
    inc = np.abs(u - p0).max()
    return float(np.abs(a - u).max() / inc)
