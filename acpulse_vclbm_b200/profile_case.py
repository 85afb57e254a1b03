"""Run a few coarse steps of one pulse case, for profilers (ncu) and quick
timing.  Prints the per-kernel device times of acp_step_timed.

usage: python -m acpulse_vclbm_b200.profile_case [--op HRR] [--storage FP32-DEV]
           [--nx 1024 --ny 512 --nz 3] [--steps 3] [--levels 1]
       python -m acpulse_vclbm_b200.profile_case --batched 64 [--steps 3]
           (the seeded batched workload, workloads.batched_cases(seed=2024), in one batch)
"""
import argparse
import ctypes as C

from . import engine
from .capi import lattice_units_case


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", default="HRR")
    ap.add_argument("--storage", default="FP32-DEV")
    ap.add_argument("--order", type=int, default=3)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nz", type=int, default=3)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--timed", type=int, default=0, help="also run N steps kernel by kernel with events")
    ap.add_argument("--levels", type=int, default=1, choices=[1, 2],
                    help="2: refine the right half 2:1 (the sweep configuration's layout)")
    ap.add_argument("--filter", default="LAG")
    ap.add_argument("--coupling", default="STD", choices=["STD", "DC1", "DC2"])
    ap.add_argument("--batched", type=int, default=0, help="run N seeded batched cases in one batch instead")
    a = ap.parse_args()
    if a.batched:
        from . import workloads
        Ls = [engine.Lattice(d).init() for d in workloads.batched_cases(seed=2024, n=a.batched)]
        B = engine.Batch(Ls)
        B.step(a.steps)
        B.sync()
        print(B.info())
        B.close()
        for L in Ls:
            L.close()
        return
    d = lattice_units_case(a.nx, a.ny, a.nz, op=a.op, nu_lu=1e-4, order=a.order, periodic=(False, True, True),
                           eps=1e-3, b=24.0, center=(a.nx / 4.0, a.ny / 2.0, 1.0), storage=a.storage)
    d.mrt_writeback = 1
    if a.levels == 2:
        from .capi import F2C_FILTER, LAYOUT_BOX
        d.max_level = 1
        d.layout = LAYOUT_BOX
        d.box_lo[:] = [a.nx // 2, 0, 0]
        d.box_hi[:] = [a.nx - 1, a.ny - 1, a.nz - 1]
        d.f2c_filter = F2C_FILTER[a.filter]
        if a.coupling != "STD":
            from .capi import C2F_REPLACE, COUPLING, F2C_REPLACE
            d.coupling = COUPLING[a.coupling]
            d.overlap = 0
            d.c2f_replace = C2F_REPLACE["Mf"]
            d.f2c_replace = F2C_REPLACE["Mc"]
    L = engine.Lattice(d).init()
    L.step(a.steps)
    L.sync()
    if a.timed:
        km = (C.c_double * 5)()
        engine.lib().acp_step_timed.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        engine.lib().acp_step_timed(L._h, a.timed, C.cast(km, C.c_void_p))
        c, f = L.active_updates()
        nodes = c + 2 * f
        b = {"FP64": 8, "FP32-DEV": 4, "FP16-DEV": 2}[a.storage] * 38
        print(f"{a.op} {a.storage} order {a.order} {a.nx}x{a.ny}x{a.nz} levels {a.levels}: "
              f"collide {km[1]*1e3:.1f} us ({nodes * b / (km[1] * 1e-3) / 1e9:.0f} GB/s algorithmic), "
              f"lodi {km[2]*1e3:.1f} us, coupling {km[3]*1e3:.1f} us, updates/step {nodes}")
    L.close()


if __name__ == "__main__":
    main()
