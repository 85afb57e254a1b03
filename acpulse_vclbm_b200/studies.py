"""Studies of the pulse configurations on the GPU.

sweep      -- the operator and scheme sweep: a quasi-2D pulse on 1024 x 512 x 3
              coarse nodes, the right half refined 2:1, eps = 1e-3, b = 24, for
              each collision operator x refinement scheme (overlap STD, direct
              coupling DC1) x restriction (LAG, TOU) x nu in {1e-5, 1e-4, 1e-3},
              over 3200 coarse steps, FP64.  Outputs per run: the reflection
              coefficient at the interface (upstream probe against the same
              pulse on the uniform coarse lattice) and, for nu = 1e-4, the L2
              and max pressure error of the FP32 deviation form against FP64.
precision  -- the precision form: a 3-D pulse in a 256^3 box with a centred
              128^3-cell patch refined 2:1, HRR, nu = 1e-4, b = 12, LODI with
              transverse terms on all six faces, eps in {1e-2, 1e-4}; FP32
              deviation and FP16 (per-population power-of-two scales) storage
              against the FP64 GPU form on the same inputs: probe and pressure
              field errors relative to the pulse amplitude.

usage: python -m acpulse_vclbm_b200.studies sweep|precision [--steps N] [--out file.json]
"""
import argparse
import json
import time

import numpy as np

from . import analysis, engine
from .capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case

OPS5 = ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"]


def _run(d, steps, probes):
    L = engine.Lattice(d).init()
    L.set_probes(probes)
    L.step(steps)
    L.sync()
    s = L.probes()
    p = [L.field(4, l) for l in range(d.max_level + 1)]
    L.close()
    return s, p


def sweep(steps=3200, nx=1024, ny=512):
    rows = []
    uni = {}
    p0 = None
    for op in OPS5:
        for nu in (1e-5, 1e-4, 1e-3):
            du = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                         center=(nx / 4.0, ny / 2.0, 1.0), refined=False)
            try:
                uni[(op, nu)], _ = _run(du, steps, analysis.interface_probes(du))
            except engine.AcpError as e:
                rows.append({"op": op, "nu": nu, "uniform_error": str(e)})
                continue
            p0 = du.density * du.speed_of_sound ** 2
            for coupling in ("STD", "DC1"):
                for filt in ("LAG", "TOU"):
                    t0 = time.perf_counter()
                    d = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                                center=(nx / 4.0, ny / 2.0, 1.0), filt=filt, coupling=coupling)
                    try:
                        s64, f64 = _run(d, steps, analysis.interface_probes(d))
                    except engine.AcpError as e:  # a numerical blow-up is a result of the sweep
                        row = {"op": op, "nu": nu, "coupling": coupling, "filter": filt, "R": None,
                               "error": str(e)}
                        rows.append(row)
                        print(json.dumps(row), flush=True)
                        continue
                    w = min(steps, analysis.window_steps(d))
                    r = analysis.reflection_coefficient(s64[:, 0], uni[(op, nu)][:, 0], p0, w)
                    row = {"op": op, "nu": nu, "coupling": coupling, "filter": filt, "R": r, "window_steps": w}
                    if nu == 1e-4:
                        d32 = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                                      center=(nx / 4.0, ny / 2.0, 1.0), filt=filt,
                                                      coupling=coupling, storage="FP32-DEV")
                        try:
                            s32, f32 = _run(d32, steps, analysis.interface_probes(d32))
                        except engine.AcpError as e:
                            row["fp32_error"] = str(e)
                            rows.append(row)
                            continue
                        amp = d.ic_eps * d.density * d.speed_of_sound ** 2
                        live = slice(0, nx // 2 + 1 + d.overlap)
                        e = [f32[0][..., live] - f64[0][..., live], f32[1] - f64[1]]
                        n = sum(x.size for x in e)
                        row["fp32_l2_err_rel_amp"] = float(np.sqrt(sum((x ** 2).sum() for x in e) / n) / amp)
                        row["fp32_max_err_rel_amp"] = float(max(np.abs(x).max() for x in e) / amp)
                        row["fp32_probe_err_rel_amp"] = float(np.abs(s32 - s64).max() / amp)
                        r32 = analysis.reflection_coefficient(s32[:, 0], uni[(op, nu)][:, 0], p0, w)
                        row["fp32_R_rel_err"] = abs(r32 - r) / r
                    row["seconds"] = time.perf_counter() - t0
                    rows.append(row)
                    print(json.dumps(row), flush=True)
    return {"study": "operator and scheme sweep", "nx": nx, "ny": ny, "nz": 3, "steps": steps, "rows": rows}


def precision_case(eps, storage, n=256):
    lo, hi = n // 4, n // 4 + n // 2
    d = lattice_units_case(n, n, n, op="HRR", nu_lu=1e-4, order=3, periodic=(False, False, False), eps=eps,
                           b=12.0, center=(n / 2.0, n / 2.0, n / 2.0), storage=storage, ic_dims=3)
    d.hybrid_sigma = 0.98
    d.transverse = 1
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [lo, lo, lo]
    d.box_hi[:] = [hi, hi, hi]
    d.f2c_filter = F2C_FILTER["LAG"]
    return d


def precision(steps=300, n=256):
    rows = []
    c = n // 2
    lo = n // 4
    probes = [(1, 2 * (lo + 10), 2 * c, 2 * c), (0, lo - 10, c, c)]  # 10 cells inside and outside the patch face
    for eps in (1e-2, 1e-4):
        ref = None
        for storage in ("FP64", "FP32-DEV", "FP16-DEV"):
            d = precision_case(eps, storage, n)
            t0 = time.perf_counter()
            L = engine.Lattice(d).init()
            L.set_probes(probes)
            L.step(steps)
            L.sync()
            ms = (time.perf_counter() - t0) * 1e3 / steps
            s = L.probes()
            f = [L.field(4, l) for l in range(2)]
            c_, fi = L.active_updates()
            L.close()
            amp = eps * d.density * d.speed_of_sound ** 2
            row = {"eps": eps, "storage": storage, "steps": steps, "ms_per_step_incl_setup": ms,
                   "updates_per_step": c_ + 2 * fi}
            if ref is None:
                ref = (s, f)
            else:
                live = np.ones(f[0].shape, dtype=bool)
                live[lo + 1:lo + n // 2, lo + 1:lo + n // 2, lo + 1:lo + n // 2] = False  # covered coarse nodes
                row["probe_err_rel_amp"] = float(np.abs(s - ref[0]).max() / amp)
                row["field_max_err_rel_amp"] = float(max(np.abs(f[0] - ref[1][0])[live].max(),
                                                         np.abs(f[1] - ref[1][1]).max()) / amp)
            rows.append(row)
            print(json.dumps(row), flush=True)
    return {"study": "precision form", "n": n, "steps": steps, "rows": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("study", choices=["sweep", "precision"])
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--out", default="")
    a = ap.parse_args()
    if a.study == "sweep":
        res = sweep(steps=a.steps or 3200)
    else:
        res = precision(steps=a.steps or 300)
    if a.out:
        json.dump(res, open(a.out, "w"), indent=1)


if __name__ == "__main__":
    main()
