"""Generate the golden fixtures of the single-level hot path from the reference.

Runs the reference's own Control/Lattice code (built from its sources by
oracle/ref_build/Makefile into oracle/_ref/acp_ref) on small single-level
cases and stores, per case:
  * the BoundaryConditions.txt it ran (so tests also exercise the parser),
  * the SHA-256 of the final FP64 population state (structure-of-arrays,
    little endian) -- the CPU oracle must reproduce it bit for bit,
  * the final density field (float64) for tolerance checks of the GPU path,
  * the reference's boundary wiring (--topo) for two grid sizes,
  * the reference's legacy VTK file of one small case (--vtk) with its case file.
This needs /root/reference; the fixtures it writes are committed.

usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from acpulse_vclbm_b200.capi import OPS, default_case  # noqa: E402
from acpulse_vclbm_b200.config import write_case_file  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "acp_ref")


def small_case(nx=38, ny=12, nz=7, spacing=0.04, nu=0.024):
    d = default_case()
    d.spacing = spacing
    d.nx, d.ny, d.nz = nx, ny, nz
    d.domain_size[:] = [(nx - 0.5) * spacing, (ny - 0.5) * spacing, (nz - 0.5) * spacing]
    d.kinematic_viscosity = nu
    return d


def run_reference(bc_path, steps, out_path):
    r = subprocess.run([REF, bc_path, str(steps), out_path], capture_output=True, text=True, check=True)
    raw = open(out_path, "rb").read()
    nx, ny, nz, _ = np.frombuffer(raw[:16], dtype=np.int32)
    f = np.frombuffer(raw[16:], dtype=np.float64).reshape(nx, ny, nz, 19)
    return np.ascontiguousarray(f.transpose(3, 2, 1, 0)), json.loads(r.stdout.strip().splitlines()[-1])


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref_build")], check=True)
    cases = []
    tmp = os.path.join(HERE, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    specs = []
    for op in ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"]:
        for order in (2, 3, 4):
            for tr in (0, 1):
                for cm in ((0, 1) if op in ("RR", "HRR") else (0,)):
                    specs.append(dict(op=op, order=order, transverse=tr, cubic=cm, steps=30, nu=0.024))
    # a longer run: the pulse leaves through the LODI faces
    specs.append(dict(op="SRT", order=3, transverse=1, cubic=0, steps=200, nu=0.024))
    specs.append(dict(op="HRR", order=3, transverse=0, cubic=0, steps=200, nu=0.024))
    # the shipped physics (air, nu = 1.49e-5 m^2/s)
    specs.append(dict(op="HRR", order=3, transverse=0, cubic=0, steps=40, nu=1.49e-5))
    rho_fields = {}
    for s in specs:
        d = small_case(nu=s["nu"])
        d.op = OPS[s["op"]]
        d.eq_order = s["order"]
        d.transverse = s["transverse"]
        d.cubic_mach = s["cubic"]
        name = f"{s['op']}_o{s['order']}_t{s['transverse']}_c{s['cubic']}_s{s['steps']}_nu{s['nu']:g}"
        bc = os.path.join(tmp, name + ".txt")
        write_case_file(d, bc, steps=s["steps"], threads=8)
        f, timing = run_reference(bc, s["steps"], os.path.join(tmp, name + ".bin"))
        h = hashlib.sha256(f.astype("<f8").tobytes()).hexdigest()
        rho_fields[name] = f.sum(axis=0)
        cases.append(dict(name=name, steps=s["steps"], sha256=h, case_file=open(bc).read(),
                          dims=[int(d.nx), int(d.ny), int(d.nz)]))
        print(name, h[:16], f"rho range {f.sum(axis=0).min():.9f}..{f.sum(axis=0).max():.9f}")
    np.savez_compressed(os.path.join(HERE, "single_level_rho.npz"), **rho_fields)
    with open(os.path.join(HERE, "single_level.json"), "w") as fh:
        json.dump(dict(generator="tests/golden/make_golden.py", reference="aleksandrShukman/acPulse_vcLBM",
                       layout="f[q][k][j][i] float64 little endian", cases=cases), fh, indent=1)
    for dims in [(7, 6, 5), (9, 5, 6)]:
        d = small_case(*dims)
        bc = os.path.join(tmp, "topo.txt")
        write_case_file(d, bc)
        out = os.path.join(HERE, "topo_%dx%dx%d.txt" % dims)
        subprocess.run([REF, "--topo", bc, out], check=True)
    vtk_golden(tmp)
    for fn in os.listdir(tmp):
        os.remove(os.path.join(tmp, fn))
    os.rmdir(tmp)


VTK_STEPS = 12


def vtk_golden(tmp):
    """the reference's own legacy VTK file (Lattice::writeResultsVTK) of a
    9 x 7 x 5 single-level HRR case after 12 coarse steps, with its case file"""
    d = small_case(9, 7, 5)
    bc = os.path.join(tmp, "vtk_case.txt")
    write_case_file(d, bc, steps=VTK_STEPS)
    subprocess.run([REF, "--vtk", bc, str(VTK_STEPS), os.path.join(tmp, "ref")], check=True)
    with open(bc) as src, open(os.path.join(HERE, "vtk_9x7x5_case.txt"), "w") as dst:
        dst.write(src.read())
    os.replace(os.path.join(tmp, "ref.vtk"), os.path.join(HERE, "vtk_9x7x5_12steps.vtk"))


if __name__ == "__main__":
    main()
