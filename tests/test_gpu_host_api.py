"""The drop-in C++ Control/Lattice classes and the reference-style driver
(acpulse_vclbm_b200/acp_main, built from host/*.cpp) on the reference's own
case files: the density field read back through Lattice::getDistribution
must match the reference's golden runs (same tolerance as the FP64 parity
tests: 1e-9 of the pulse amplitude)."""
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MAIN = os.path.join(ROOT, "acpulse_vclbm_b200", "acp_main")
GOLD = json.load(open(os.path.join(HERE, "golden", "single_level.json")))
RHO = np.load(os.path.join(HERE, "golden", "single_level_rho.npz"))

pytestmark = pytest.mark.gpu

CASES = [c for c in GOLD["cases"] if c["name"] in (
    "SRT_o3_t1_c0_s200_nu0.024", "HRR_o4_t1_c1_s30_nu0.024", "MRT-GS_o2_t0_c0_s30_nu0.024",
    "HRR_o3_t0_c0_s40_nu1.49e-05")]


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_driver_matches_reference(c, tmp_path):
    bc = tmp_path / "BoundaryConditions.txt"
    bc.write_text(c["case_file"])
    out = tmp_path / "rho.bin"
    r = subprocess.run([MAIN, str(bc), str(c["steps"]), "--dump-rho", str(out), "--no-vtk"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    nx, ny, nz = c["dims"]
    rho = np.fromfile(out, dtype=np.float64).reshape(nz, ny, nx)
    err = np.abs(rho - RHO[c["name"]]).max() / (0.01 * 1.17621)
    assert err < 1e-9, err


def test_driver_writes_vtk(tmp_path):
    c = CASES[0]
    text = c["case_file"].replace("Save-as /tmp/acp_unused", f"Save-as {tmp_path}/pulse")
    text = text.replace("WriteInterval 1000000000", "WriteInterval 5")
    bc = tmp_path / "BoundaryConditions.txt"
    bc.write_text(text)
    r = subprocess.run([MAIN, str(bc), "10"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    vtk = open(tmp_path / "pulse_10.vtk").read()
    assert "DATASET STRUCTURED_POINTS" in vtk and "SCALARS Pressure" in vtk
