"""The CPU oracle against the reference's own single-level runs.

The fixtures (tests/golden/single_level.json, single_level_rho.npz) were made
by tests/golden/make_golden.py from the reference built from its sources.  The
oracle restates the reference with the same floating-point evaluation order,
so the final population state must agree bit for bit (SHA-256 of the FP64
state) for every operator, equilibrium order, LODI variant and cubic-Mach
switch.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from acpulse_vclbm_b200.config import read_case_file

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "single_level.json")))
RHO = np.load(os.path.join(HERE, "golden", "single_level_rho.npz"))


def _case(c, tmp_path):
    p = tmp_path / "bc.txt"
    p.write_text(c["case_file"])
    return read_case_file(str(p))


@pytest.mark.parametrize("c", GOLD["cases"], ids=[c["name"] for c in GOLD["cases"]])
def test_oracle_bit_exact_vs_reference(c, tmp_path, oracle_lib):
    d = _case(c, tmp_path)
    assert [d.nx, d.ny, d.nz] == c["dims"]
    o = oracle_lib.OracleLattice(d, threads=4)
    o.init()
    o.step(c["steps"])
    f = o.populations()
    h = hashlib.sha256(f.astype("<f8").tobytes()).hexdigest()
    if h != c["sha256"]:
        # report how far off, to tell a rounding change from a logic error
        rho = f.sum(axis=0)
        err = np.abs(rho - RHO[c["name"]]).max()
        pytest.fail(f"state hash differs from the reference; max |drho| = {err:.3e}")
    np.testing.assert_array_equal(f.sum(axis=0), RHO[c["name"]])
