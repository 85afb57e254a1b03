"""BoundaryConditions.txt reading and writing.

The reference reads its case from a keyword file (Control.cpp:8-37): each line
is "<Keyword> <value>", the first whitespace-separated token must equal the
keyword exactly, the value is read with stream extraction (so a trailing ';'
or comment after the number is ignored), and a missing mandatory keyword is
fatal (Control.cpp:163-164).  This module mirrors those rules in Python for
tests and tools; the engine's C parser (acp_parse_case_file) applies the same
rules.  Keywords this engine adds are optional and keep the reference's
behaviour when absent.
"""
import math
import re

from .capi import (BC_LODI, BC_PERIODIC, C2F_REPLACE, COUPLING, F2C_FILTER, F2C_REPLACE, IC_GAUSSIAN,
                   IC_REFERENCE, LAYOUT_BOX, LAYOUT_SHELL, OPS, OP_NAMES, SCALING, STORAGE, CaseDesc, default_case)

_INV = lambda m: {v: k for k, v in m.items()}  # noqa: E731


def write_case_file(d: CaseDesc, path: str, steps: int = 100, threads: int = 8) -> None:
    """Write a BoundaryConditions.txt that the reference (and this engine) reads as `d`."""
    lines = [
        f"Max-Time-Step {steps}",
        "WriteInterval 1000000000",
        "Save-as /tmp/acp_unused",
        f"Threads {threads}",
        f"Density {d.density!r}",
        f"KinematicViscosity {d.kinematic_viscosity!r}",
        f"SpeedOfSound {d.speed_of_sound!r}",
        f"MACH-Number {d.mach!r}",
        f"Order-Of-Equilibrium {d.eq_order}",
        f"Collision-Model {OP_NAMES[d.op]}",
        f"Hybrid-Parameter {d.hybrid_sigma!r}",
        f"Cubic-Mach-Correction {'yes' if d.cubic_mach else 'no'}",
        f"Coupling-Approach {_INV(COUPLING)[d.coupling]}",
        "Non-Reflecting yes",
        f"Transverse {'yes' if d.transverse else 'no'}",
        f"K1-Relaxation {d.k1!r}",
        "K2-Relaxation 1.0",
        f"F2C-Filter {_INV(F2C_FILTER)[d.f2c_filter]}",
        f"Coarse-to-Fine {_INV(C2F_REPLACE)[d.c2f_replace]}",
        f"Fine-to-Coarse {_INV(F2C_REPLACE)[d.f2c_replace]}",
        "Hanging-Node-Reconstruction hAll",
        f"Scaling-Style {_INV(SCALING)[d.scaling_style]}",
        f"Domain-Size-X {d.domain_size[0]!r}",
        f"Domain-Size-Y {d.domain_size[1]!r}",
        f"Domain-Size-Z {d.domain_size[2]!r}",
        f"Spacing {d.spacing!r}",
        f"MaxLevel {d.max_level}",
        f"RefinementLayerYZ {d.ref_layer_yz}",
        f"RefinementLayerX {d.ref_layer_x}",
        f"Overlap {d.overlap}",
    ]
    # optional keywords of this engine (ignored by the reference)
    ext = []
    for a, name in enumerate("XYZ"):
        if d.bc[a] == BC_PERIODIC:
            ext.append(f"Periodic-{name} yes")
    if d.mrt_writeback:
        ext.append("MRT-Write-Back yes")
    if d.storage:
        ext.append(f"Storage {_INV(STORAGE)[d.storage]}")
    if d.layout == LAYOUT_BOX:
        ext.append("Refinement-Layout BOX")
        ext.append("Refinement-Box-Lo " + " ".join(str(v) for v in d.box_lo))
        ext.append("Refinement-Box-Hi " + " ".join(str(v) for v in d.box_hi))
    if d.ic == IC_GAUSSIAN:
        ext.append(f"Pulse-Amplitude {d.ic_eps!r}")
        ext.append(f"Pulse-Halfwidth {d.ic_b!r}")
        ext.append("Pulse-Center " + " ".join(repr(v) for v in d.ic_center))
        ext.append(f"Pulse-Dimensions {d.ic_dims}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines + ext) + "\n")


def _first_token_lines(path):
    with open(path) as fh:
        for line in fh:
            toks = line.split()
            if toks:
                yield toks[0], line


def _value(path, key, required=True, default=None):
    for tok, line in _first_token_lines(path):
        if tok == key:
            rest = line.split(None, 1)[1] if len(line.split(None, 1)) > 1 else ""
            return rest
    if required:
        raise KeyError(f'No Value for keyword "{key}" found in {path}')
    return default


def _num(s):
    m = re.match(r"\s*([-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?)", s)
    if not m:
        return 0.0
    return float(m.group(1))


def _word(s):
    toks = s.split()
    return toks[0] if toks else ""


def read_case_file(path: str) -> CaseDesc:
    """Parse a BoundaryConditions.txt with the reference's keyword rules."""
    d = default_case()
    d.density = _num(_value(path, "Density"))
    d.kinematic_viscosity = _num(_value(path, "KinematicViscosity"))
    d.speed_of_sound = _num(_value(path, "SpeedOfSound"))
    d.mach = _num(_value(path, "MACH-Number"))
    d.eq_order = int(_num(_value(path, "Order-Of-Equilibrium")))
    d.op = OPS[_word(_value(path, "Collision-Model"))]
    d.hybrid_sigma = _num(_value(path, "Hybrid-Parameter"))
    d.cubic_mach = 1 if _word(_value(path, "Cubic-Mach-Correction")) == "yes" else 0
    d.coupling = COUPLING[_word(_value(path, "Coupling-Approach"))]
    d.transverse = 1 if _word(_value(path, "Transverse")) == "yes" else 0
    d.k1 = _num(_value(path, "K1-Relaxation"))
    d.f2c_filter = F2C_FILTER[_word(_value(path, "F2C-Filter"))]
    d.c2f_replace = C2F_REPLACE[_word(_value(path, "Coarse-to-Fine"))]
    d.f2c_replace = F2C_REPLACE[_word(_value(path, "Fine-to-Coarse"))]
    d.scaling_style = SCALING[_word(_value(path, "Scaling-Style"))]
    for a, name in enumerate("XYZ"):
        d.domain_size[a] = _num(_value(path, f"Domain-Size-{name}"))
    d.spacing = _num(_value(path, "Spacing"))
    d.max_level = int(_num(_value(path, "MaxLevel")))
    d.ref_layer_yz = int(_num(_value(path, "RefinementLayerYZ")))
    d.ref_layer_x = int(_num(_value(path, "RefinementLayerX")))
    d.overlap = int(_num(_value(path, "Overlap")))
    eps = 1e-8  # Control.cpp:40-45
    d.nx = int(math.ceil(d.domain_size[0] / d.spacing + eps))
    d.ny = int(math.ceil(d.domain_size[1] / d.spacing + eps))
    d.nz = int(math.ceil(d.domain_size[2] / d.spacing + eps))
    for a, name in enumerate("XYZ"):
        d.bc[a] = BC_PERIODIC if _word(_value(path, f"Periodic-{name}", False, "no")) == "yes" else BC_LODI
    d.mrt_writeback = 1 if _word(_value(path, "MRT-Write-Back", False, "no")) == "yes" else 0
    d.storage = STORAGE[_word(_value(path, "Storage", False, "FP64"))]
    if _word(_value(path, "Refinement-Layout", False, "SHELL")) == "BOX":
        d.layout = LAYOUT_BOX
        d.box_lo[:] = [int(v) for v in _value(path, "Refinement-Box-Lo").split()[:3]]
        d.box_hi[:] = [int(v) for v in _value(path, "Refinement-Box-Hi").split()[:3]]
    amp = _value(path, "Pulse-Amplitude", False, None)
    if amp is not None:
        d.ic = IC_GAUSSIAN
        d.ic_eps = _num(amp)
        d.ic_b = _num(_value(path, "Pulse-Halfwidth"))
        d.ic_center[:] = [float(v) for v in _value(path, "Pulse-Center").split()[:3]]
        d.ic_dims = int(_num(_value(path, "Pulse-Dimensions", False, "2")))
    else:
        d.ic = IC_REFERENCE
    return d
