"""ctypes mirror of include/acp.h (the engine's C ABI).

The struct layout and enum values here must match include/acp.h exactly; the
CPU test suite checks the library's exported symbols against the header.
"""
import ctypes as C

ACP_OK = 0
ACP_ERR_INVALID = -1
ACP_ERR_CUDA = -2
ACP_ERR_NOMEM = -3
ACP_ERR_UNSUPPORTED = -4
ACP_ERR_NUMERIC = -5
ACP_ERR_TIMEOUT = -6
ACP_ERR_BUDGET = -7
ACP_ERR_STATE = -8

OPS = {"SRT": 0, "MRT-GS": 1, "MRT-RM": 2, "RR": 3, "HRR": 4}
OP_NAMES = {v: k for k, v in OPS.items()}
BC_LODI, BC_PERIODIC = 0, 1
STORAGE = {"FP64": 0, "FP32-DEV": 1, "FP16-DEV": 2}
COUPLING = {"STD": 0, "DC1": 1, "DC2": 2}
F2C_FILTER = {"NOFI": 0, "LAG": 1, "TOU": 2}
SCALING = {"SRTSTYLE": 0, "MRTSTYLE": 1}
C2F_REPLACE = {"Mf": 0, "MfP": 1, "fAll": 2}
F2C_REPLACE = {"Mc": 0, "McP": 1, "cAll": 2}
LAYOUT_SHELL, LAYOUT_BOX = 0, 1
IC_REFERENCE, IC_GAUSSIAN = 0, 1
FIELD_RHO, FIELD_UX, FIELD_UY, FIELD_UZ, FIELD_P = 0, 1, 2, 3, 4


class CaseDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("spacing", C.c_double),
        ("domain_size", C.c_double * 3),
        ("density", C.c_double), ("kinematic_viscosity", C.c_double),
        ("speed_of_sound", C.c_double), ("mach", C.c_double),
        ("op", C.c_int), ("eq_order", C.c_int), ("cubic_mach", C.c_int),
        ("hybrid_sigma", C.c_double),
        ("mrt_writeback", C.c_int),
        ("bc", C.c_int * 3),
        ("transverse", C.c_int),
        ("k1", C.c_double),
        ("max_level", C.c_int), ("layout", C.c_int),
        ("ref_layer_yz", C.c_int), ("ref_layer_x", C.c_int), ("overlap", C.c_int),
        ("box_lo", C.c_int * 3), ("box_hi", C.c_int * 3),
        ("coupling", C.c_int), ("f2c_filter", C.c_int), ("scaling_style", C.c_int),
        ("c2f_replace", C.c_int), ("f2c_replace", C.c_int),
        ("ic", C.c_int),
        ("ic_eps", C.c_double), ("ic_b", C.c_double),
        ("ic_center", C.c_double * 3),
        ("ic_dims", C.c_int),
        ("storage", C.c_int),
        ("lodi_length_nodes", C.c_int * 3),
        ("reserved", C.c_int * 5),
    ]

    def copy(self):
        c = CaseDesc()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(CaseDesc))
        return c


def default_case() -> CaseDesc:
    """The reference's shipped BoundaryConditions.txt values, single level."""
    d = CaseDesc()
    d.spacing = 2.0e-2
    d.domain_size[:] = [3.0, 3.0, 0.4]
    d.nx, d.ny, d.nz = 151, 151, 21
    d.density = 1.17621
    d.kinematic_viscosity = 1.49e-5
    d.speed_of_sound = 347.3
    d.mach = 0.0
    d.op = OPS["HRR"]
    d.eq_order = 3
    d.cubic_mach = 0
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 0
    d.bc[:] = [BC_LODI, BC_LODI, BC_LODI]
    d.transverse = 0
    d.k1 = 1.0
    d.max_level = 0
    d.layout = LAYOUT_SHELL
    d.ref_layer_yz, d.ref_layer_x, d.overlap = 4, 75, 1
    d.coupling = COUPLING["STD"]
    d.f2c_filter = F2C_FILTER["NOFI"]
    d.scaling_style = SCALING["SRTSTYLE"]
    d.c2f_replace = C2F_REPLACE["fAll"]
    d.f2c_replace = F2C_REPLACE["cAll"]
    d.ic = IC_REFERENCE
    d.ic_eps, d.ic_b = 1e-3, 6.0
    d.ic_dims = 2
    d.storage = STORAGE["FP64"]
    return d


def lattice_units_case(nx, ny, nz, op="SRT", nu_lu=1e-3, order=3, periodic=(False, True, True),
                       eps=1e-3, b=6.0, center=None, storage="FP64", ic_dims=2) -> CaseDesc:
    """A pulse case in lattice units: spacing 1, speed of sound 1/sqrt(3) (so the
    molecular velocity and time step are 1) and KinematicViscosity = nu in
    lattice units, giving tau = 0.5 + 3 nu (Control.cpp:52-54)."""
    d = default_case()
    d.nx, d.ny, d.nz = nx, ny, nz
    d.spacing = 1.0
    d.domain_size[:] = [nx - 0.5, ny - 0.5, nz - 0.5]
    d.density = 1.0
    d.speed_of_sound = 1.0 / 3.0 ** 0.5
    d.kinematic_viscosity = nu_lu
    d.op = OPS[op]
    d.eq_order = order
    d.bc[:] = [BC_PERIODIC if p else BC_LODI for p in periodic]
    d.ic = IC_GAUSSIAN
    d.ic_eps, d.ic_b = eps, b
    c = center if center is not None else ((nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0)
    d.ic_center[:] = list(c)
    d.ic_dims = ic_dims
    d.storage = STORAGE[storage]
    return d
