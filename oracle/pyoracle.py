"""ctypes wrapper of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, to check the engine's results.  The engine never
calls it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from acpulse_vclbm_b200.capi import CaseDesc

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile oracle/liboracle.so (and, where the reference's sources are
    present, its single-level binary oracle/_ref/acp_ref).  The sources are
    found at the recipe's default location (oracle/ref_build/Makefile, REF) or
    at $ACP_REFERENCE_SRC."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    ref = os.environ.get("ACP_REFERENCE_SRC")
    cmd = ["make", "-s", "-C", os.path.join(_HERE, "ref_build")] + ([f"REF={ref}"] if ref else [])
    if subprocess.run(cmd + ["have-ref"], capture_output=True).returncode == 0:
        subprocess.run(cmd, check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(CaseDesc), C.c_int, C.c_char_p, C.c_int]
        L.orc_init.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_dims.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.orc_read_populations.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_write_populations.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_write_current.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_steps_done.restype = C.c_longlong
        L.orc_steps_done.argtypes = [C.c_void_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_probe_pressures.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        _LIB = L
    return _LIB


class OracleLattice:
    """FP64 CPU oracle of one case; same call pattern as the engine."""

    def __init__(self, desc: CaseDesc, threads: int = 0):
        err = C.create_string_buffer(256)
        self._h = lib().orc_create(C.byref(desc), threads, err, 256)
        if not self._h:
            raise ValueError(err.value.decode())
        self.desc = desc

    def init(self):
        lib().orc_init(self._h)

    def step(self, n=1):
        lib().orc_step(self._h, n)

    def dims(self, level=0):
        d = (C.c_int * 3)()
        if lib().orc_dims(self._h, level, d) != 0:
            raise ValueError("no such level")
        return tuple(d)

    def populations(self, level=0):
        nx, ny, nz = self.dims(level)
        out = np.empty((19, nz, ny, nx), dtype=np.float64)
        lib().orc_read_populations(self._h, level, out.ctypes.data)
        return out

    def probe_series(self, probes, steps):
        """pressure at probes (level, i, j, k) after each of `steps` coarse steps: [steps, n]"""
        arr = np.ascontiguousarray(np.asarray(probes, dtype=np.int32).reshape(-1, 4))
        out = np.empty((steps, len(arr)), dtype=np.float64)
        for s in range(steps):
            self.step(1)
            if lib().orc_probe_pressures(self._h, len(arr), arr.ctypes.data, out[s].ctypes.data) != 0:
                raise ValueError("probe outside its level")
        return out

    def write_populations(self, f, level=0, current_only=False):
        """FP64 f_i of a level into both arrays, or the current one only"""
        f = np.ascontiguousarray(f, dtype=np.float64)
        fn = lib().orc_write_current if current_only else lib().orc_write_populations
        fn(self._h, level, f.ctypes.data)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
