"""Python binding of the engine's C ABI (include/acp.h) for tests, tools and
bench.py.  The binding loads the in-tree libacp_cuda.so; there is no other
implementation behind it, so every call fails loudly when the library or a
CUDA device is missing.
"""
import ctypes as C
import os

import numpy as np

from .capi import ACP_OK, CaseDesc

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libacp_cuda.so")
_LIB = None


class AcpError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"acp status {status}: {message}")
        self.status = status


def lib():
    """Load libacp_cuda.so (building it first when it is absent)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            from .build import build
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.acp_default_case.argtypes = [C.POINTER(CaseDesc)]
        L.acp_default_case.restype = None
        L.acp_parse_case_file.argtypes = [C.c_char_p, C.POINTER(CaseDesc), C.c_char_p, C.c_size_t]
        L.acp_create.argtypes = [C.POINTER(CaseDesc), C.c_int, C.POINTER(vp)]
        for name in ["acp_init", "acp_sync", "acp_destroy"]:
            getattr(L, name).argtypes = [vp]
        L.acp_step.argtypes = [vp, C.c_int]
        L.acp_level_dims.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        L.acp_active_updates.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.acp_read_populations.argtypes = [vp, C.c_int, vp]
        L.acp_read_populations_other.argtypes = [vp, C.c_int, vp]
        L.acp_get_columns.argtypes = [vp, C.c_int, C.c_int, vp]
        L.acp_put_columns.argtypes = [vp, C.c_int, C.c_int, vp]
        L.acp_copy_columns.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int]
        L.acp_write_populations.argtypes = [vp, C.c_int, vp]
        L.acp_read_field.argtypes = [vp, C.c_int, C.c_int, vp]
        L.acp_set_probes.argtypes = [vp, C.c_int, vp]
        L.acp_read_probes.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_int)]
        L.acp_steps_done.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.acp_checkpoint_save.argtypes = [vp, C.c_char_p]
        L.acp_checkpoint_load.argtypes = [vp, C.c_char_p]
        L.acp_write_vtk.argtypes = [vp, C.c_char_p, C.c_int]
        L.acp_set_stream.argtypes = [vp, vp]
        L.acp_device_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
        L.acp_estimate_bytes.argtypes = [C.POINTER(CaseDesc), C.POINTER(C.c_size_t)]
        L.acp_last_error.argtypes = [vp]
        L.acp_last_error.restype = C.c_char_p
        L.acp_status_string.argtypes = [C.c_int]
        L.acp_status_string.restype = C.c_char_p
        L.acp_abi_version.restype = C.c_int
        L.acp_batch_create.argtypes = [vp, C.c_int, C.POINTER(vp)]
        L.acp_batch_step.argtypes = [vp, C.c_int]
        L.acp_batch_sync.argtypes = [vp]
        L.acp_batch_tune.argtypes = [vp, C.c_int, C.c_char_p, C.c_size_t]
        L.acp_batch_configure.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.acp_batch_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        L.acp_batch_destroy.argtypes = [vp]
        L.acp_batch_last_error.argtypes = [vp]
        L.acp_batch_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def parse_case_file(path: str) -> CaseDesc:
    d = CaseDesc()
    err = C.create_string_buffer(512)
    s = lib().acp_parse_case_file(path.encode(), C.byref(d), err, 512)
    if s != ACP_OK:
        raise AcpError(s, err.value.decode())
    return d


def estimate_bytes(desc: CaseDesc) -> int:
    b = C.c_size_t(0)
    s = lib().acp_estimate_bytes(C.byref(desc), C.byref(b))
    if s != ACP_OK:
        raise AcpError(s, lib().acp_status_string(s).decode())
    return b.value


class Lattice:
    """One solve on the GPU: acp_create / acp_init / acp_step / reads."""

    def __init__(self, desc: CaseDesc, device: int = -1):
        self.desc = desc.copy()
        self._h = C.c_void_p()
        s = lib().acp_create(C.byref(self.desc), device, C.byref(self._h))
        if s != ACP_OK:
            msg = lib().acp_last_error(self._h).decode() if self._h else ""
            self.close()
            raise AcpError(s, msg)

    def _check(self, s):
        if s != ACP_OK:
            raise AcpError(s, lib().acp_last_error(self._h).decode())

    def init(self):
        self._check(lib().acp_init(self._h))
        return self

    def step(self, n=1):
        self._check(lib().acp_step(self._h, n))

    def sync(self):
        self._check(lib().acp_sync(self._h))

    def dims(self, level=0):
        d = (C.c_int * 3)()
        self._check(lib().acp_level_dims(self._h, level, d))
        return tuple(d)

    def active_updates(self):
        c, f = C.c_longlong(), C.c_longlong()
        self._check(lib().acp_active_updates(self._h, C.byref(c), C.byref(f)))
        return c.value, f.value

    def populations(self, level=0, other=False):
        """FP64 f_i of a level, (19, nz, ny, nx): the current state, or with
        other=True the level's other ping-pong array (acp_read_populations_other)"""
        nx, ny, nz = self.dims(level)
        out = np.empty((19, nz, ny, nx), dtype=np.float64)
        fn = lib().acp_read_populations_other if other else lib().acp_read_populations
        self._check(fn(self._h, level, out.ctypes.data))
        return out

    def write_populations(self, f, level=0):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self._check(lib().acp_write_populations(self._h, level, f.ctypes.data))

    def field(self, which, level=0, out=None):
        """FP64 field `which` (ACP_FIELD_*) of a level as an (nz, ny, nx)
        array; `out`, if given, is filled instead (C-contiguous float64 of that
        shape -- a page-locked buffer makes the copy a direct DMA)"""
        nx, ny, nz = self.dims(level)
        if out is None:
            out = np.empty((nz, ny, nx), dtype=np.float64)
        elif out.shape != (nz, ny, nx) or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"field output must be C-contiguous float64 of shape {(nz, ny, nx)}")
        self._check(lib().acp_read_field(self._h, level, which, out.ctypes.data))
        return out

    def set_probes(self, probes):
        arr = np.ascontiguousarray(np.asarray(probes, dtype=np.int32).reshape(-1, 4))
        self._check(lib().acp_set_probes(self._h, len(arr), arr.ctypes.data))
        self._nprobes = len(arr)

    def probes(self, max_samples=1 << 16):
        n = C.c_int(0)
        out = np.empty((max_samples, max(self._nprobes, 1)), dtype=np.float64)
        self._check(lib().acp_read_probes(self._h, out.ctypes.data, max_samples, C.byref(n)))
        return out[: n.value, : self._nprobes]

    def steps_done(self):
        s = C.c_longlong()
        self._check(lib().acp_steps_done(self._h, C.byref(s)))
        return s.value

    def write_vtk(self, prefix, binary=False):
        """Legacy VTK files of every level (acp_write_vtk): ASCII as the reference writes them, or binary."""
        self._check(lib().acp_write_vtk(self._h, os.fsencode(prefix), 1 if binary else 0))

    def save_checkpoint(self, path):
        """Write the case's complete device state to `path` (acp_checkpoint_save)."""
        self._check(lib().acp_checkpoint_save(self._h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Restore a state written by save_checkpoint into this initialised case."""
        self._check(lib().acp_checkpoint_load(self._h, os.fsencode(path)))
        return self

    def device_bytes(self):
        b = C.c_size_t()
        self._check(lib().acp_device_bytes(self._h, C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            if getattr(self, "_batch", None) is not None:
                self._batch.close()
            lib().acp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Initialised lattices advanced together (acp_batch_*): one CUDA graph
    per coarse step, every phase one persistent launch per group of cases
    with the same kernels.  The lattices stay readable; they are stepped
    only through the batch until it is closed."""

    def __init__(self, lattices):
        self.lattices = list(lattices)
        arr = (C.c_void_p * len(self.lattices))(*[L._h.value for L in self.lattices])
        self._b = C.c_void_p()
        s = lib().acp_batch_create(arr, len(self.lattices), C.byref(self._b))
        if s != ACP_OK:
            msg = lib().acp_batch_last_error(self._b).decode() if self._b else ""
            self.close()
            raise AcpError(s, msg)
        for L in self.lattices:
            L._batch = self

    def _check(self, s):
        if s != ACP_OK:
            raise AcpError(s, lib().acp_batch_last_error(self._b).decode())

    def step(self, n=1):
        self._check(lib().acp_batch_step(self._b, n))

    def sync(self):
        self._check(lib().acp_batch_sync(self._b))

    def tune(self, trial_steps=5):
        """Time every candidate schedule over trial_steps real coarse steps
        each (the cases advance) and keep the fastest; returns the report."""
        rep = C.create_string_buffer(4096)
        self._check(lib().acp_batch_tune(self._b, trial_steps, rep, 4096))
        return rep.value.decode()

    def configure(self, persist=0, largest_first=False, chunk_scale=1):
        self._check(lib().acp_batch_configure(self._b, persist, int(largest_first), chunk_scale))

    def info(self):
        g, l, u = C.c_int(), C.c_int(), C.c_longlong()
        self._check(lib().acp_batch_info(self._b, C.byref(g), C.byref(l), C.byref(u)))
        return {"groups": g.value, "launches_per_step": l.value, "updates_per_step": u.value}

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            lib().acp_batch_destroy(self._b)
            self._b = C.c_void_p()
            for L in self.lattices:
                L._batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
