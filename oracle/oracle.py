"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, as the checker.  The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_PKG = _HERE.parent / "nim-conv22-shared_b200"
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))

from nimgpu import _abi  # noqa: E402

SEQUENTIAL = 0
PARALLEL = 1
LEVELS = 2        # SEQUENTIAL arithmetic, cells and wall faces in level order
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _HERE / "_build" / "libnim_oracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run make -C oracle")
        L = C.CDLL(str(path))
        vp = C.c_void_p
        L.nim_oracle_create.argtypes = [C.POINTER(_abi.MeshDesc), C.POINTER(_abi.Params), C.c_int32,
                                        C.c_int32, C.POINTER(vp)]
        L.nim_oracle_create.restype = C.c_int
        for n in ("nim_oracle_init", "nim_oracle_begin_step"):
            getattr(L, n).argtypes = [vp]
            getattr(L, n).restype = C.c_int
        L.nim_oracle_integrate.argtypes = [vp, C.POINTER(_abi.StepStats)]
        L.nim_oracle_integrate.restype = C.c_int
        L.nim_oracle_iterate.argtypes = [vp, C.c_int32, C.POINTER(_abi.StepStats)]
        L.nim_oracle_iterate.restype = C.c_int
        L.nim_oracle_end_step.argtypes = [vp, C.POINTER(_abi.StepStats)]
        L.nim_oracle_end_step.restype = C.c_int
        L.nim_oracle_step.argtypes = [vp, C.c_int32, C.POINTER(_abi.StepStats), C.POINTER(C.c_int32)]
        L.nim_oracle_step.restype = C.c_int
        L.nim_oracle_get.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.c_int64]
        L.nim_oracle_get.restype = C.c_int
        L.nim_oracle_set.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.c_int64]
        L.nim_oracle_set.restype = C.c_int
        L.nim_oracle_max_rc.argtypes = [vp]
        L.nim_oracle_max_rc.restype = C.c_double
        L.nim_oracle_destroy.argtypes = [vp]
        L.nim_oracle_destroy.restype = None
        L.nim_oracle_set_threads.argtypes = [vp, C.c_int32]
        L.nim_oracle_set_threads.restype = None
        L.nim_oracle_nim_coefficients.argtypes = [C.c_double] * 5 + [C.POINTER(C.c_double)]
        L.nim_oracle_nim_coefficients.restype = None
        _lib = L
    return _lib


class Oracle:
    """The reference algorithm on the CPU, one call per reference subroutine."""

    def __init__(self, mesh, params: _abi.Params, schedule: int = SEQUENTIAL, threads: int = 1):
        self.mesh = mesh
        self.params = params
        self._h = C.c_void_p()
        st = lib().nim_oracle_create(C.byref(mesh.desc), C.byref(params), schedule, threads,
                                     C.byref(self._h))
        _abi.check(st, "nim_oracle_create")

    def close(self):
        if self._h:
            lib().nim_oracle_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        _abi.check(lib().nim_oracle_init(self._h), "nim_oracle_init")

    def begin_step(self):
        _abi.check(lib().nim_oracle_begin_step(self._h), "nim_oracle_begin_step")

    def integrate(self) -> _abi.StepStats:
        s = _abi.StepStats()
        st = lib().nim_oracle_integrate(self._h, C.byref(s))
        s.status = st
        return s

    def iterate(self, n: int) -> _abi.StepStats:
        s = _abi.StepStats()
        _abi.check(lib().nim_oracle_iterate(self._h, n, C.byref(s)), "nim_oracle_iterate")
        return s

    def end_step(self) -> _abi.StepStats:
        s = _abi.StepStats()
        _abi.check(lib().nim_oracle_end_step(self._h, C.byref(s)), "nim_oracle_end_step")
        return s

    def step(self, n: int):
        arr = (_abi.StepStats * max(n, 1))()
        done = C.c_int32()
        st = lib().nim_oracle_step(self._h, n, arr, C.byref(done))
        return st, [arr[i] for i in range(done.value)]

    def get(self, field: int, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.float64)
        _abi.check(lib().nim_oracle_get(self._h, field, out.ctypes.data_as(C.POINTER(C.c_double)), n),
                   "nim_oracle_get")
        return out

    def set(self, field: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        _abi.check(lib().nim_oracle_set(self._h, field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
                   "nim_oracle_set")

    def set_threads(self, n: int):
        lib().nim_oracle_set_threads(self._h, n)

    def max_rc(self) -> float:
        return lib().nim_oracle_max_rc(self._h)


def nim1_coefficients(u: float, F: float, D: float, v_limit: float = 1e-2):
    """Formulation 1: B, C, E, F, G, H, I, J_nim of one direction (nim.f90:758-875)."""
    out = (C.c_double * 8)()
    lib().nim_oracle_nim1_coefficients(C.c_double(u), C.c_double(F), C.c_double(D), C.c_double(v_limit), out)
    return np.array(out[:])


def nim_coefficients(u: float, k: float, gminus: float = 1.0, gplus: float = 1.0, v_limit: float = 1e-2):
    """M_A(d,1:6) of one direction (nim.f90:181-287)."""
    A = (C.c_double * 6)()
    lib().nim_oracle_nim_coefficients(u, k, gminus, gplus, v_limit, A)
    return np.array(A[:])
