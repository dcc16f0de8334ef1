"""Builds and loads tests/exp_harness.cpp (host libm exp and the host build
of nim_exp side by side) for the exp tests."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "nim-conv22-shared_b200" / "csrc"


def build(dirpath: Path) -> C.CDLL:
    so = Path(dirpath) / "libexp_harness.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=c++17",
                    "-I", str(CSRC), str(ROOT / "tests" / "exp_harness.cpp"), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    dp = C.POINTER(C.c_double)
    for n in ("libm_exp_batch", "nim_exp_batch"):
        getattr(L, n).argtypes = [dp, dp, C.c_long]
        getattr(L, n).restype = None
    L.make_args.argtypes = [dp, C.c_long, C.c_uint64, C.c_int, C.c_double, C.c_double]
    L.make_args.restype = None
    L.count_mismatch.argtypes = [C.c_long, C.c_uint64, C.c_int, C.c_double, C.c_double]
    L.count_mismatch.restype = C.c_long
    return L


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def args(L, n: int, seed: int, kind: int = 0, lo: float = 1e-2, hi: float = 50.0) -> np.ndarray:
    x = np.empty(n, dtype=np.float64)
    L.make_args(ptr(x), n, seed, kind, lo, hi)
    return x


def libm_exp(L, x: np.ndarray) -> np.ndarray:
    y = np.empty_like(x)
    L.libm_exp_batch(ptr(x), ptr(y), x.size)
    return y
