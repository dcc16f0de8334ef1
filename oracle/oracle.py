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
_tl_lib = None


def _bind(L: C.CDLL, pre: str):
    """argtypes of the time-advance entry points <pre>create ... <pre>set_threads."""
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)

    def sig(name, args, res=C.c_int):
        f = getattr(L, pre + name)
        f.argtypes, f.restype = args, res
    sig("create", [C.POINTER(_abi.MeshDesc), C.POINTER(_abi.Params), C.c_int32, C.c_int32, C.POINTER(vp)])
    sig("init", [vp])
    sig("begin_step", [vp])
    sig("integrate", [vp, C.POINTER(_abi.StepStats)])
    sig("iterate", [vp, C.c_int32, C.POINTER(_abi.StepStats)])
    sig("end_step", [vp, C.POINTER(_abi.StepStats)])
    sig("step", [vp, C.c_int32, C.POINTER(_abi.StepStats), C.POINTER(C.c_int32)])
    sig("get", [vp, C.c_int32, dp, C.c_int64])
    sig("set", [vp, C.c_int32, dp, C.c_int64])
    sig("max_rc", [vp], C.c_double)
    sig("destroy", [vp], None)
    sig("set_threads", [vp, C.c_int32], None)
    sig("nim_coefficients", [C.c_double] * 5 + [dp], None)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _HERE / "_build" / "libnim_oracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run make -C oracle")
        L = C.CDLL(str(path))
        _bind(L, "nim_oracle_")
        ip = C.POINTER(C.c_int32)
        L.nim_oracle_mesh_build.argtypes = [C.POINTER(_abi.MeshParams), C.POINTER(C.c_double)] + [ip] * 8
        L.nim_oracle_mesh_build.restype = C.c_int
        _lib = L
    return _lib


def tl_lib() -> C.CDLL:
    """The tangent-linear build (nim_oracle_tl.cpp): dual-number values."""
    global _tl_lib
    if _tl_lib is None:
        path = _HERE / "_build" / "libnim_oracle_tl.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run make -C oracle")
        L = C.CDLL(str(path))
        _bind(L, "nim_oracle_tl_")
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.nim_oracle_tl_seed_params.argtypes = [vp, C.c_double, C.c_double]
        L.nim_oracle_tl_seed_params.restype = C.c_int
        for n in ("get_tangent", "set_tangent"):
            getattr(L, "nim_oracle_tl_" + n).argtypes = [vp, C.c_int32, dp, C.c_int64]
            getattr(L, "nim_oracle_tl_" + n).restype = C.c_int
        L.nim_oracle_tl_nu_tangent.argtypes = [vp, dp]
        L.nim_oracle_tl_nu_tangent.restype = C.c_int
        _tl_lib = L
    return _tl_lib


class OracleMesh:
    """The cylinder mesh built by the oracle's own restatement of the
    reference's mesh set-up (nim_oracle_mesh_build), with the attributes of
    nimgpu.Mesh; loads no product library."""

    def __init__(self, mp: _abi.MeshParams):
        n1, n2, n3 = mp.n_theta, mp.n_r, mp.n_z
        self.params = mp
        self.n_theta, self.n_r, self.n_z = n1, n2, n3
        self.nnode = n1 * (n2 + 1) * (n3 + 1)          # parameters.f90:119
        self.nmesh = n1 * n2 * n3
        self.nface = 3 * n1 * n2 * n3 + n1 * n3 + n1 * n2  # parameters.f90:117
        self.nbcface = 2 * n1 * n2 + 2 * n1 * n3
        self.node_xyz = np.zeros((self.nnode, 3), dtype=np.float64)
        self.meshes_nodes = np.zeros((self.nmesh, 8), dtype=np.int32)
        self.meshes_faces = np.zeros((self.nmesh, 6), dtype=np.int32)
        self.meshes_neighbors = np.zeros((self.nmesh, 6), dtype=np.int32)
        self.faces_bc = np.zeros(self.nface, dtype=np.int32)
        self.bcs_faces = np.zeros(self.nbcface, dtype=np.int32)
        self.bcs_faces_id = np.zeros(self.nbcface, dtype=np.int32)
        self.bcs_faces_position = np.zeros(self.nbcface, dtype=np.int32)
        self.bcs_faces_mesh_num = np.zeros(self.nbcface, dtype=np.int32)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
        st = lib().nim_oracle_mesh_build(
            C.byref(mp), self.node_xyz.ctypes.data_as(C.POINTER(C.c_double)), ip(self.meshes_nodes),
            ip(self.meshes_faces), ip(self.meshes_neighbors), ip(self.faces_bc), ip(self.bcs_faces),
            ip(self.bcs_faces_id), ip(self.bcs_faces_position), ip(self.bcs_faces_mesh_num))
        if st != 0:
            raise ValueError("nim_oracle_mesh_build: bad mesh parameters")
        d = _abi.MeshDesc()
        d.n_theta, d.n_r, d.n_z = n1, n2, n3
        d.nnode, d.nmesh, d.nface, d.nbcface = self.nnode, self.nmesh, self.nface, self.nbcface
        d.node_xyz = self.node_xyz.ctypes.data_as(C.POINTER(C.c_double))
        for name in ("meshes_nodes", "meshes_faces", "meshes_neighbors", "faces_bc", "bcs_faces", "bcs_faces_id",
                     "bcs_faces_position", "bcs_faces_mesh_num"):
            setattr(d, name, ip(getattr(self, name)))
        self.desc = d

    @property
    def interior_faces(self) -> np.ndarray:
        return self.faces_bc == 1


def temperature_noise(mesh, amp: float, seed: int):
    """The benchmark cases' seeded U(-amp, amp) initial-temperature noise,
    one value per cell and per interior face (the same draws as the
    library's host helper, so both sides start from the same state)."""
    rng = np.random.default_rng(seed)
    cells = rng.uniform(-amp, amp, size=mesh.nmesh)
    faces = rng.uniform(-amp, amp, size=mesh.nface)
    faces[~mesh.interior_faces] = 0.0
    return cells, faces


class Oracle:
    """The reference algorithm on the CPU, one call per reference subroutine."""

    _pre = "nim_oracle_"

    def _lib(self) -> C.CDLL:
        return lib()

    def _f(self, name: str):
        return getattr(self._lib(), self._pre + name)

    def __init__(self, mesh, params: _abi.Params, schedule: int = SEQUENTIAL, threads: int = 1):
        self.mesh = mesh
        self.params = params
        self._h = C.c_void_p()
        st = self._f("create")(C.byref(mesh.desc), C.byref(params), schedule, threads, C.byref(self._h))
        _abi.check(st, self._pre + "create")

    def close(self):
        if self._h:
            self._f("destroy")(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        _abi.check(self._f("init")(self._h), "init")

    def begin_step(self):
        _abi.check(self._f("begin_step")(self._h), "begin_step")

    def integrate(self) -> _abi.StepStats:
        s = _abi.StepStats()
        st = self._f("integrate")(self._h, C.byref(s))
        s.status = st
        return s

    def iterate(self, n: int) -> _abi.StepStats:
        s = _abi.StepStats()
        _abi.check(self._f("iterate")(self._h, n, C.byref(s)), "iterate")
        return s

    def end_step(self) -> _abi.StepStats:
        s = _abi.StepStats()
        _abi.check(self._f("end_step")(self._h, C.byref(s)), "end_step")
        return s

    def step(self, n: int):
        arr = (_abi.StepStats * max(n, 1))()
        done = C.c_int32()
        st = self._f("step")(self._h, n, arr, C.byref(done))
        return st, [arr[i] for i in range(done.value)]

    def get(self, field: int, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.float64)
        _abi.check(self._f("get")(self._h, field, out.ctypes.data_as(C.POINTER(C.c_double)), n), "get")
        return out

    def set(self, field: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        _abi.check(self._f("set")(self._h, field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size), "set")

    def add_temperature_noise(self, amp: float, seed: int):
        """The seeded initial-temperature noise of the benchmark cases."""
        if amp == 0.0:
            return
        cells, faces = temperature_noise(self.mesh, amp, seed)
        self.set(_abi.FACES_T, self.get(_abi.FACES_T, self.mesh.nface) + faces)
        for f in (_abi.MESHES_T, _abi.MESHES_T_OLD, _abi.MESHES_TT):
            self.set(f, self.get(f, self.mesh.nmesh) + cells)

    def set_threads(self, n: int):
        self._f("set_threads")(self._h, n)

    def max_rc(self) -> float:
        return self._f("max_rc")(self._h)


class TangentOracle(Oracle):
    """The oracle's tangent-linear build: the FP64 oracle's values bit for
    bit, and along one seeded direction their derivatives.  Seeds: d nu and
    d alpha (seed_params; with_respect_to gives the seeds of Ra and Pr), and
    the derivatives of the state fields (set_tangent after init(): e.g. the
    outer-wall Dirichlet faces of faces_T)."""

    _pre = "nim_oracle_tl_"

    def _lib(self) -> C.CDLL:
        return tl_lib()

    def seed_params(self, dnu: float, dalpha: float):
        _abi.check(self._f("seed_params")(self._h, dnu, dalpha), "seed_params")

    @staticmethod
    def with_respect_to(name: str, Ra: float, Pr: float):
        """(d nu, d alpha) for d/dRa or d/dPr: nu = sqrt(Pr / Ra), alpha =
        nu / Pr (parameters.f90:169-173 with g_beta = th_tc = 1)."""
        nu = (Pr / Ra) ** 0.5
        alpha = nu / Pr
        if name == "Ra":
            return -nu / (2 * Ra), -alpha / (2 * Ra)
        if name == "Pr":
            return nu / (2 * Pr), -alpha / (2 * Pr)
        raise ValueError(name)

    def get_tangent(self, field: int, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.float64)
        _abi.check(self._f("get_tangent")(self._h, field, out.ctypes.data_as(C.POINTER(C.c_double)), n),
                   "get_tangent")
        return out

    def set_tangent(self, field: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        _abi.check(self._f("set_tangent")(self._h, field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
                   "set_tangent")

    def nu_tangent(self):
        """(d Nu_inner, d Nu_outer) of the last end_step."""
        out = np.zeros(2, dtype=np.float64)
        _abi.check(self._f("nu_tangent")(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "nu_tangent")
        return float(out[0]), float(out[1])


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
