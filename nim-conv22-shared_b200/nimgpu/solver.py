"""Python host mirror of the reference's solver interface over the C ABI.

Method names follow the reference subroutines a Fortran host calls
(solve_nse, nse.f90:23-85); each one is a single call into libnimgpu.so.
There is no CPU path: without the CUDA library or a GPU the constructor
raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .mesh import Mesh, apply_temperature_noise


def field_len(field: int, mesh: Mesh) -> int:
    nf, nm, nb = mesh.nface, mesh.nmesh, mesh.nbcface
    table = {
        _abi.FACES_AREA: nf, _abi.FACES_NORMAL: 3 * nf, _abi.FACES_MID: 3 * nf,
        _abi.FACES_TANGENTIAL: 3 * nf, _abi.FACES_BITANGENTIAL: 3 * nf,
        _abi.MESHES_VOLUME: nm, _abi.MESHES_GIJ: 9 * nm, _abi.MESHES_XI_X: 9 * nm,
        _abi.MESHES_G: 3 * nm, _abi.MESHES_GIJ_FACES: 54 * nm,
        _abi.BCS_FACES_A: 5 * nb, _abi.BCS_FACES_AP: 8 * nb,
        _abi.AA_PX: 15 * nm, _abi.AA_PY: 15 * nm, _abi.AA_PZ: 15 * nm,
        _abi.M_F4: 8 * nm, _abi.M_F1: 5 * nm, _abi.M_F2: 5 * nm, _abi.M_F3: 5 * nm,
    }
    if field in table:
        return table[field]
    if field <= _abi.FACES_T:
        return nf
    if field <= _abi.MESHES_DILA_OLD:
        return nm
    raise ValueError(f"unknown field {field}")


class NimSolver:
    """One device-resident NIM context (include/nim_gpu.h)."""

    def __init__(self, mesh: Mesh, params: _abi.Params):
        self.lib = _abi.gpu_lib()
        self.mesh = mesh
        self.params = params
        self._h = C.c_void_p()
        _abi.check(self.lib.nim_gpu_create(C.byref(mesh.desc), C.byref(params), C.byref(self._h)),
                   "nim_gpu_create")

    # -- lifetime
    def close(self):
        if self._h:
            self.lib.nim_gpu_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's call sites (nse.f90:34-73)
    def initialize_nse(self):
        """initialize_nse + apply_all_dirichlet_bcs (nse.f90:34-38)."""
        _abi.check(self.lib.nim_gpu_init(self._h), "nim_gpu_init")

    def calculate_velocity_nim_constants(self):
        """calculate_velocity_nim_constants_formulation2 (nse.f90:52)."""
        _abi.check(self.lib.nim_gpu_begin_step(self._h), "nim_gpu_begin_step")

    def integrate_nse(self, raise_on_error: bool = True) -> _abi.StepStats:
        """integrate_nse (nse.f90:57) with the max_iters guard."""
        s = _abi.StepStats()
        st = self.lib.nim_gpu_integrate(self._h, C.byref(s))
        s.status = st
        if raise_on_error:
            _abi.check(st, "nim_gpu_integrate")
        return s

    def iterate(self, n: int) -> _abi.StepStats:
        """Exactly n inner passes without the stop test."""
        s = _abi.StepStats()
        _abi.check(self.lib.nim_gpu_iterate(self._h, n, C.byref(s)), "nim_gpu_iterate")
        return s

    def update_time_step(self) -> _abi.StepStats:
        """update_time_step + find_Nu2 (nse.f90:72-73)."""
        s = _abi.StepStats()
        _abi.check(self.lib.nim_gpu_end_step(self._h, C.byref(s)), "nim_gpu_end_step")
        return s

    def solve_nse(self, nsteps: int, raise_on_error: bool = True):
        """nsteps of the time loop (nse.f90:47-75); returns per-step stats."""
        arr = (_abi.StepStats * max(nsteps, 1))()
        done = C.c_int32()
        st = self.lib.nim_gpu_step(self._h, nsteps, arr, C.byref(done))
        if raise_on_error:
            _abi.check(st, "nim_gpu_step")
        return [arr[i] for i in range(done.value)]

    # -- timing hooks
    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the context (for events on the launching stream)."""
        return int(self.lib.nim_gpu_stream(self._h) or 0)

    def launch_count(self) -> int:
        return int(self.lib.nim_gpu_launch_count(self._h))

    def profile_iterations(self, n: int) -> dict:
        """Mean device time (ms) of each kernel (launch group) over n
        un-graphed passes of the context's schedule."""
        ms = (C.c_double * 32)()
        nk = self.lib.nim_gpu_profile_iterations(self._h, n, ms, 32)
        if nk < 0:
            _abi.check(nk, "nim_gpu_profile_iterations")
        return {self.lib.nim_gpu_profile_name(self._h, k).decode(): ms[k] for k in range(nk)}

    def synchronize(self):
        _abi.check(self.lib.nim_gpu_synchronize(self._h), "nim_gpu_synchronize")

    # -- host copies (write_data / write_restart / read_restart)
    def download(self, field: int, out: np.ndarray | None = None) -> np.ndarray:
        """The field in the reference layout, into out when given (a
        contiguous float64 array, e.g. a view of page-locked memory, which
        the copy then lands in directly), else into a new array."""
        n = field_len(field, self.mesh)
        if out is None:
            out = np.empty(n, dtype=np.float64)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size < n:
            raise ValueError("out must be a contiguous float64 array of at least the field's length")
        _abi.check(self.lib.nim_gpu_download(self._h, field, out.ctypes.data_as(C.POINTER(C.c_double)), n),
                   "nim_gpu_download")
        return out

    def upload(self, field: int, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64)
        _abi.check(self.lib.nim_gpu_upload(self._h, field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
                   "nim_gpu_upload")

    # -- output sets packed on the device (write_data / write_restart)
    def output_array(self, which: int) -> np.ndarray:
        """A host array shaped for one output set: float32 (6, NMESH) for
        OUTPUT_PLOT, float64 (5 NFACE + 9 NMESH,) for OUTPUT_RESTART."""
        n = int(self.lib.nim_gpu_output_bytes(self._h, which))
        if n < 0:
            _abi.check(n, "nim_gpu_output_bytes")
        if which == _abi.OUTPUT_PLOT:
            return np.empty((6, self.mesh.nmesh), dtype=np.float32)
        return np.empty(n // 8, dtype=np.float64)

    def output_begin(self, which: int, out: np.ndarray) -> int:
        """Pack the set on the device and start copying it into out (keep
        out alive and untouched until output_wait); returns the ticket."""
        if not out.flags.c_contiguous:
            raise ValueError("output buffer must be contiguous")
        t = C.c_int32()
        _abi.check(self.lib.nim_gpu_output_begin(self._h, which, C.c_void_p(out.ctypes.data), out.nbytes,
                                                 C.byref(t)), "nim_gpu_output_begin")
        return t.value

    def set_graph_iters(self, n: int):
        """Inner iterations per graph launch (results do not depend on it)."""
        _abi.check(self.lib.nim_gpu_set_graph_iters(self._h, n), "nim_gpu_set_graph_iters")

    def output_wait(self, ticket: int):
        _abi.check(self.lib.nim_gpu_output_wait(self._h, ticket), "nim_gpu_output_wait")

    def get(self, field: int, n: int | None = None) -> np.ndarray:
        return self.download(field)

    # -- tangent-linear steps (forward-mode derivatives of the time advance)
    def tangent_begin(self):
        """Dual copy of the current state, zero derivatives and seeds."""
        _abi.check(self.lib.nim_gpu_tangent_begin(self._h), "nim_gpu_tangent_begin")

    def tangent_seed(self, dnu: float, dalpha: float):
        _abi.check(self.lib.nim_gpu_tangent_seed(self._h, dnu, dalpha), "nim_gpu_tangent_seed")

    @staticmethod
    def tangent_seed_of(name: str, Ra: float, Pr: float):
        """(d nu, d alpha) of d/dRa or d/dPr: nu = sqrt(Pr / Ra), alpha =
        nu / Pr (parameters.f90:169-173 with g_beta = th_tc = 1)."""
        nu = (Pr / Ra) ** 0.5
        alpha = nu / Pr
        if name == "Ra":
            return -nu / (2 * Ra), -alpha / (2 * Ra)
        if name == "Pr":
            return nu / (2 * Pr), -alpha / (2 * Pr)
        raise ValueError(name)

    def tangent_seed_field(self, field: int, tangent: np.ndarray):
        a = np.ascontiguousarray(tangent, dtype=np.float64)
        _abi.check(self.lib.nim_gpu_tangent_seed_field(self._h, field, a.ctypes.data_as(C.POINTER(C.c_double)),
                                                       a.size), "nim_gpu_tangent_seed_field")

    def tangent_step(self, nsteps: int):
        """nsteps dual steps: (per-step statistics of the values, array
        (nsteps, 2) of d Nu_inner, d Nu_outer)."""
        arr = (_abi.StepStats * max(nsteps, 1))()
        dnu = np.zeros((max(nsteps, 1), 2), dtype=np.float64)
        st = self.lib.nim_gpu_tangent_step(self._h, nsteps, arr, dnu.ctypes.data_as(C.POINTER(C.c_double)))
        _abi.check(st, "nim_gpu_tangent_step")
        return [arr[i] for i in range(nsteps)], dnu[:nsteps]

    def tangent_get(self, field: int):
        """(value, derivative) of a state field of the dual state."""
        n = field_len(field, self.mesh)
        v, t = np.empty(n), np.empty(n)
        _abi.check(self.lib.nim_gpu_tangent_get(self._h, field, v.ctypes.data_as(C.POINTER(C.c_double)),
                                                t.ctypes.data_as(C.POINTER(C.c_double)), n), "nim_gpu_tangent_get")
        return v, t

    def set(self, field: int, values: np.ndarray):
        self.upload(field, values)

    def add_temperature_noise(self, amp: float, seed: int):
        apply_temperature_noise(self.get, self.set, self.mesh, amp, seed)


def batch_step(solvers, nsteps: int, raise_on_error: bool = True, fused: bool = False):
    """nim_batch_step: advance several NimSolvers (one device) by nsteps
    together; returns per-solver lists of step records.  fused: every pass
    kernel launched once for the whole batch (nim_batch_step_fused)."""
    n = len(solvers)
    lib = _abi.gpu_lib()
    handles = (C.c_void_p * n)(*[s._h.value for s in solvers])
    per = (_abi.StepStats * max(n * nsteps, 1))()
    done = (C.c_int32 * n)()
    fn = lib.nim_batch_step_fused if fused else lib.nim_batch_step
    st = fn(n, handles, nsteps, per, done)
    if raise_on_error:
        _abi.check(st, "nim_batch_step_fused" if fused else "nim_batch_step")
    return [[per[i * nsteps + k] for k in range(done[i])] for i in range(n)]


def autotune_batch(solvers, candidates=(4, 8, 16, 32), steps_each: int = 1, fused: bool = False):
    """Pick the graph length of a batch by measurement: advance the batch
    steps_each steps with each candidate (these are real steps of the run:
    the iterates do not depend on the graph length) and keep the fastest
    per cell-iteration.  Returns (best, {candidate: seconds per
    cell-iteration}, records of the steps taken)."""
    import time
    timing, recs_all = {}, []
    cells = [s.mesh.nmesh for s in solvers]
    for g in candidates:
        for s in solvers:
            s.set_graph_iters(g)
        t0 = time.perf_counter()
        recs = batch_step(solvers, steps_each, fused=fused)
        dt = time.perf_counter() - t0
        work = sum(c * sum(r.iters for r in rr) for c, rr in zip(cells, recs))
        timing[g] = dt / max(work, 1)
        recs_all.append(recs)
    best = min(timing, key=timing.get)
    for s in solvers:
        s.set_graph_iters(best)
    return best, timing, recs_all