"""ctypes mirror of include/nim_gpu.h and include/nim_mesh.h.

Struct layouts here must match the C headers field for field; tests/
test_abi.py checks the sizes against the compiled libraries.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent.parent          # nim-conv22-shared_b200/
LIB_DIR = PKG_DIR / "lib"
REPO_DIR = PKG_DIR.parent

NIM_OK = 0
NIM_ERR_BAD_ARG = -1
NIM_ERR_CUDA = -2
NIM_ERR_NOT_CONVERGED = -3
NIM_ERR_NONFINITE = -4
NIM_ERR_TIMEOUT = -5
NIM_ERR_STATE = -6
NIM_NBC = 5

# nim_field
FACES_U, FACES_V, FACES_W, FACES_P, FACES_T = 0, 1, 2, 3, 4
MESHES_U, MESHES_V, MESHES_W, MESHES_T = 5, 6, 7, 8
MESHES_U_OLD, MESHES_V_OLD, MESHES_W_OLD, MESHES_T_OLD = 9, 10, 11, 12
MESHES_UT, MESHES_VT, MESHES_WT, MESHES_TT = 13, 14, 15, 16
MESHES_P, MESHES_DILA, MESHES_DILA_OLD = 17, 18, 19
MESHES_VOLUME, FACES_AREA, FACES_NORMAL, FACES_MID = 32, 33, 34, 35
MESHES_GIJ, MESHES_XI_X, MESHES_G, MESHES_GIJ_FACES = 36, 37, 38, 39
FACES_TANGENTIAL, FACES_BITANGENTIAL, BCS_FACES_A, BCS_FACES_AP = 40, 41, 42, 43
AA_PX, AA_PY, AA_PZ = 44, 45, 46
M_F4, M_F1, M_F2, M_F3 = 48, 49, 50, 51

CLUSTER_NONE, CLUSTER_POWER, CLUSTER_TANH = 0, 1, 2
SCHEDULE_PARALLEL, SCHEDULE_REFERENCE = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
OUTPUT_PLOT, OUTPUT_RESTART = 0, 1   # nim_output_set


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_theta", C.c_int32), ("n_r", C.c_int32), ("n_z", C.c_int32),
        ("nnode", C.c_int32), ("nmesh", C.c_int32), ("nface", C.c_int32),
        ("nbcface", C.c_int32),
        ("node_xyz", C.POINTER(C.c_double)),
        ("meshes_nodes", C.POINTER(C.c_int32)),
        ("meshes_faces", C.POINTER(C.c_int32)),
        ("meshes_neighbors", C.POINTER(C.c_int32)),
        ("faces_bc", C.POINTER(C.c_int32)),
        ("bcs_faces", C.POINTER(C.c_int32)),
        ("bcs_faces_id", C.POINTER(C.c_int32)),
        ("bcs_faces_position", C.POINTER(C.c_int32)),
        ("bcs_faces_mesh_num", C.POINTER(C.c_int32)),
    ]


class Params(C.Structure):
    _fields_ = [
        ("DT", C.c_double), ("nu", C.c_double), ("alpha", C.c_double),
        ("rho", C.c_double), ("g_beta", C.c_double),
        ("w_u", C.c_double), ("w_v", C.c_double), ("w_w", C.c_double),
        ("w_p", C.c_double), ("w_p2", C.c_double), ("w_T", C.c_double),
        ("tol_u", C.c_double), ("tol_v", C.c_double), ("tol_w", C.c_double),
        ("tol_p", C.c_double), ("tol_T", C.c_double),
        ("v_limit", C.c_double), ("dudt_epsilon", C.c_double),
        ("R_i", C.c_double), ("R_o", C.c_double),
        ("bc_value", (C.c_double * NIM_NBC) * 5),
        ("max_iters", C.c_int32), ("check_steady", C.c_int32),
        ("dpdx_tolerance", C.c_int32), ("schedule", C.c_int32), ("formulation", C.c_int32),
        ("precision", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("step", C.c_int32), ("iters", C.c_int32),
        ("err_u", C.c_double), ("err_v", C.c_double), ("err_w", C.c_double),
        ("err_p", C.c_double), ("err_T", C.c_double),
        ("dilatation", C.c_double), ("dudt_max", C.c_double), ("dTdt_max", C.c_double),
        ("nu_outer", C.c_double), ("nu_inner", C.c_double),
        ("area_outer", C.c_double), ("area_inner", C.c_double),
        ("time", C.c_double), ("steady", C.c_int32), ("status", C.c_int32),
        ("iters_fp32", C.c_int32), ("pad", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class MeshParams(C.Structure):
    _fields_ = [
        ("n_theta", C.c_int32), ("n_r", C.c_int32), ("n_z", C.c_int32),
        ("R_i", C.c_double), ("R_o", C.c_double), ("L", C.c_double),
        ("cluster", C.c_int32), ("cluster_factor", C.c_double),
        ("hexagon", C.c_int32), ("blend_r1", C.c_double), ("blend_r2", C.c_double),
        ("blend_n", C.c_double),
    ]


class NimError(RuntimeError):
    def __init__(self, status: int, where: str, text: str = ""):
        self.status = status
        super().__init__(f"{where}: status {status} {text}".strip())


def _load(path: Path) -> C.CDLL:
    if not path.exists():
        raise FileNotFoundError(
            f"{path} is missing; build it first (python -c 'import __graft_entry__ as g; g.build()')")
    return C.CDLL(str(path))


_host = None
_gpu = None


def host_lib() -> C.CDLL:
    """libnim_host.so: the host mesh builder (no CUDA)."""
    global _host
    if _host is None:
        lib = _load(LIB_DIR / "libnim_host.so")
        lib.nim_mesh_params_reference.argtypes = [C.POINTER(MeshParams)]
        lib.nim_mesh_params_reference.restype = None
        lib.nim_mesh_sizes.argtypes = [C.POINTER(MeshParams)] + [C.POINTER(C.c_int32)] * 4
        lib.nim_mesh_sizes.restype = C.c_int
        lib.nim_mesh_build.argtypes = [C.POINTER(MeshParams), C.POINTER(C.c_double)] + \
            [C.POINTER(C.c_int32)] * 8
        lib.nim_mesh_build.restype = C.c_int
        _host = lib
    return _host


def gpu_lib() -> C.CDLL:
    """libnimgpu.so: the CUDA library behind include/nim_gpu.h."""
    global _gpu
    if _gpu is None:
        lib = _load(LIB_DIR / "libnimgpu.so")
        vp = C.c_void_p
        lib.nim_params_reference.argtypes = [C.POINTER(Params)]
        lib.nim_params_reference.restype = None
        lib.nim_gpu_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Params), C.POINTER(vp)]
        lib.nim_gpu_create.restype = C.c_int
        for name in ("nim_gpu_init", "nim_gpu_begin_step", "nim_gpu_synchronize"):
            getattr(lib, name).argtypes = [vp]
            getattr(lib, name).restype = C.c_int
        lib.nim_gpu_integrate.argtypes = [vp, C.POINTER(StepStats)]
        lib.nim_gpu_integrate.restype = C.c_int
        lib.nim_gpu_iterate.argtypes = [vp, C.c_int32, C.POINTER(StepStats)]
        lib.nim_gpu_iterate.restype = C.c_int
        lib.nim_gpu_end_step.argtypes = [vp, C.POINTER(StepStats)]
        lib.nim_gpu_end_step.restype = C.c_int
        lib.nim_gpu_step.argtypes = [vp, C.c_int32, C.POINTER(StepStats), C.POINTER(C.c_int32)]
        lib.nim_gpu_step.restype = C.c_int
        lib.nim_gpu_download.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.c_int64]
        lib.nim_gpu_download.restype = C.c_int
        lib.nim_gpu_tangent_begin.argtypes = [vp]
        lib.nim_gpu_tangent_begin.restype = C.c_int
        lib.nim_gpu_tangent_seed.argtypes = [vp, C.c_double, C.c_double]
        lib.nim_gpu_tangent_seed.restype = C.c_int
        lib.nim_gpu_tangent_seed_field.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.c_int64]
        lib.nim_gpu_tangent_seed_field.restype = C.c_int
        lib.nim_gpu_tangent_step.argtypes = [vp, C.c_int32, C.POINTER(StepStats), C.POINTER(C.c_double)]
        lib.nim_gpu_tangent_step.restype = C.c_int
        lib.nim_gpu_tangent_get.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64]
        lib.nim_gpu_tangent_get.restype = C.c_int
        lib.nim_gpu_upload.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.c_int64]
        lib.nim_gpu_upload.restype = C.c_int
        lib.nim_gpu_set_graph_iters.argtypes = [vp, C.c_int32]
        lib.nim_gpu_set_graph_iters.restype = C.c_int
        lib.nim_batch_step.argtypes = [C.c_int32, C.POINTER(vp), C.c_int32, C.POINTER(StepStats),
                                       C.POINTER(C.c_int32)]
        lib.nim_batch_step.restype = C.c_int
        lib.nim_batch_step_fused.argtypes = [C.c_int32, C.POINTER(vp), C.c_int32, C.POINTER(StepStats),
                                             C.POINTER(C.c_int32)]
        lib.nim_batch_step_fused.restype = C.c_int
        lib.nim_slab_layout.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]
        lib.nim_slab_layout.restype = C.c_int
        lib.nim_slab_halo.argtypes = [C.c_int32] * 6 + [C.POINTER(C.c_int64)] * 2
        lib.nim_slab_halo.restype = C.c_int
        lib.nim_gpu_create_slab.argtypes = [C.POINTER(MeshDesc), C.POINTER(Params), C.c_int32, C.c_int32,
                                            C.POINTER(vp)]
        lib.nim_gpu_create_slab.restype = C.c_int
        lib.nim_slab_step.argtypes = [C.c_int32, C.POINTER(vp), C.c_int32, C.POINTER(StepStats),
                                      C.POINTER(C.c_int32)]
        lib.nim_slab_step.restype = C.c_int
        lib.nim_slab_part.argtypes = [vp, C.c_int32]
        lib.nim_slab_part.restype = C.c_int
        lib.nim_slab_arrays.argtypes = [vp, C.c_int32, C.POINTER(vp), C.POINTER(C.c_int32), C.c_int32]
        lib.nim_slab_arrays.restype = C.c_int
        lib.nim_slab_pack_doubles.argtypes = [vp, C.c_int32, C.c_int32]
        lib.nim_slab_pack_doubles.restype = C.c_int64
        lib.nim_slab_pack.argtypes = [vp, C.c_int32, C.c_int32, vp]
        lib.nim_slab_pack.restype = C.c_int
        lib.nim_slab_unpack.argtypes = [vp, C.c_int32, C.c_int32, vp]
        lib.nim_slab_unpack.restype = C.c_int
        lib.nim_slab_maxima.argtypes = [vp, C.POINTER(vp)]
        lib.nim_slab_maxima.restype = C.c_int
        lib.nim_slab_loop_state.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        lib.nim_slab_loop_state.restype = C.c_int
        lib.nim_slab_after_loop.argtypes = [vp, C.POINTER(C.c_double)]
        lib.nim_slab_after_loop.restype = C.c_int
        lib.nim_slab_end_step.argtypes = [vp, C.POINTER(C.c_double)]
        lib.nim_slab_end_step.restype = C.c_int
        lib.nim_gpu_output_bytes.argtypes = [vp, C.c_int32]
        lib.nim_gpu_output_bytes.restype = C.c_int64
        lib.nim_gpu_output_begin.argtypes = [vp, C.c_int32, vp, C.c_int64, C.POINTER(C.c_int32)]
        lib.nim_gpu_output_begin.restype = C.c_int
        lib.nim_gpu_output_wait.argtypes = [vp, C.c_int32]
        lib.nim_gpu_output_wait.restype = C.c_int
        lib.nim_gpu_destroy.argtypes = [vp]
        lib.nim_gpu_destroy.restype = None
        lib.nim_gpu_strerror.argtypes = [C.c_int]
        lib.nim_gpu_strerror.restype = C.c_char_p
        lib.nim_gpu_stream.argtypes = [vp]
        lib.nim_gpu_stream.restype = vp
        lib.nim_gpu_launch_count.argtypes = [vp]
        lib.nim_gpu_launch_count.restype = C.c_int64
        lib.nim_gpu_profile_iterations.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.c_int32]
        lib.nim_gpu_profile_iterations.restype = C.c_int
        lib.nim_gpu_profile_name.argtypes = [vp, C.c_int32]
        lib.nim_gpu_profile_name.restype = C.c_char_p
        lib.nim_gpu_selftest_exp.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64]
        lib.nim_gpu_selftest_exp.restype = C.c_int
        lib.nim_gpu_selftest_nim_coef.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64,
                                                  C.c_int32, C.c_double, C.POINTER(C.c_double)]
        lib.nim_gpu_selftest_nim_coef.restype = C.c_int
        lib.nim_gpu_selftest_wait_timeout.argtypes = [vp, C.c_int32]
        lib.nim_gpu_selftest_wait_timeout.restype = C.c_int
        lib.nim_gpu_nusselt_noalloc.argtypes = [vp, C.POINTER(C.c_double)]
        lib.nim_gpu_nusselt_noalloc.restype = C.c_int
        _gpu = lib
    return _gpu


def gpu_lib_path() -> Path:
    return LIB_DIR / "libnimgpu.so"


def strerror(status: int) -> str:
    try:
        return gpu_lib().nim_gpu_strerror(status).decode()
    except FileNotFoundError:
        return ""


def check(status: int, where: str) -> int:
    if status != NIM_OK:
        raise NimError(status, where, strerror(status))
    return status


def env_flag(name: str) -> bool:
    return os.environ.get(name, "") not in ("", "0")
