"""The C-ABI libraries load and export every entry point include/*.h
declares, and the ctypes structs match the C layouts.  No GPU needed: only
argument checks and pure host functions are called."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from nimgpu import _abi, config

ROOT = Path(__file__).resolve().parent.parent
INCLUDE = ROOT / "include"


def declared(header: str):
    text = (INCLUDE / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nim_\w+)\s*\(", text)))


def test_host_library_exports_mesh_header():
    lib = _abi.host_lib()
    names = declared("nim_mesh.h")
    assert names, "no declarations parsed"
    for n in names:
        assert hasattr(lib, n), n


@pytest.fixture(scope="module")
def gpu_lib():
    path = _abi.gpu_lib_path()
    if not path.exists():
        pytest.skip("libnimgpu.so not built (needs nvcc: __graft_entry__.build())")
    return _abi.gpu_lib()


def test_gpu_library_exports_abi_header(gpu_lib):
    for n in declared("nim_gpu.h"):
        assert hasattr(gpu_lib, n), n


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "nim_gpu.h"\n#include "nim_mesh.h"\n'
                   "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(nim_mesh_desc), "
                   "sizeof(nim_params), sizeof(nim_step_stats), sizeof(nim_mesh_params), "
                   "offsetof(nim_params, bc_value), offsetof(nim_step_stats, time)); return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(INCLUDE), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(_abi.MeshDesc), C.sizeof(_abi.Params), C.sizeof(_abi.StepStats), C.sizeof(_abi.MeshParams),
            _abi.Params.bc_value.offset, _abi.StepStats.time.offset]
    assert got == want


def test_reference_params_agree(gpu_lib):
    p = _abi.Params()
    gpu_lib.nim_params_reference(C.byref(p))
    q = config.reference_params()
    for name, _ in _abi.Params._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if name == "bc_value":
            assert [list(r) for r in a] == [list(r) for r in b]
        else:
            assert a == b, name


def test_argument_errors_without_device(gpu_lib):
    h = C.c_void_p()
    assert gpu_lib.nim_gpu_create(None, None, C.byref(h)) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_gpu_init(None) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_gpu_step(None, 1, None, None) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_gpu_output_bytes(None, 0) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_gpu_output_begin(None, 0, None, 0, None) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_gpu_output_wait(None, 0) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_batch_step(0, None, 1, None, None) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_batch_step_fused(0, None, 1, None, None) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_batch_step_fused(257, None, 1, None, None) == _abi.NIM_ERR_BAD_ARG
    # an unknown schedule is refused before any device call
    import nimgpu
    mesh = nimgpu.Mesh(config.small_case().mesh_params())
    desc = mesh.make_desc()
    p = config.small_case().params(schedule=7)
    assert gpu_lib.nim_gpu_create(C.byref(desc), C.byref(p), C.byref(h)) == _abi.NIM_ERR_BAD_ARG
    assert gpu_lib.nim_gpu_strerror(_abi.NIM_ERR_NOT_CONVERGED).decode().startswith("inner iteration")
