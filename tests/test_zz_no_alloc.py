"""nim_gpu_nusselt_noalloc: the Nusselt numbers for hosts that cannot call
cudaMalloc (all free device memory already handed to another allocator, or
no allocation allowed once the time loop runs).  Its scratch is a static
device array set up by nim_gpu_create, so the call itself allocates
nothing; it must give what nim_gpu_end_step reports for the same state,
call after call.  Collected last (file name) so a failure here comes after
every other test has run."""
import ctypes as C

import pytest

import nimgpu
from nimgpu import _abi, config

pytestmark = pytest.mark.gpu


def _noalloc(solver):
    out = (C.c_double * 4)()
    st = _abi.gpu_lib().nim_gpu_nusselt_noalloc(solver._h, out)
    assert st == _abi.NIM_OK, _abi.strerror(st)
    return list(out)


@pytest.mark.parametrize("dims", [(16, 6, 6), (48, 12, 20)])
def test_nusselt_noalloc_matches_end_step(dims):
    case = config.small_case(*dims)
    mesh = nimgpu.Mesh(case.mesh_params())
    solver = nimgpu.NimSolver(mesh, case.params())
    solver.initialize_nse()
    solver.add_temperature_noise(case.noise, case.seed)
    for _ in range(2):
        solver.calculate_velocity_nim_constants()
        solver.integrate_nse()
        ref = solver.update_time_step()
        want = [ref.nu_outer, ref.nu_inner, ref.area_outer, ref.area_inner]
        for _call in range(2):  # two calls in a row reuse the same scratch
            got = _noalloc(solver)
            assert got == pytest.approx(want, rel=1e-12, abs=1e-300)
    solver.close()


def test_nusselt_noalloc_rejects_bad_arguments():
    lib = _abi.gpu_lib()
    assert lib.nim_gpu_nusselt_noalloc(None, None) == _abi.NIM_ERR_BAD_ARG
    case = config.small_case()
    solver = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params())
    assert lib.nim_gpu_nusselt_noalloc(solver._h, None) == _abi.NIM_ERR_BAD_ARG
    out = (C.c_double * 4)()
    assert lib.nim_gpu_nusselt_noalloc(solver._h, out) == _abi.NIM_ERR_STATE  # before init
    solver.initialize_nse()
    solver.calculate_velocity_nim_constants()
    # inside a step the face temperatures are mid-iteration: refused
    assert lib.nim_gpu_nusselt_noalloc(solver._h, out) == _abi.NIM_ERR_STATE
    solver.integrate_nse()
    assert lib.nim_gpu_nusselt_noalloc(solver._h, out) == _abi.NIM_ERR_STATE
    ref = solver.update_time_step()
    assert _noalloc(solver) == pytest.approx([ref.nu_outer, ref.nu_inner, ref.area_outer, ref.area_inner],
                                             rel=1e-12, abs=1e-300)
    solver.close()
