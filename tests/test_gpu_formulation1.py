"""nim_formulation = 1 on the GPU (calculate_velocity_nim_constants,
nim.f90:17-157, and integrate_velocity_field_i, nse.f90:330-828) against
the CPU oracle: the parallel schedule against the oracle's PARALLEL order,
the reference-order schedule against its SEQUENTIAL (reference) order."""
import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config
import oracle as O

pytestmark = pytest.mark.gpu

STATE = [
    _abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
    _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T,
]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(mesh_params, params, schedule, noise=None):
    params.formulation = 1
    params.schedule = schedule
    mesh = nimgpu.Mesh(mesh_params)
    gpu = nimgpu.NimSolver(mesh, params)
    gpu.initialize_nse()
    ref = O.Oracle(mesh, params, schedule=O.PARALLEL if schedule == _abi.SCHEDULE_PARALLEL else O.SEQUENTIAL)
    ref.init()
    if noise:
        gpu.add_temperature_noise(*noise)
        nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, *noise)
    return gpu, ref


def worst(gpu, ref, fields):
    out = {}
    for f in fields:
        a = gpu.download(f)
        b = ref.get(f, a.size)
        if f == _abi.FACES_P:
            a, b = a - a.mean(), b - b.mean()
        out[f] = rel(a, b)
    return out


@pytest.mark.parametrize("schedule", [_abi.SCHEDULE_PARALLEL, _abi.SCHEDULE_REFERENCE])
@pytest.mark.parametrize("n", [1, 4])
def test_fixed_iterations(schedule, n):
    case = config.small_case(16, 5, 7)
    gpu, ref = pair(case.mesh_params(), case.params(), schedule, (case.noise, case.seed))
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    gpu.iterate(n)
    ref.iterate(n)
    bad = {f: e for f, e in worst(gpu, ref, STATE).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


@pytest.mark.parametrize("schedule", [_abi.SCHEDULE_PARALLEL, _abi.SCHEDULE_REFERENCE])
def test_steps(schedule):
    case = config.small_case(12, 6, 6, steps=3)
    gpu, ref = pair(case.mesh_params(), case.params(), schedule, (case.noise, case.seed))
    sg = gpu.solve_nse(3)
    _, so = ref.step(3)
    assert [a.iters for a in sg] == [b.iters for b in so]
    for a, b in zip(sg, so):
        assert abs(a.nu_inner - b.nu_inner) <= 1e-13 * abs(b.nu_inner)
        assert abs(a.nu_outer - b.nu_outer) <= 1e-13 * abs(b.nu_outer) + 1e-14
    bad = {f: e for f, e in worst(gpu, ref, STATE + [_abi.MESHES_P]).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


@pytest.mark.parametrize("schedule", [_abi.SCHEDULE_PARALLEL, _abi.SCHEDULE_REFERENCE])
def test_series_branch_is_bitwise(schedule):
    """v_limit above every cell Peclet number: no exp anywhere, so the GPU
    reproduces the oracle to the last bit, iteration counts included."""
    gpu, ref = pair(config.reference_mesh(), config.reference_params(v_limit=1e300), schedule)
    sg = gpu.solve_nse(2)
    _, so = ref.step(2)
    assert [a.iters for a in sg] == [b.iters for b in so]
    bad = {f: e for f, e in worst(gpu, ref, STATE).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


def test_formulation_is_validated():
    case = config.small_case()
    with pytest.raises(nimgpu.NimError) as e:
        nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(formulation=3))
    assert e.value.status == _abi.NIM_ERR_BAD_ARG
