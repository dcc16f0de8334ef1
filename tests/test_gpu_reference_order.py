"""The reference-order schedule (NIM_SCHEDULE_REFERENCE) against the
oracle's SEQUENTIAL schedule, the reference's own Gauss-Seidel order
(run.sh:2 runs one OpenMP thread).  The kernels sweep level by level in
place; the iterates, the iteration counts and the stopping step must be the
reference's, not only its fixed point."""
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


def pair(mesh_params, params, noise=None):
    mesh = nimgpu.Mesh(mesh_params)
    params.schedule = _abi.SCHEDULE_REFERENCE
    gpu = nimgpu.NimSolver(mesh, params)
    gpu.initialize_nse()
    ref = O.Oracle(mesh, params, schedule=O.SEQUENTIAL)
    ref.init()
    if noise:
        gpu.add_temperature_noise(*noise)
        nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, *noise)
    return mesh, gpu, ref


def worst(gpu, ref, fields):
    out = {}
    for f in fields:
        a = gpu.download(f)
        out[f] = rel(a, ref.get(f, a.size))
    return out


@pytest.mark.parametrize("dims", [(12, 6, 6), (16, 5, 7), (6, 4, 4)])
@pytest.mark.parametrize("n", [1, 3])
def test_fixed_iterations_match_reference_order(dims, n):
    case = config.small_case(*dims)
    _, gpu, ref = pair(case.mesh_params(), case.params(), (case.noise, case.seed))
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    sg = gpu.iterate(n)
    so = ref.iterate(n)
    assert (sg.err_u, sg.err_v, sg.err_w, sg.err_p, sg.err_T) == (so.err_u, so.err_v, so.err_w, so.err_p, so.err_T)
    bad = {f: e for f, e in worst(gpu, ref, STATE).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


def test_series_branch_reference_order_is_bitwise():
    """Series branch only (no exp): the level sweeps reproduce the
    reference's order to the last bit over whole steps, iteration counts
    included."""
    _, gpu, ref = pair(config.reference_mesh(), config.reference_params(v_limit=1e300))
    sg = gpu.solve_nse(2)
    _, so = ref.step(2)
    assert [a.iters for a in sg] == [b.iters for b in so]
    for a, b in zip(sg, so):
        assert a.nu_inner == pytest.approx(b.nu_inner, rel=1e-14)
        assert a.nu_outer == pytest.approx(b.nu_outer, rel=1e-14)
    bad = {f: e for f, e in worst(gpu, ref, STATE).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


def test_reference_case_reference_order():
    """parameters.f90 as shipped (36x6x12 cells, DT=0.01, Ra=1e5, Pr=0.7),
    reference order, exponential branch included: the reference's iteration
    counts, its steady-state maxima exactly and its fields bit for bit."""
    _, gpu, ref = pair(config.reference_mesh(), config.reference_params())
    sg = gpu.solve_nse(2)
    _, so = ref.step(2)
    assert [a.iters for a in sg] == [b.iters for b in so]
    for a, b in zip(sg, so):
        assert abs(a.nu_inner - b.nu_inner) <= 1e-13 * abs(b.nu_inner)
        assert abs(a.nu_outer - b.nu_outer) <= 1e-13 * abs(b.nu_outer) + 1e-14
        assert a.dudt_max == b.dudt_max and a.dTdt_max == b.dTdt_max
    bad = {f: e for f, e in worst(gpu, ref, STATE).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


def test_reference_order_steps_with_pressure_gradient_tolerance():
    case = config.small_case(16, 5, 7, steps=3)
    _, gpu, ref = pair(case.mesh_params(), case.params(dpdx_tolerance=1, tol_p=1e-5),
                       (case.noise, case.seed))
    sg = gpu.solve_nse(3)
    _, so = ref.step(3)
    assert [a.iters for a in sg] == [b.iters for b in so]
    bad = {f: e for f, e in worst(gpu, ref, STATE + [_abi.MESHES_P, _abi.MESHES_TT]).items() if e != 0.0}
    assert not bad, bad
    gpu.close()


def test_reference_order_runs_are_deterministic_and_roundtrip():
    outs = []
    for _ in range(2):
        case = config.small_case()
        mesh, gpu, _ = pair(case.mesh_params(), case.params(), (case.noise, case.seed))
        gpu.solve_nse(2)
        outs.append([gpu.download(f) for f in STATE])
        v = np.random.default_rng(5).standard_normal(mesh.nface)
        gpu.upload(_abi.FACES_P, v)
        assert np.array_equal(gpu.download(_abi.FACES_P), v)
        gpu.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_reference_order_kernel_profile():
    case = config.small_case()
    _, gpu, _ = pair(case.mesh_params(), case.params())
    prof = gpu.profile_iterations(2)
    assert list(prof) == ["k_vel_cell(src)", "k_seq_vel", "k_p_src", "k_seq_pbc", "k_seq_p", "k_zero_flux",
                          "k_T_coef", "k_T_cell(src)", "k_seq_T", "k_iter_end"]
    assert all(v > 0 for v in prof.values())
    gpu.close()
