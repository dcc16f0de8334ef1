"""GPU parity: the CUDA library through its C ABI against the CPU oracle.

Two checks per quantity:
  * against the oracle's PARALLEL schedule (the same iteration order as the
    kernels): bit for bit for every field and coefficient (the device's exp
    is glibc's, so no operation differs); the Nusselt numbers and the
    dilatation, which the device sums in another order, to 1e-13;
  * against the oracle's SEQUENTIAL schedule (the reference's own order):
    the same discrete fixed point, checked at a tightened tolerance.
"""
import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config
import oracle as O

pytestmark = pytest.mark.gpu

GEOMETRY = [
    _abi.MESHES_VOLUME, _abi.FACES_AREA, _abi.FACES_NORMAL, _abi.FACES_MID, _abi.FACES_TANGENTIAL,
    _abi.FACES_BITANGENTIAL, _abi.MESHES_GIJ, _abi.MESHES_XI_X, _abi.MESHES_G, _abi.MESHES_GIJ_FACES,
    _abi.BCS_FACES_A, _abi.BCS_FACES_AP, _abi.AA_PX, _abi.AA_PY, _abi.AA_PZ,
]
STATE = [
    _abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
    _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T,
]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(case=None, schedule=O.PARALLEL, mesh_params=None, params=None, noise=True, **over):
    case = case or config.small_case()
    mesh = nimgpu.Mesh(mesh_params if mesh_params is not None else case.mesh_params())
    p = params if params is not None else case.params(**over)
    gpu = nimgpu.NimSolver(mesh, p)
    gpu.initialize_nse()
    ref = O.Oracle(mesh, p, schedule=schedule)
    ref.init()
    if noise and case.noise:
        gpu.add_temperature_noise(case.noise, case.seed)
        nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, case.noise, case.seed)
    return mesh, gpu, ref


def compare(gpu, ref, fields, tol, label=""):
    worst = {}
    for f in fields:
        a = gpu.download(f)
        b = ref.get(f, a.size)
        if f == _abi.FACES_P:
            a, b = a - a.mean(), b - b.mean()
        worst[f] = rel(a, b)
    bad = {f: e for f, e in worst.items() if not e <= tol}
    assert not bad, f"{label} fields above {tol}: {bad}"
    return worst


@pytest.mark.parametrize("dims", [(12, 6, 6), (16, 5, 7)])
def test_geometry_matches_oracle(dims):
    case = config.small_case(*dims)
    _, gpu, ref = pair(case, noise=False)
    compare(gpu, ref, GEOMETRY, 1e-13, "init geometry")
    gpu.close()


def test_reference_geometry_matches_oracle():
    _, gpu, ref = pair(mesh_params=config.reference_mesh(), params=config.reference_params(), noise=False)
    compare(gpu, ref, GEOMETRY, 1e-13, "reference geometry")
    compare(gpu, ref, [_abi.FACES_T, _abi.FACES_U], 0.0, "dirichlet")


def test_velocity_coefficients_match_oracle():
    _, gpu, ref = pair()
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    gpu.iterate(3)
    ref.iterate(3)
    gpu.update_time_step()
    ref.end_step()
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    compare(gpu, ref, [_abi.M_F4, _abi.M_F1, _abi.M_F2, _abi.M_F3], 0.0, "M_F")


@pytest.mark.parametrize("n", [1, 2, 7])
def test_fixed_iterations_match_parallel_oracle(n):
    _, gpu, ref = pair()
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    sg = gpu.iterate(n)
    so = ref.iterate(n)
    compare(gpu, ref, STATE, 0.0, f"{n} iterations")
    for k in ("err_u", "err_v", "err_w", "err_p", "err_T"):
        assert getattr(sg, k) == getattr(so, k), k


def test_steps_match_parallel_oracle():
    case = config.small_case(steps=3)
    _, gpu, ref = pair(case)
    sg = gpu.solve_nse(3)
    st, so = ref.step(3)
    assert st == 0 and len(sg) == len(so) == 3
    for a, b in zip(sg, so):
        assert a.iters == b.iters
        assert abs(a.nu_inner - b.nu_inner) <= 1e-13 * abs(b.nu_inner)
        assert abs(a.nu_outer - b.nu_outer) <= 1e-13 * abs(b.nu_outer) + 1e-14
        assert abs(a.dilatation - b.dilatation) <= 1e-13 * abs(b.dilatation)
        assert a.area_inner == pytest.approx(b.area_inner, rel=1e-14)
    compare(gpu, ref, STATE + [_abi.MESHES_P, _abi.MESHES_UT, _abi.MESHES_TT], 0.0, "3 steps")


def test_reference_case_two_steps():
    """parameters.f90 as shipped: 36x6x12 cells, DT=0.01, Ra=1e5, Pr=0.7."""
    mesh = nimgpu.Mesh(config.reference_mesh())
    p = config.reference_params()
    gpu = nimgpu.NimSolver(mesh, p)
    gpu.initialize_nse()
    par = O.Oracle(mesh, p, schedule=O.PARALLEL)
    par.init()
    seq = O.Oracle(mesh, p, schedule=O.SEQUENTIAL)
    seq.init()
    sg = gpu.solve_nse(2)
    _, sp = par.step(2)
    _, ss = seq.step(2)
    for a, b, c in zip(sg, sp, ss):
        assert a.iters == b.iters
        assert abs(a.nu_inner - b.nu_inner) <= 1e-13 * abs(b.nu_inner)
        # the reference's own order stops at its 1e-6 tolerance on another
        # path: agreement to the tolerance's scale
        assert abs(a.nu_inner - c.nu_inner) <= 1e-4 * abs(c.nu_inner)
    # the exponential form of M_A(.,5) amplifies one ulp of exp by ~12/|Pe|^3
    # near |Pe| = v_limit; with glibc's exp on the device nothing differs
    compare(gpu, par, STATE, 0.0, "reference case")


def test_series_branch_is_bitwise_reproducible():
    """With v_limit above every cell Peclet number the coefficients come
    from the series branch only (no exp): the kernels then reproduce the
    oracle's parallel order to the last bit over whole steps."""
    mesh = nimgpu.Mesh(config.reference_mesh())
    p = config.reference_params(v_limit=1e300)
    gpu = nimgpu.NimSolver(mesh, p)
    gpu.initialize_nse()
    par = O.Oracle(mesh, p, schedule=O.PARALLEL)
    par.init()
    sg = gpu.solve_nse(2)
    _, sp = par.step(2)
    for a, b in zip(sg, sp):
        # Nu is a sum: tree order on the device, serial on the host
        assert a.iters == b.iters and a.nu_inner == pytest.approx(b.nu_inner, rel=1e-14)
    compare(gpu, par, STATE, 0.0, "series-only steps")


def test_tight_tolerance_matches_sequential_oracle():
    """Converged to 1e-13 (pressure gradients, is_dpdx_tolerance) both orders
    reach the same fixed point: T and the Nusselt history to <= 1e-10."""
    case = config.small_case(steps=2)
    tight = dict(tol_u=1e-13, tol_v=1e-13, tol_w=1e-13, tol_T=1e-13, tol_p=1e-13, dpdx_tolerance=1,
                 max_iters=200000)
    _, gpu, ref = pair(case, schedule=O.SEQUENTIAL, **tight)
    sg = gpu.solve_nse(2)
    st, so = ref.step(2)
    assert st == 0
    for a, b in zip(sg, so):
        assert abs(a.nu_inner - b.nu_inner) <= 1e-10 * abs(b.nu_inner)
        assert abs(a.nu_outer - b.nu_outer) <= 1e-10 * abs(b.nu_outer)
    compare(gpu, ref, [_abi.FACES_T, _abi.MESHES_T], 1e-10, "tight T")


def test_max_iters_reports_not_converged():
    _, gpu, _ = pair(max_iters=3)
    gpu.calculate_velocity_nim_constants()
    s = gpu.integrate_nse(raise_on_error=False)
    assert s.status == _abi.NIM_ERR_NOT_CONVERGED and s.iters == 3


def test_nonfinite_is_reported():
    mesh, gpu, _ = pair()
    t = gpu.download(_abi.FACES_T)
    t[mesh.interior_faces.nonzero()[0][5]] = np.nan
    gpu.upload(_abi.FACES_T, t)
    gpu.calculate_velocity_nim_constants()
    s = gpu.integrate_nse(raise_on_error=False)
    assert s.status == _abi.NIM_ERR_NONFINITE


def test_download_upload_roundtrip():
    mesh, gpu, _ = pair()
    rng = np.random.default_rng(3)
    for f in (_abi.FACES_P, _abi.MESHES_U, _abi.MESHES_T_OLD):
        v = rng.standard_normal(nimgpu.field_len(f, mesh))
        gpu.upload(f, v)
        assert np.array_equal(gpu.download(f), v)
        out = np.full(v.size, np.nan)
        assert gpu.download(f, out=out) is out and np.array_equal(out, v)


def test_runs_are_bitwise_deterministic():
    outs = []
    for _ in range(2):
        _, gpu, _ = pair(noise=True)
        gpu.solve_nse(2)
        outs.append([gpu.download(f) for f in STATE])
        gpu.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_bad_mesh_is_refused():
    mesh = nimgpu.Mesh(config.small_case().mesh_params())
    mesh.meshes_neighbors[5, 2] = 1  # break the O-grid pattern
    with pytest.raises(nimgpu.NimError) as e:
        nimgpu.NimSolver(mesh, config.small_case().params())
    assert e.value.status == _abi.NIM_ERR_BAD_ARG
