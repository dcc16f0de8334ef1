"""Mixed precision (nim_params.precision = NIM_PRECISION_MIXED): each step's
inner loop first sweeps a float mirror of the iterate, the NIM constants and
the geometry, then continues in FP64 from the widened FP32 iterate until the
reference's stop test holds.  The extension has no counterpart in the
reference; its oracle is the FP64 GPU path (itself pinned to the CPU oracle
by tests/test_gpu_parity.py) and, converged, the CPU oracle."""
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
# converged: every field's largest change per pass below 1e-13, pressure
# measured by its gradients (is_dpdx_tolerance, nse.f90:292-307)
TIGHT = dict(tol_u=1e-13, tol_v=1e-13, tol_w=1e-13, tol_T=1e-13, tol_p=1e-13, dpdx_tolerance=1,
             max_iters=200000)


def make(case, precision, **over):
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(precision=precision, **over))
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    return s


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def rel_field(f, a, b):
    """Pressure is compared modulo its mean: the gradient stop test
    (is_dpdx_tolerance) leaves its additive constant free."""
    if f == _abi.FACES_P:
        a, b = a - a.mean(), b - b.mean()
    return rel(a, b)


def test_converged_steps_reach_the_fp64_fixed_point():
    """Converged to 1e-13, the FP32 passes stop at their rounding floor and
    the FP64 passes carry the iterate to the same fixed point the FP64 path
    reaches: Nusselt history and fields to <= 1e-9 relative (pressure
    modulo its mean)."""
    case = config.small_case(16, 6, 6, Ra=1e4, steps=3)
    a, b = make(case, _abi.PRECISION_FP64, **TIGHT), make(case, _abi.PRECISION_MIXED, **TIGHT)
    ra, rb = a.solve_nse(3), b.solve_nse(3)
    for x, y in zip(ra, rb):
        assert 0 < y.iters_fp32 < y.iters
        assert x.iters_fp32 == 0
        assert abs(y.nu_inner - x.nu_inner) <= 1e-9 * abs(x.nu_inner)
        assert abs(y.nu_outer - x.nu_outer) <= 1e-9 * abs(x.nu_outer)
        for e in (y.err_u, y.err_v, y.err_w, y.err_p, y.err_T):
            assert e <= 1e-13
    bad = {f: rel_field(f, b.download(f), a.download(f)) for f in STATE}
    bad = {f: e for f, e in bad.items() if not e <= 1e-9}
    assert not bad, bad
    a.close()
    b.close()


def test_converged_steps_match_the_cpu_oracle():
    """The same converged run against the CPU oracle (parallel schedule,
    FP64): temperature and the Nusselt history to <= 1e-9."""
    case = config.small_case(12, 6, 6, steps=2)
    mesh = nimgpu.Mesh(case.mesh_params())
    params = case.params(precision=_abi.PRECISION_MIXED, **TIGHT)
    gpu = nimgpu.NimSolver(mesh, params)
    gpu.initialize_nse()
    gpu.add_temperature_noise(case.noise, case.seed)
    ref = O.Oracle(mesh, case.params(**TIGHT), schedule=O.PARALLEL)
    ref.init()
    nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, case.noise, case.seed)
    sg = gpu.solve_nse(2)
    st, so = ref.step(2)
    assert st == 0
    for a, b in zip(sg, so):
        assert abs(a.nu_inner - b.nu_inner) <= 1e-9 * abs(b.nu_inner)
        assert abs(a.nu_outer - b.nu_outer) <= 1e-9 * abs(b.nu_outer)
    for f in (_abi.FACES_T, _abi.MESHES_T):
        g = gpu.download(f)
        assert rel(g, ref.get(f, g.size)) <= 1e-9
    gpu.close()


def test_reference_tolerances_end_on_an_fp64_pass():
    """At the reference tolerances each step's last pass is FP64 and meets
    the stop test; the result differs from the FP64 path only by what the
    tolerances themselves leave open (both stop once a pass changes every
    field by less than its tolerance)."""
    case = config.small_case(24, 12, 12, Ra=1e4, steps=3)
    a, b = make(case, _abi.PRECISION_FP64), make(case, _abi.PRECISION_MIXED)
    ra, rb = a.solve_nse(3), b.solve_nse(3)
    p = case.params()
    for x, y in zip(ra, rb):
        assert y.status == _abi.NIM_OK
        assert 0 < y.iters_fp32 < y.iters
        assert y.err_u <= p.tol_u and y.err_v <= p.tol_v and y.err_w <= p.tol_w
        assert y.err_p <= p.tol_p and y.err_T <= p.tol_T
        assert abs(y.iters - x.iters) <= 0.1 * x.iters + 2
        assert abs(y.nu_inner - x.nu_inner) <= 1e-4 * abs(x.nu_inner)
        assert abs(y.nu_outer - x.nu_outer) <= 1e-2 * abs(x.nu_outer)
    for f in (_abi.FACES_T, _abi.MESHES_T):
        assert rel(b.download(f), a.download(f)) <= 1e-4
    a.close()
    b.close()


def test_mixed_runs_are_bitwise_deterministic():
    case = config.small_case(16, 6, 6, steps=2)
    outs = []
    for _ in range(2):
        s = make(case, _abi.PRECISION_MIXED)
        recs = s.solve_nse(2)
        outs.append(([(r.iters, r.iters_fp32, r.nu_inner, r.nu_outer) for r in recs],
                     [s.download(f) for f in STATE]))
        s.close()
    assert outs[0][0] == outs[1][0]
    for x, y in zip(outs[0][1], outs[1][1]):
        assert np.array_equal(x, y)


def test_fixed_pass_count_runs_fp64():
    """nim_gpu_iterate runs FP64 passes in a mixed context too: the same
    bits as an FP64 context."""
    case = config.small_case(12, 6, 6)
    a, b = make(case, _abi.PRECISION_FP64), make(case, _abi.PRECISION_MIXED)
    for s in (a, b):
        s.calculate_velocity_nim_constants()
    sa, sb = a.iterate(4), b.iterate(4)
    assert (sa.err_u, sa.err_p, sa.err_T) == (sb.err_u, sb.err_p, sb.err_T)
    assert sb.iters_fp32 == 0
    for f in STATE:
        assert np.array_equal(a.download(f), b.download(f))
    a.close()
    b.close()


def test_profile_runs_fp32_passes_and_keeps_fp64_fields():
    case = config.small_case(12, 6, 6)
    a, b = make(case, _abi.PRECISION_FP64), make(case, _abi.PRECISION_MIXED)
    b.calculate_velocity_nim_constants()
    before = [b.download(f) for f in STATE]
    pa, pb = a.profile_iterations(2), b.profile_iterations(2)
    # the same sweeps, each in whichever form (one, two or four cells a
    # thread; gathered or staged) the storage type and mesh select
    def base(k):
        return k.rstrip("N").replace("k_vel_cell2", "k_vel_cell").replace("k_vel_face_tile", "k_vel_face")
    assert [base(k) for k in pa] == [base(k) for k in pb]
    assert all(v > 0 for v in pb.values())
    for f, v in zip(STATE, before):
        assert np.array_equal(b.download(f), v)
    a.close()
    b.close()


def test_max_iters_bounds_both_phases():
    case = config.small_case(12, 6, 6)
    s = make(case, _abi.PRECISION_MIXED, max_iters=3)
    s.calculate_velocity_nim_constants()
    r = s.integrate_nse(raise_on_error=False)
    assert r.status == _abi.NIM_ERR_NOT_CONVERGED
    assert r.iters == 3 and r.iters_fp32 == 3
    s.close()


def test_nonfinite_in_the_fp32_phase_is_reported():
    case = config.small_case(12, 6, 6)
    mesh = nimgpu.Mesh(case.mesh_params())
    s = nimgpu.NimSolver(mesh, case.params(precision=_abi.PRECISION_MIXED))
    s.initialize_nse()
    t = s.download(_abi.FACES_T)
    t[mesh.interior_faces.nonzero()[0][5]] = np.nan
    s.upload(_abi.FACES_T, t)
    s.calculate_velocity_nim_constants()
    r = s.integrate_nse(raise_on_error=False)
    assert r.status == _abi.NIM_ERR_NONFINITE
    assert r.iters == r.iters_fp32
    s.close()


@pytest.mark.parametrize("over", [dict(schedule=_abi.SCHEDULE_REFERENCE), dict(formulation=1),
                                  dict(precision=2)])
def test_unsupported_combinations_are_refused(over):
    case = config.small_case(12, 6, 6)
    over = {"precision": _abi.PRECISION_MIXED, **over}
    with pytest.raises(_abi.NimError) as e:
        nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(**over))
    assert e.value.status == _abi.NIM_ERR_BAD_ARG
