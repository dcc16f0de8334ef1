"""Tangent-linear steps on the GPU (nim_gpu_tangent_*, through the C ABI):
the dual instantiations of the step's kernels advance a copy of the state
with its derivative along one seeded direction.

* against the oracle's tangent-linear build (the same seeds, the parallel
  schedule): the per-step iteration counts, the values of every state field
  and their derivatives bit for bit, the Nusselt numbers and their
  derivatives to 1e-12 relative (the GPU sums the wall integrals in another
  order);
* against central finite differences of the FP64 GPU path (every inner
  loop converged to changes below 1e-11, pressure by its gradients):
  d Nu_hot / dRa and dPr with relative step 1e-6, and along a random field
  of outer-wall temperatures with absolute step 1e-4, to 1e-5;
* the context's own FP64 state is untouched by the dual steps."""
import numpy as np
import pytest

import nimgpu
import oracle as O
from nimgpu import _abi, config

pytestmark = pytest.mark.gpu

FIELDS = (_abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
          _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T)


def outer_wall_direction(mesh, seed):
    dirv = np.zeros(mesh.nface)
    w = mesh.bcs_faces[mesh.bcs_faces_id == 5] - 1
    dirv[w] = np.random.default_rng(seed).standard_normal(w.size)
    return dirv


def gpu_solver(case, params):
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), params)
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    return s


@pytest.mark.parametrize("seed", ["Ra", "Pr", "wall"])
def test_dual_steps_match_tangent_oracle(seed):
    case = config.small_case(16, 6, 8, steps=3)
    mesh = nimgpu.Mesh(case.mesh_params())
    params = case.params()
    gpu = gpu_solver(case, params)
    gpu.tangent_begin()
    ref = O.TangentOracle(mesh, params, schedule=O.PARALLEL, threads=4)
    ref.init()
    ref.add_temperature_noise(case.noise, case.seed)
    if seed == "wall":
        dirv = outer_wall_direction(mesh, 11)
        gpu.tangent_seed_field(_abi.FACES_T, dirv)
        ref.set_tangent(_abi.FACES_T, dirv)
    else:
        sd = nimgpu.NimSolver.tangent_seed_of(seed, case.Ra, case.Pr)
        gpu.tangent_seed(*sd)
        ref.seed_params(*sd)
    for step in range(1, case.steps + 1):
        recs, dnu = gpu.tangent_step(1)
        st, so = ref.step(1)
        assert st == _abi.NIM_OK and recs[0].status == _abi.NIM_OK
        assert recs[0].iters == so[0].iters, step
        assert abs(recs[0].nu_inner - so[0].nu_inner) <= 1e-12 * abs(so[0].nu_inner)
        dref = ref.nu_tangent()
        for k in range(2):
            assert abs(dnu[0][k] - dref[k]) <= 1e-12 * abs(dref[k]) + 1e-300, (step, k, dnu[0][k], dref[k])
        for f in FIELDS:
            n = mesh.nface if f <= _abi.FACES_T else mesh.nmesh
            v, t = gpu.tangent_get(f)
            assert np.array_equal(v, ref.get(f, n)), (step, f)
            assert np.array_equal(t, ref.get_tangent(f, n)), (step, f)
    gpu.close()


def test_fp64_state_is_left_alone():
    case = config.small_case(16, 6, 8, steps=2)
    a, b = gpu_solver(case, case.params()), gpu_solver(case, case.params())
    b.tangent_begin()
    b.tangent_seed(*nimgpu.NimSolver.tangent_seed_of("Ra", case.Ra, case.Pr))
    b.tangent_step(2)
    ra, rb = a.solve_nse(2), b.solve_nse(2)
    assert [(r.iters, r.nu_inner) for r in ra] == [(r.iters, r.nu_inner) for r in rb]
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f))
    a.close()
    b.close()


TOL = 1e-11
H = 1e-6


def converged(case):
    return case.params(tol_u=TOL, tol_v=TOL, tol_w=TOL, tol_T=TOL, tol_p=TOL, dpdx_tolerance=1, max_iters=200000)


def nu_history(case, steps, wall=None):
    s = gpu_solver(case, converged(case))
    if wall is not None:
        s.upload(_abi.FACES_T, s.download(_abi.FACES_T) + wall)
    out = np.array([r.nu_inner for r in s.solve_nse(steps)])
    s.close()
    return out


@pytest.mark.parametrize("seed", ["Ra", "Pr", "wall"])
def test_derivatives_match_central_differences(seed):
    case = config.small_case(24, 8, 12, steps=2)
    mesh = nimgpu.Mesh(case.mesh_params())
    s = gpu_solver(case, converged(case))
    s.tangent_begin()
    if seed == "wall":
        dirv = outer_wall_direction(mesh, 5)
        s.tangent_seed_field(_abi.FACES_T, dirv)
    else:
        s.tangent_seed(*nimgpu.NimSolver.tangent_seed_of(seed, case.Ra, case.Pr))
    _, dnu = s.tangent_step(case.steps)
    s.close()
    d = dnu[:, 0]
    if seed == "wall":
        # the outer-wall temperatures are 0, so the step is absolute: 1e-4,
        # which keeps the Nusselt change well above the inner loop's
        # convergence floor (a step of 1e-6 moves Nu by ~1e-10)
        hw = 1e-4
        fd = (nu_history(case, case.steps, hw * dirv) - nu_history(case, case.steps, -hw * dirv)) / (2 * hw)
    else:
        base = case.Ra if seed == "Ra" else case.Pr
        up = config.small_case(24, 8, 12, steps=2, **{seed: base * (1 + H)})
        dn = config.small_case(24, 8, 12, steps=2, **{seed: base * (1 - H)})
        fd = (nu_history(up, case.steps) - nu_history(dn, case.steps)) / (2 * H * base)
    assert np.all(np.abs(d - fd) <= 1e-5 * np.abs(fd)), (d, fd)


def test_tangent_calls_check_their_state():
    case = config.small_case(16, 6, 8)
    s = gpu_solver(case, case.params())
    assert s.lib.nim_gpu_tangent_seed(s._h, 1.0, 1.0) == _abi.NIM_ERR_STATE
    assert s.lib.nim_gpu_tangent_step(s._h, 1, None, None) == _abi.NIM_ERR_STATE
    s.close()
    seq = gpu_solver(case, case.params(schedule=_abi.SCHEDULE_REFERENCE))
    assert seq.lib.nim_gpu_tangent_begin(seq._h) == _abi.NIM_ERR_BAD_ARG
    seq.close()
