"""The oracle's tangent-linear build (oracle/nim_oracle_tl.cpp: the oracle's
source with dual-number values, oracle/nim_dual.h): the FP64 tangent-linear
reference gradient of the hot-wall Nusselt number (find_Nu2,
nse.f90:2794) with respect to Ra, Pr and the outer-wall Dirichlet
temperatures.

* its values are the FP64 oracle's, bit for bit, in both schedules;
* its derivatives match central finite differences of the FP64 oracle with
  relative step 1e-6 (the adjoint's check) to 1e-5, with every inner loop
  converged to changes below 1e-11 (pressure by its gradients) so that the
  Nusselt history is a smooth function of the inputs;
* it is linear in the seeds."""
import numpy as np
import pytest

import oracle as O
from nimgpu import _abi, config

STEPS = 2
TOL = 1e-11
H = 1e-6


def case(**kw):
    return config.small_case(12, 6, 6, steps=STEPS, **kw)


@pytest.fixture(scope="module")
def mesh():
    return O.OracleMesh(case().mesh_params())


def converged(c):
    return c.params(tol_u=TOL, tol_v=TOL, tol_w=TOL, tol_T=TOL, tol_p=TOL, dpdx_tolerance=1,
                    max_iters=100000)


def history(o, tangent=False):
    nus, dnus = [], []
    for _ in range(STEPS):
        st, so = o.step(1)
        assert st == _abi.NIM_OK
        nus.append(so[0].nu_inner)
        if tangent:
            dnus.append(o.nu_tangent()[0])
    return np.array(nus), np.array(dnus)


def start(cls, mesh, c, params, schedule=O.PARALLEL, wall=None):
    # the reference's own order is deterministic on one thread only (its
    # OpenMP loops race, as the reference's do)
    o = cls(mesh, params, schedule=schedule, threads=4 if schedule == O.PARALLEL else 1)
    o.init()
    o.add_temperature_noise(c.noise, c.seed)
    if wall is not None:
        o.set(_abi.FACES_T, o.get(_abi.FACES_T, mesh.nface) + wall)
    return o


def outer_wall(mesh):
    return mesh.bcs_faces[mesh.bcs_faces_id == 5] - 1


@pytest.mark.parametrize("schedule", [O.PARALLEL, O.SEQUENTIAL])
def test_values_are_the_fp64_oracles(mesh, schedule):
    c = case()
    a = start(O.Oracle, mesh, c, c.params(), schedule)
    b = start(O.TangentOracle, mesh, c, c.params(), schedule)
    b.seed_params(*O.TangentOracle.with_respect_to("Ra", c.Ra, c.Pr))
    sa, sb = a.step(STEPS)[1], b.step(STEPS)[1]
    assert [(r.iters, r.nu_inner, r.nu_outer, r.dilatation) for r in sa] == \
        [(r.iters, r.nu_inner, r.nu_outer, r.dilatation) for r in sb]
    for f in (_abi.FACES_U, _abi.FACES_P, _abi.FACES_T, _abi.MESHES_W, _abi.MESHES_T):
        n = mesh.nface if f <= _abi.FACES_T else mesh.nmesh
        assert np.array_equal(a.get(f, n), b.get(f, n))


@pytest.mark.parametrize("name", ["Ra", "Pr"])
def test_parameter_derivatives_match_central_differences(mesh, name):
    c = case()
    o = start(O.TangentOracle, mesh, c, converged(c))
    o.seed_params(*O.TangentOracle.with_respect_to(name, c.Ra, c.Pr))
    _, d = history(o, tangent=True)
    base = c.Ra if name == "Ra" else c.Pr
    side = []
    for sgn in (1, -1):
        v = base * (1 + sgn * H)
        cc = case(Ra=v) if name == "Ra" else case(Pr=v)
        side.append(history(start(O.Oracle, mesh, c, converged(cc)))[0])
    fd = (side[0] - side[1]) / (2 * H * base)
    assert np.all(np.abs(d - fd) <= 1e-5 * np.abs(fd)), (d, fd)


def test_wall_temperature_derivative_matches_central_differences(mesh):
    c = case()
    dirv = np.zeros(mesh.nface)
    w = outer_wall(mesh)
    dirv[w] = np.random.default_rng(7).standard_normal(w.size)
    o = start(O.TangentOracle, mesh, c, converged(c))
    o.set_tangent(_abi.FACES_T, dirv)
    _, d = history(o, tangent=True)
    eps = 1e-6
    vp = history(start(O.Oracle, mesh, c, converged(c), wall=eps * dirv))[0]
    vm = history(start(O.Oracle, mesh, c, converged(c), wall=-eps * dirv))[0]
    fd = (vp - vm) / (2 * eps)
    assert np.all(np.abs(d - fd) <= 1e-5 * np.abs(fd)), (d, fd)


def test_derivatives_are_linear_in_the_seeds(mesh):
    """Seeds a (Ra) + b (wall direction) give a dRa + b dwall, to rounding."""
    c = case()
    dirv = np.zeros(mesh.nface)
    w = outer_wall(mesh)
    dirv[w] = np.random.default_rng(3).standard_normal(w.size)
    sRa = np.array(O.TangentOracle.with_respect_to("Ra", c.Ra, c.Pr))
    outs = []
    for a, b in ((1.0, 0.0), (0.0, 1.0), (2.0, -3.0)):
        o = start(O.TangentOracle, mesh, c, c.params())
        o.seed_params(*(a * sRa))
        o.set_tangent(_abi.FACES_T, b * dirv)
        outs.append(history(o, tangent=True)[1])
    want = 2.0 * outs[0] - 3.0 * outs[1]
    assert np.allclose(outs[2], want, rtol=1e-10, atol=1e-14 * np.abs(want).max())
