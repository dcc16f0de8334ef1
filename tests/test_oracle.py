"""The CPU oracle against the only pins available (no reference test,
fixture or output exists and the Fortran cannot be built here): its own
committed golden fixtures, exact geometric identities, the continuity of
the NIM exact/series branches, the pressure system's null space, the
analytic conduction limit, and schedule independence of the fixed point."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config
import oracle as O

GOLDEN = json.loads((Path(__file__).parent / "golden" / "oracle_golden.json").read_text())
FIELDS = {"faces_u": _abi.FACES_U, "faces_v": _abi.FACES_V, "faces_w": _abi.FACES_W, "faces_p": _abi.FACES_P,
          "faces_T": _abi.FACES_T, "meshes_u": _abi.MESHES_U, "meshes_v": _abi.MESHES_V,
          "meshes_w": _abi.MESHES_W, "meshes_T": _abi.MESHES_T}


def _case(name):
    if name.startswith("reference"):
        return config.reference_mesh(), config.reference_params(), None
    sc = config.small_case(16, 6, 6)
    if name.startswith("formulation1"):
        return sc.mesh_params(), sc.params(formulation=1), (sc.noise, sc.seed)
    return sc.mesh_params(), sc.params(), (sc.noise, sc.seed)


@pytest.mark.parametrize("gold", GOLDEN, ids=[g["name"] for g in GOLDEN])
@pytest.mark.parametrize("sched", ["sequential", "parallel"])
def test_golden_fixture(gold, sched):
    mp, p, noise = _case(gold["name"])
    mesh = nimgpu.Mesh(mp)
    o = O.Oracle(mesh, p, schedule=O.SEQUENTIAL if sched == "sequential" else O.PARALLEL)
    o.init()
    if noise:
        nimgpu.apply_temperature_noise(o.get, o.set, mesh, *noise)
    st, recs = o.step(gold["steps"])
    assert st == 0
    for r, g in zip(recs, gold[sched]["stats"]):
        assert r.iters == g["iters"]
        for k in ("nu_inner", "nu_outer", "dilatation", "area_inner", "area_outer", "err_T"):
            assert getattr(r, k) == pytest.approx(g[k], rel=1e-11, abs=1e-300), k
    for name, f in FIELDS.items():
        n = mesh.nface if f <= _abi.FACES_T else mesh.nmesh
        v = o.get(f, n)
        g = gold[sched]["fields"][name]
        scale = max(g["max_abs"], 1e-300)
        assert np.max(np.abs(v[g["idx"]] - np.array(g["samples"]))) <= 1e-11 * scale, name


def test_convection_correction_is_zero():
    """calculate_R_c_new (nse.f90:1393-1434) subtracts two copies of the same
    expression; R_C must be exactly 0 in the reference order."""
    mesh = nimgpu.Mesh(config.reference_mesh())
    o = O.Oracle(mesh, config.reference_params(), schedule=O.SEQUENTIAL)
    o.init()
    o.step(2)
    assert o.max_rc() == 0.0


def test_volumes_and_wall_areas_are_exact():
    """Cells are vertical prisms over plane quadrilaterals: the 125-point
    volume integral is exact, so the sum equals the shoelace areas times
    dz; the wall areas equal the polygon perimeters times the height."""
    mesh = nimgpu.Mesh(config.reference_mesh())
    o = O.Oracle(mesh, config.reference_params())
    o.init()
    vol = o.get(_abi.MESHES_VOLUME, mesh.nmesh)
    xyz = mesh.node_xyz
    nd = mesh.meshes_nodes - 1
    q = xyz[nd[:, [0, 1, 2, 3]], :2]            # bottom quad, nodes 1-2-3-4
    x, y = q[..., 0], q[..., 1]
    shoelace = 0.5 * np.abs((x * np.roll(y, -1, 1) - np.roll(x, -1, 1) * y).sum(1))
    dz = xyz[nd[:, 4], 2] - xyz[nd[:, 0], 2]
    assert np.allclose(vol, shoelace * dz, rtol=1e-12, atol=0)
    area = o.get(_abi.FACES_AREA, mesh.nface)
    inner = mesh.bcs_faces[mesh.bcs_faces_position == 1] - 1
    n1, n2, n3 = 36, 6, 12
    ring = xyz.reshape(n3 + 1, n2 + 1, n1, 3)[0, 0, :, :2]
    perim = np.linalg.norm(ring - np.roll(ring, -1, 0), axis=1).sum()
    assert area[inner].sum() == pytest.approx(perim * 2.0, rel=1e-12)


@pytest.mark.parametrize("Re", [-0.05, -0.01, -0.003, 0.003, 0.01, 0.05])
def test_nim_series_and_exact_branches_agree(Re):
    """nim.f90:184-287: the 10th-order series and the exponential form of
    M_A must agree where the code switches between them.  The exponential
    form cancels: exp(Re)-1 carries eps/Re, and M_A(.,5) subtracts k from
    k(1 + Re^2/12), so it keeps only ~12 eps/|Re|^3; the others lose eps/Re^2."""
    eps = 2.2e-16
    k = 0.37
    u = Re * k / 2
    series = O.nim_coefficients(u, k, 0.9, 1.1, v_limit=1e300)
    exact = O.nim_coefficients(u, k, 0.9, 1.1, v_limit=0.0)
    tol = np.full(6, 1e-12 + 40 * eps / Re ** 2 + abs(Re) ** 11)
    tol[4] = 1e-12 + 30 * eps / abs(Re) ** 3
    assert np.all(np.abs(series - exact) <= tol * np.abs(exact))


@pytest.mark.parametrize("Re", [-0.05, -0.01, -0.003, 0.003, 0.01, 0.05])
def test_formulation1_series_and_exact_branches_agree(Re):
    """nim.f90:758-875: C, E, F, G, H, I, J_nim in their series and
    exponential forms agree where condition() switches between them, up to
    the exponential form's cancellation (C: ~eps/|Re|^3; the others
    ~eps/Re^2) and the series' truncation.  B_nim is 0 in the series branch
    by definition and enters only the exponential forms."""
    eps = 2.2e-16
    F, D = 0.37, -1.7
    u = Re * F / 2
    series = O.nim1_coefficients(u, F, D, v_limit=1e300)[1:]
    exact = O.nim1_coefficients(u, F, D, v_limit=0.0)[1:]
    tol = np.full(7, 1e-12 + 200 * eps / Re ** 2 + 100 * abs(Re) ** 9)
    tol[0] += 10 * eps / abs(Re) ** 3
    assert np.all(np.abs(series - exact) <= tol * np.abs(exact))


def test_pressure_system_has_constant_null_space():
    """The pressure equations are of pure-Neumann type: a constant shift of
    all face pressures solves the homogeneous system (sum of the 11 face
    coefficients and of the 6 wall coefficients is zero)."""
    mesh = nimgpu.Mesh(config.small_case(16, 6, 6).mesh_params())
    o = O.Oracle(mesh, config.small_case().params())
    o.init()
    for f in (_abi.AA_PX, _abi.AA_PY, _abi.AA_PZ):
        A = o.get(f, 15 * mesh.nmesh).reshape(mesh.nmesh, 15)[:, :11]
        live = np.abs(A).sum(1) > 0
        assert live.any()
        assert np.all(np.abs(A[live].sum(1)) <= 1e-12 * np.abs(A[live]).sum(1))
    ap = o.get(_abi.BCS_FACES_AP, 8 * mesh.nbcface).reshape(mesh.nbcface, 8)[:, :6]
    assert np.all(np.abs(ap.sum(1)) <= 1e-12 * np.abs(ap).sum(1))


@pytest.mark.parametrize("formulation", [2, 1])
def test_conduction_limit_nusselt(formulation):
    """Concentric annulus (no hexagon), negligible buoyancy: both wall
    Nusselt numbers tend to 1/ln(R_o/R_i).  The inner wall shows the time
    element's odd/even oscillation at this large step, so two steps are
    averaged."""
    mp = config.reference_mesh(n_theta=18, n_r=6, n_z=3, R_i=0.5, R_o=1.0, L=1.0, cluster=0, hexagon=0)
    mesh = nimgpu.Mesh(mp)
    p = config.reference_params(Ra=1.0, Pr=1.0, DT=0.05, R_i=0.5, R_o=1.0, formulation=formulation)
    o = O.Oracle(mesh, p)
    o.init()
    st, recs = o.step(40)
    assert st == 0 and len(recs) == 40
    exact = 1.0 / math.log(2.0)
    inner = -(recs[-1].nu_inner + recs[-2].nu_inner) / 2
    outer = -recs[-1].nu_outer
    assert inner == pytest.approx(exact, rel=0.05)
    assert outer == pytest.approx(exact, rel=0.05)


def test_both_orders_reach_the_same_fixed_point():
    """Sequential (reference) and parallel (kernel) order, converged to
    1e-13 on the pressure gradients: T and Nu agree to <= 1e-10."""
    case = config.small_case(12, 6, 6)
    mesh = nimgpu.Mesh(case.mesh_params())
    tight = dict(tol_u=1e-13, tol_v=1e-13, tol_w=1e-13, tol_T=1e-13, tol_p=1e-13, dpdx_tolerance=1,
                 max_iters=200000)
    out = []
    for sched in (O.SEQUENTIAL, O.PARALLEL):
        o = O.Oracle(mesh, case.params(**tight), schedule=sched)
        o.init()
        nimgpu.apply_temperature_noise(o.get, o.set, mesh, case.noise, case.seed)
        st, recs = o.step(2)
        assert st == 0
        out.append((recs, o.get(_abi.FACES_T, mesh.nface), o.get(_abi.MESHES_T, mesh.nmesh)))
    (ra, fa, ca), (rb, fb, cb) = out
    for a, b in zip(ra, rb):
        assert a.nu_inner == pytest.approx(b.nu_inner, rel=1e-10)
        assert a.nu_outer == pytest.approx(b.nu_outer, rel=1e-10)
    assert np.abs(fa - fb).max() <= 1e-10 * np.abs(fb).max()
    assert np.abs(ca - cb).max() <= 1e-10 * np.abs(cb).max()


@pytest.mark.parametrize("dims,formulation", [((12, 6, 6), 2), ((16, 5, 7), 2), ((6, 4, 4), 2), ((7, 3, 9), 2),
                                              ((12, 6, 6), 1), ((7, 3, 9), 1)])
def test_level_order_reproduces_reference_order(dims, formulation):
    """The CUDA library's reference-order schedule sweeps cells by the level
    i + 2j + 3k and wall faces by their in-wall level.  The oracle's LEVELS
    order visits them that way (numbers descending inside a level, walls top
    before bottom and outer before inner) with the reference's arithmetic:
    bit-for-bit equal to the reference's number order over whole steps, so no
    sweep dependence joins two faces or cells that share a level."""
    case = config.small_case(*dims)
    mesh = nimgpu.Mesh(case.mesh_params())
    out = []
    for sched in (O.SEQUENTIAL, O.LEVELS):
        o = O.Oracle(mesh, case.params(formulation=formulation), schedule=sched)
        o.init()
        nimgpu.apply_temperature_noise(o.get, o.set, mesh, case.noise, case.seed)
        st, recs = o.step(2)
        assert st == 0
        out.append(([r.iters for r in recs], [o.get(f, nimgpu.field_len(f, mesh)) for f in range(19)]))
    (ia, fa), (ib, fb) = out
    assert ia == ib
    for f, (a, b) in enumerate(zip(fa, fb)):
        assert np.array_equal(a, b), f"field {f}"


def test_iteration_cap_and_nonfinite():
    mesh = nimgpu.Mesh(config.small_case().mesh_params())
    o = O.Oracle(mesh, config.small_case().params(max_iters=2))
    o.init()
    o.begin_step()
    s = o.integrate()
    assert s.status == _abi.NIM_ERR_NOT_CONVERGED and s.iters == 2
