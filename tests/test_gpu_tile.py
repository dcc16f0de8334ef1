"""The TMA-staged sweeps of u, v, w: k_vel_face_tile (+xi face updates,
nse.f90:878-1005) and k_vel_cell_tile (sources and cell update,
nse.f90:199-211, 839-872), which march up z in chunks with their face
operands staged in shared memory by TMA boxes.  They replace k_vel_face and
k_vel_cell when n_theta is a multiple of 4 (at most 256): the face sweep by
itself when the mesh fills the GPU with blocks, the cell sweep on request
(NIM_CELL_SWEEP=tile); NIM_FACE_SWEEP=tile forces the face sweep on the
small meshes here.  Each restates its gather twin with the same
arithmetic, so the passes match the CPU oracle's parallel schedule to
round-off and the two forms agree to the bit.  The meshes below reach every
edge of the tiling: several z-chunks, both z walls and the top level, theta
tiles that read real halo columns, seam tiles on both sides (one of fewer
than 32 cells), and patches cut short in r."""
import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def force_tile(monkeypatch):
    monkeypatch.setenv("NIM_FACE_SWEEP", "tile")
    monkeypatch.setenv("NIM_CELL_SWEEP", "tile")


STATE = [
    _abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
    _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T,
]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(dims, **over):
    case = config.small_case(*dims)
    mesh = nimgpu.Mesh(case.mesh_params())
    p = case.params(**over)
    gpu = nimgpu.NimSolver(mesh, p)
    gpu.initialize_nse()
    gpu.add_temperature_noise(case.noise, case.seed)
    ref = O.Oracle(mesh, p, schedule=O.PARALLEL)
    ref.init()
    nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, case.noise, case.seed)
    return gpu, ref


@pytest.mark.parametrize("dims", [(40, 6, 30), (12, 5, 13), (36, 9, 12), (64, 4, 25)])
def test_tiled_passes_match_parallel_oracle(dims):
    gpu, ref = pair(dims)
    prof = gpu.profile_iterations(1)
    assert "k_vel_face_tile" in prof and "k_vel_cell_tile" in prof
    gpu.close()
    gpu, ref = pair(dims)
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    sg, so = gpu.iterate(3), ref.iterate(3)
    for k in ("err_u", "err_v", "err_w", "err_p", "err_T"):
        assert getattr(sg, k) == getattr(so, k), k
    for f in STATE:
        a = gpu.download(f)
        assert np.array_equal(a, ref.get(f, a.size)), f
    gpu.close()


def test_tiled_steps_match_parallel_oracle():
    gpu, ref = pair((40, 6, 14))
    sg = gpu.solve_nse(2)
    _, so = ref.step(2)
    assert [a.iters for a in sg] == [b.iters for b in so]
    for a, b in zip(sg, so):
        assert abs(a.nu_inner - b.nu_inner) <= 1e-13 * abs(b.nu_inner)
    for f in STATE:
        a = gpu.download(f)
        assert np.array_equal(a, ref.get(f, a.size)), f
    gpu.close()


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_tile_and_gather_forms_are_bitwise_equal(monkeypatch, precision):
    """Same arithmetic on the same stored values: whole steps agree to the
    bit in FP64 and in the mixed path's FP32 passes."""
    case = config.small_case(40, 6, 26, steps=2)
    outs = []
    for form in ("gather", "tile"):
        monkeypatch.setenv("NIM_FACE_SWEEP", form)
        monkeypatch.setenv("NIM_CELL_SWEEP", form)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(precision=precision))
        s.initialize_nse()
        s.add_temperature_noise(case.noise, case.seed)
        recs = s.solve_nse(2)
        outs.append(([(r.iters, r.iters_fp32, r.nu_inner) for r in recs], [s.download(f) for f in STATE]))
        prof = s.profile_iterations(1)
        suffix = "_tile" if form == "tile" else ""
        assert "k_vel_face" + suffix in prof and "k_vel_cell" + suffix in prof
        s.close()
    assert outs[0][0] == outs[1][0]
    for a, b in zip(outs[0][1], outs[1][1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
@pytest.mark.parametrize("dims", [(40, 6, 26), (130, 5, 7)])
def test_pair_and_gather_cell_sweeps_are_bitwise_equal(monkeypatch, precision, dims):
    """k_vel_cell2 (two theta-adjacent cells per thread, paired loads), and
    in FP64 k_p_srcN / k_p_faceN with two cells a thread, against k_vel_cell,
    k_p_src and k_p_face: whole steps to the bit (theta seams, walls, a
    partial 64-cell patch)."""
    case = config.small_case(*dims, steps=2)
    monkeypatch.setenv("NIM_FACE_SWEEP", "gather")
    outs = []
    for form in ("gather", "pair"):
        monkeypatch.setenv("NIM_CELL_SWEEP", form)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(precision=precision))
        s.initialize_nse()
        s.add_temperature_noise(case.noise, case.seed)
        recs = s.solve_nse(2)
        outs.append(([(r.iters, r.iters_fp32, r.nu_inner) for r in recs], [s.download(f) for f in STATE]))
        prof = s.profile_iterations(1)
        assert ("k_vel_cell2" if form == "pair" else "k_vel_cell") in prof
        if precision == _abi.PRECISION_FP64:  # the FP64 pressure sweeps take the pairs too
            want = ("k_p_srcN", "k_p_faceN") if form == "pair" else ("k_p_src", "k_p_face")
            assert all(k in prof for k in want), list(prof)
        s.close()
    assert outs[0][0] == outs[1][0]
    for a, b in zip(outs[0][1], outs[1][1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("dims", [(40, 6, 26), (132, 5, 7)])
def test_quad_and_pair_float_cell_sweeps_are_bitwise_equal(monkeypatch, dims):
    """The mixed path's FP32 passes with the four-cells-a-thread sweeps
    (k_vel_cellN, k_vel_faceN, k_p_srcN, k_p_faceN, k_T_cellN, k_T_faceN:
    float4 loads; the default for n_theta % 4 == 0 when n_theta / 4 fills
    3/4 of a warp, forced here) against k_vel_cell2,
    k_vel_face, k_p_src, k_p_face, k_T_cell and k_T_face: whole steps to
    the bit (theta seams, walls, a partial 128-cell patch)."""
    case = config.small_case(*dims, steps=2)
    outs = []
    for form, kernels in (("pair", ("k_vel_cell2", "k_vel_face", "k_p_src", "k_p_face", "k_T_cell", "k_T_face")),
                          ("quad", ("k_vel_cellN", "k_vel_faceN", "k_p_srcN", "k_p_faceN", "k_T_cellN", "k_T_faceN"))):
        monkeypatch.setenv("NIM_CELL_SWEEP", form)  # quad: forced on these narrow meshes
        if form == "pair":
            monkeypatch.setenv("NIM_FACE_SWEEP", "gather")
        else:
            monkeypatch.delenv("NIM_FACE_SWEEP", raising=False)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(precision=_abi.PRECISION_MIXED))
        s.initialize_nse()
        s.add_temperature_noise(case.noise, case.seed)
        recs = s.solve_nse(2)
        outs.append(([(r.iters, r.iters_fp32, r.nu_inner) for r in recs], [s.download(f) for f in STATE]))
        prof = s.profile_iterations(1)
        assert all(k in prof for k in kernels), list(prof)
        s.close()
    assert outs[0][0] == outs[1][0]
    assert all(r[1] > 0 for r in outs[0][0])  # the FP32 phase ran
    for a, b in zip(outs[0][1], outs[1][1]):
        assert np.array_equal(a, b)


def test_n_cell_forms_follow_lane_use(monkeypatch):
    """Without an override the NP-cells-a-thread sweeps run only when
    n_theta / NP threads fill at least 3/4 of a warp's lanes: four float
    cells at n_theta = 128 and 96, not at 40; two FP64 cells in the pressure
    sweeps at n_theta = 64 and 48, not at 40."""
    monkeypatch.delenv("NIM_FACE_SWEEP", raising=False)
    monkeypatch.delenv("NIM_CELL_SWEEP", raising=False)
    for nt, quad in ((128, True), (96, True), (40, False)):
        case = config.small_case(nt, 8, 6)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(precision=_abi.PRECISION_MIXED))
        s.initialize_nse()
        prof = s.profile_iterations(1)  # the FP32 passes
        assert ("k_vel_cellN" in prof) == quad and ("k_p_faceN" in prof) == quad, (nt, list(prof))
        s.close()
    for nt, pair in ((64, True), (48, True), (40, False)):
        case = config.small_case(nt, 8, 6)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params())
        s.initialize_nse()
        prof = s.profile_iterations(1)
        assert ("k_p_srcN" in prof) == pair and ("k_p_faceN" in prof) == pair, (nt, list(prof))
        s.close()


def test_automatic_choice(monkeypatch):
    """Without the override: the tile form on a mesh with enough patches,
    the gather form on one that cannot fill the GPU."""
    monkeypatch.delenv("NIM_FACE_SWEEP")
    monkeypatch.delenv("NIM_CELL_SWEEP")
    for dims, suffix in (((128, 128, 48), "_tile"), ((128, 64, 32), "")):
        case = config.small_case(*dims)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params())
        s.initialize_nse()
        prof = s.profile_iterations(1)
        # the cell sweep: the paired-load form for even n_theta, the tile only on request
        assert "k_vel_face" + suffix in prof and "k_vel_cell2" in prof
        s.close()


def test_kernel_choice_follows_n_theta(monkeypatch):
    """With both tiles requested: n_theta = 16 gets them; 18 (not a multiple
    of 4) keeps the gather face sweep and the paired cell sweep; 19 (odd)
    the gather forms of both."""
    for nt, face, cell in ((16, "k_vel_face_tile", "k_vel_cell_tile"), (18, "k_vel_face", "k_vel_cell2"),
                           (19, "k_vel_face", "k_vel_cell")):
        case = config.small_case(nt, 5, 6)
        s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params())
        s.initialize_nse()
        prof = s.profile_iterations(1)
        names = [k for k in prof if k.startswith("k_vel_")]
        assert names == [cell, face], names
        s.close()


def test_formulation_one_keeps_the_gather_cell_sweep():
    case = config.small_case(16, 5, 6)
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()),
                         case.params(formulation=1, schedule=_abi.SCHEDULE_PARALLEL))
    s.initialize_nse()
    prof = s.profile_iterations(1)
    assert "k_vel_cell" in prof and "k_vel_cell_tile" not in prof
    s.close()


def test_plain_face_kernel_matches_parallel_oracle():
    """n_theta = 18 (not a multiple of 4) keeps the gather form."""
    gpu, ref = pair((18, 6, 7))
    gpu.calculate_velocity_nim_constants()
    ref.begin_step()
    gpu.iterate(3)
    ref.iterate(3)
    for f in (_abi.FACES_U, _abi.FACES_W, _abi.FACES_T):
        a = gpu.download(f)
        assert rel(a, ref.get(f, a.size)) <= 1e-12
    gpu.close()
