"""z-slab decomposition on one device (nim_gpu_create_slab + nim_slab_step):
the owned planes of a group of slabs, with the halo exchange after each
part of every pass and the merged maxima, hold exactly the whole-mesh
context's fields with the same iteration counts; the group's dilatation and
Nusselt numbers are the whole mesh's sums in another order."""
import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config

pytestmark = pytest.mark.gpu

FIELDS = [_abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T, _abi.MESHES_P,
          _abi.FACES_U, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T]


# a bound well above the passes these steps take, so a wrong exchange ends
# the step with NIM_ERR_NOT_CONVERGED instead of running on
CAP = dict(max_iters=5000)


def whole(case, steps):
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(**CAP))
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    recs = s.solve_nse(steps)
    out = [s.download(f) for f in FIELDS]
    s.close()
    return recs, out


# even n_theta: the paired cell sweep; odd: one cell per thread
@pytest.mark.parametrize("dims,nslab", [((16, 12, 12), 2), ((16, 12, 12), 3), ((16, 12, 12), 6), ((15, 10, 9), 2)])
def test_slabs_equal_whole_mesh(dims, nslab):
    case = config.small_case(*dims, Ra=1e5, steps=3)
    want_recs, want = whole(case, case.steps)
    mesh = nimgpu.Mesh(case.mesh_params())
    with nimgpu.SlabGroup(mesh, case.params(**CAP), nslab) as g:
        g.initialize_nse()
        g.add_temperature_noise(case.noise, case.seed)
        recs = g.solve_nse(case.steps)
        assert len(recs) == len(want_recs)
        for r, w in zip(recs, want_recs):
            assert (r.step, r.iters, r.status) == (w.step, w.iters, w.status)
            for a in ("err_u", "err_v", "err_w", "err_p", "err_T", "dudt_max", "dTdt_max", "time"):
                assert getattr(r, a) == getattr(w, a), a
            for a in ("dilatation", "nu_inner", "nu_outer", "area_inner", "area_outer"):
                assert getattr(r, a) == pytest.approx(getattr(w, a), rel=1e-10, abs=1e-300), a
        for f, w in zip(FIELDS, want):
            got = g.gather(f)
            assert np.array_equal(got, w), f


def test_slab_group_checks_its_members():
    case = config.small_case(16, 12, 12)
    mesh = nimgpu.Mesh(case.mesh_params())
    lib = _abi.gpu_lib()
    import ctypes as C
    # the reference order, formulation 1 and mixed precision are whole-mesh only
    for over in (dict(schedule=_abi.SCHEDULE_REFERENCE), dict(formulation=1),
                 dict(precision=_abi.PRECISION_MIXED)):
        h = C.c_void_p()
        st = lib.nim_gpu_create_slab(C.byref(mesh.desc), C.byref(case.params(**over)), 2, 0, C.byref(h))
        assert st == _abi.NIM_ERR_BAD_ARG
    with nimgpu.SlabGroup(mesh, case.params(), 3) as g:
        g.initialize_nse()
        n = 3
        wrong = (C.c_void_p * 2)(g._h[0].value, g._h[1].value)  # two of three slabs
        assert lib.nim_slab_step(2, wrong, 1, None, None) == _abi.NIM_ERR_BAD_ARG
        swapped = (C.c_void_p * n)(g._h[1].value, g._h[0].value, g._h[2].value)
        assert lib.nim_slab_step(n, swapped, 1, None, None) == _abi.NIM_ERR_BAD_ARG
        # a slab alone would step with a stale halo
        assert lib.nim_gpu_step(g._h[1], 1, None, None) == _abi.NIM_ERR_BAD_ARG
        one = (C.c_void_p * 1)(g._h[0].value)
        assert lib.nim_batch_step(1, one, 1, None, None) == _abi.NIM_ERR_BAD_ARG


def test_slab_rank_single_process_equals_whole_mesh():
    """SlabRank drives the pass part by part with the maxima all-reduced over
    a one-rank NCCL group (no neighbour: the exchange is empty); the result
    is the whole-mesh context's to the bit."""
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist
    case = config.small_case(16, 12, 12, Ra=1e5, steps=3)
    want_recs, want = whole(case, case.steps)
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        r = nimgpu.SlabRank(nimgpu.Mesh(case.mesh_params()), case.params(**CAP))
        r.initialize_nse()
        r.add_temperature_noise(case.noise, case.seed)
        recs = r.solve_nse(case.steps)
        assert [(x.step, x.iters, x.status) for x in recs] == [(w.step, w.iters, w.status) for w in want_recs]
        for x, w in zip(recs, want_recs):
            for a in ("err_u", "err_v", "err_w", "err_p", "err_T", "dudt_max", "dTdt_max", "time", "nu_inner",
                      "nu_outer", "dilatation"):
                assert getattr(x, a) == getattr(w, a), a
        for f, w in zip(FIELDS, want):
            assert np.array_equal(r.gather(f), w), f
        r.close()
    finally:
        dist.destroy_process_group()


def test_pack_unpack_restores_halos():
    """nim_slab_pack / nim_slab_unpack between the slabs of one device (no
    collective): halos overwritten with junk, the whole state moved through
    packed device buffers, every held plane again holds the whole mesh's
    values (cells, and the faces of the current half)."""
    import ctypes as C

    import torch
    from nimgpu.slabs import HALO_STATE, slab_face_planes, structured_faces
    case = config.small_case(16, 12, 12, Ra=1e5)
    mesh = nimgpu.Mesh(case.mesh_params())
    ref = structured_faces(mesh)
    pl = mesh.n_theta * mesh.n_r
    offZ = mesh.n_theta * (mesh.n_r + 1) * mesh.n_z + pl * mesh.n_z
    w = nimgpu.NimSolver(mesh, case.params())
    w.initialize_nse()
    w.add_temperature_noise(1e-3, 5)
    cells_T, faces_T = w.download(_abi.MESHES_T), w.download(_abi.FACES_T)
    w.close()
    with nimgpu.SlabGroup(mesh, case.params(), 3) as g:
        g.initialize_nse()
        g.add_temperature_noise(1e-3, 5)
        for s in g.slabs:
            lo, hi, olo, ohi = g.layout[s]
            c = g.download(s, _abi.MESHES_T)
            for k in range(lo, hi):
                if not olo <= k < ohi:
                    c[(k - lo) * pl:(k - lo + 1) * pl] = -7.0
            g.upload(s, _abi.MESHES_T, c)
            glob, plane = slab_face_planes(mesh, lo, hi)
            z = glob >= offZ
            own = (plane >= olo) & (plane < ohi)
            halo = np.where(z, ~(own | ((plane - 1 >= olo) & (plane - 1 < ohi))), ~own)
            f = g.download(s, _abi.FACES_T)
            f[halo] = -7.0
            g.upload(s, _abi.FACES_T, f)
        lib = g.lib
        for s in range(g.nslab - 1):
            for a, sa, b, sb in ((s, 1, s + 1, 0), (s + 1, 0, s, 1)):
                ha, hb = g._handle(a), g._handle(b)
                n = lib.nim_slab_pack_doubles(ha, HALO_STATE, sa)
                assert n == lib.nim_slab_pack_doubles(hb, HALO_STATE, sb) > 0
                buf = torch.empty(n, dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                _abi.check(lib.nim_slab_pack(ha, HALO_STATE, sa, C.c_void_p(buf.data_ptr())), "nim_slab_pack")
                _abi.check(lib.nim_gpu_synchronize(ha), "sync")
                _abi.check(lib.nim_slab_unpack(hb, HALO_STATE, sb, C.c_void_p(buf.data_ptr())), "nim_slab_unpack")
                _abi.check(lib.nim_gpu_synchronize(hb), "sync")
        for s in g.slabs:
            lo, hi = g.layout[s][:2]
            assert np.array_equal(g.download(s, _abi.MESHES_T), cells_T[lo * pl:hi * pl])
            glob, _ = slab_face_planes(mesh, lo, hi)
            assert np.array_equal(g.download(s, _abi.FACES_T), faces_T[ref[glob]])
        assert lib.nim_slab_pack_doubles(g._handle(0), HALO_STATE, 0) == _abi.NIM_ERR_BAD_ARG  # no slab below 0


def test_slabs_with_tiled_face_sweep(monkeypatch):
    """Slab contexts running the TMA-staged face sweep (its per-plane masked
    maxima), forced on a small mesh: still the whole mesh's fields and
    iteration counts."""
    import ctypes as C
    case = config.small_case(16, 12, 12, Ra=1e5, steps=3)
    want_recs, want = whole(case, case.steps)
    monkeypatch.setenv("NIM_FACE_SWEEP", "tile")
    mesh = nimgpu.Mesh(case.mesh_params())
    with nimgpu.SlabGroup(mesh, case.params(**CAP), 3) as g:
        g.initialize_nse()
        g.add_temperature_noise(case.noise, case.seed)
        recs = g.solve_nse(case.steps)
        assert [(r.iters, r.err_u, r.err_T) for r in recs] == [(w.iters, w.err_u, w.err_T) for w in want_recs]
        for f, w in zip(FIELDS, want):
            assert np.array_equal(g.gather(f), w), f
        # the slabs did run the staged sweep
        ms = (C.c_double * 32)()
        h = g._handle(1)
        nk = g.lib.nim_gpu_profile_iterations(h, 1, ms, 32)
        assert nk > 0
        assert "k_vel_face_tile" in [g.lib.nim_gpu_profile_name(h, k).decode() for k in range(nk)]


def test_nusselt_noalloc_on_slabs_combines_to_whole_mesh():
    """nim_gpu_nusselt_noalloc on a z-slab context sums over the slab's owned
    planes only: the slabs' Nusselt numbers, weighted by their wall areas,
    give the whole mesh's."""
    import ctypes as C
    case = config.small_case(16, 12, 12, Ra=1e5, steps=2)
    want_recs, _ = whole(case, case.steps)
    w = want_recs[-1]
    mesh = nimgpu.Mesh(case.mesh_params())
    with nimgpu.SlabGroup(mesh, case.params(**CAP), 2) as g:
        g.initialize_nse()
        g.add_temperature_noise(case.noise, case.seed)
        g.solve_nse(case.steps)
        parts = []
        for s in g.slabs:
            out = (C.c_double * 4)()
            st = g.lib.nim_gpu_nusselt_noalloc(g._handle(s), out)
            assert st == _abi.NIM_OK, _abi.strerror(st)
            parts.append(list(out))
    area_out = sum(p[2] for p in parts)
    area_in = sum(p[3] for p in parts)
    nu_out = sum(p[0] * p[2] for p in parts) / area_out
    nu_in = sum(p[1] * p[3] for p in parts) / area_in
    # each slab holds part of each wall, not all of it
    assert all(0 < p[3] < w.area_inner for p in parts)
    assert area_out == pytest.approx(w.area_outer, rel=1e-12)
    assert area_in == pytest.approx(w.area_inner, rel=1e-12)
    assert nu_out == pytest.approx(w.nu_outer, rel=1e-12)
    assert nu_in == pytest.approx(w.nu_inner, rel=1e-12)
