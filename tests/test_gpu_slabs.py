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
