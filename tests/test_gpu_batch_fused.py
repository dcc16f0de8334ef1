"""nim_batch_step_fused: every kernel of a pass launched once for the whole
batch, each launch a persistent grid walking a work list of (enclosure,
block) items.  Per enclosure the arithmetic is that of its own launches, so
every record and every field equals, bit for bit, what nim_gpu_step gives
for that enclosure alone, in FP64 and in the mixed FP32/FP64 inner loop;
enclosures leave the work list when their own loop stops."""
import ctypes as C

import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config

pytestmark = pytest.mark.gpu

STATE = [_abi.FACES_U, _abi.FACES_V, _abi.FACES_P, _abi.FACES_T, _abi.MESHES_U, _abi.MESHES_W, _abi.MESHES_T,
         _abi.MESHES_TT]


def make(case, **kw):
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(**kw))
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    return s


def records(recs):
    return [(r.status, r.iters, r.iters_fp32, r.nu_inner, r.nu_outer, r.dilatation, r.err_u, r.err_T, r.time)
            for r in recs]


def uneven_cases():
    # odd and even n_theta (one-cell and paired velocity sweeps), n_theta up
    # to 48 (the paired FP64 pressure sweeps), uneven Ra and Pr
    cases = config.batch_cases(5, seed=7, a_min=9, a_max=48)
    for c, Ra in zip(cases, (1e4, 3e3, 1e5, 2e4, 5e4)):
        c.Ra = Ra
    return cases


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_fused_batch_equals_one_at_a_time(precision):
    cases = uneven_cases()
    alone = []
    for c in cases:
        s = make(c, precision=precision)
        recs = s.solve_nse(3)
        alone.append((records(recs), [s.download(f) for f in STATE]))
        s.close()
    batch = [make(c, precision=precision) for c in cases]
    recs = nimgpu.batch_step(batch, 3, fused=True)
    for s, r, (want_recs, want_fields) in zip(batch, recs, alone):
        assert records(r) == want_recs
        for f, w in zip(STATE, want_fields):
            assert np.array_equal(s.download(f), w), f
    # the contexts carry on alone afterwards, on their own streams
    more = [s.solve_nse(1)[0].iters for s in batch]
    assert all(m > 0 for m in more)
    for s in batch:
        s.close()


def test_fused_batch_against_the_oracle():
    import oracle as O
    case = config.small_case(16, 6, 8, steps=2)
    mesh = nimgpu.Mesh(case.mesh_params())
    params = case.params()
    other = config.small_case(21, 7, 6, Ra=3e4)
    batch = [make(case), make(other)]
    recs = nimgpu.batch_step(batch, 2, fused=True)
    ref = O.Oracle(mesh, params, schedule=O.PARALLEL, threads=4)
    ref.init()
    nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, case.noise, case.seed)
    _, so = ref.step(2)
    assert [r.iters for r in recs[0]] == [r.iters for r in so]
    for f in STATE:
        a = batch[0].download(f)
        assert np.array_equal(a, ref.get(f, a.size)), f
    for s in batch:
        s.close()


def test_fused_batch_stops_each_instance_on_its_own():
    cases = config.batch_cases(3, seed=11, a_min=8, a_max=14)
    solvers = [make(cases[0]), make(cases[1], max_iters=3), make(cases[2])]
    lib = _abi.gpu_lib()
    n, nsteps = 3, 2
    h = (C.c_void_p * n)(*[s._h.value for s in solvers])
    per = (_abi.StepStats * (n * nsteps))()
    done = (C.c_int32 * n)()
    st = lib.nim_batch_step_fused(n, h, nsteps, per, done)
    assert st == _abi.NIM_ERR_NOT_CONVERGED
    assert list(done) == [2, 1, 2]
    assert per[1 * nsteps].status == _abi.NIM_ERR_NOT_CONVERGED and per[1 * nsteps].iters == 3
    for s in solvers:
        s.close()


def test_fused_batch_arguments():
    lib = _abi.gpu_lib()
    a = make(config.small_case())
    b = make(config.small_case(), precision=_abi.PRECISION_MIXED)
    seq = make(config.small_case(), schedule=_abi.SCHEDULE_REFERENCE)
    for pair in ((a, a), (a, b), (a, seq)):
        h = (C.c_void_p * 2)(*[s._h.value for s in pair])
        assert lib.nim_batch_step_fused(2, h, 1, None, None) == _abi.NIM_ERR_BAD_ARG
    for s in (a, b, seq):
        s.close()


def test_grid_form_equals_persistent_form(monkeypatch):
    """NIM_BATCH_FORM=grid: the pass kernels as plain launches over groups of
    enclosures whose arguments are kernel parameters; the same bits as the
    persistent form and as one at a time."""
    cases = uneven_cases()[:3]
    alone = []
    for c in cases:
        s = make(c, precision=_abi.PRECISION_MIXED)
        alone.append((records(s.solve_nse(2)), [s.download(f) for f in STATE]))
        s.close()
    monkeypatch.setenv("NIM_BATCH_FORM", "grid")
    batch = [make(c, precision=_abi.PRECISION_MIXED) for c in cases]
    recs = nimgpu.batch_step(batch, 2, fused=True)
    for s, r, (want_recs, want_fields) in zip(batch, recs, alone):
        assert records(r) == want_recs
        for f, w in zip(STATE, want_fields):
            assert np.array_equal(s.download(f), w), f
        s.close()
