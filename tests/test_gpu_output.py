"""Device-packed output sets (nim_gpu_output_begin / _wait) against the
per-field copies of nim_gpu_download: write_data's zone variables as
REAL(.,4) (postprocess.f90:92-103) and write_restart's arrays
(restart.f90:24-37), taken while the next step already runs."""
import numpy as np
import pytest
import torch

import nimgpu
from nimgpu import _abi, config

pytestmark = pytest.mark.gpu

PLOT = [_abi.MESHES_UT, _abi.MESHES_VT, _abi.MESHES_WT, _abi.MESHES_P, _abi.MESHES_TT, _abi.MESHES_DILA]
RESTART = [_abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
           _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T,
           _abi.MESHES_U_OLD, _abi.MESHES_V_OLD, _abi.MESHES_W_OLD, _abi.MESHES_T_OLD,
           _abi.MESHES_DILA_OLD]


def pinned_like(a: np.ndarray) -> np.ndarray:
    t = torch.empty(a.shape, dtype=torch.float32 if a.dtype == np.float32 else torch.float64).pin_memory()
    return t.numpy()


def solver(dims=(16, 6, 6), schedule=_abi.SCHEDULE_PARALLEL):
    case = config.small_case(*dims)
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(schedule=schedule))
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    return s


@pytest.mark.parametrize("schedule", [_abi.SCHEDULE_PARALLEL, _abi.SCHEDULE_REFERENCE])
def test_output_sets_match_downloads(schedule):
    s = solver(schedule=schedule)
    s.solve_nse(2)
    plot = pinned_like(s.output_array(_abi.OUTPUT_PLOT))
    rest = pinned_like(s.output_array(_abi.OUTPUT_RESTART))
    tp = s.output_begin(_abi.OUTPUT_PLOT, plot)
    tr = s.output_begin(_abi.OUTPUT_RESTART, rest)
    s.output_wait(tp)
    s.output_wait(tr)
    want_plot = np.stack([s.download(f).astype(np.float32) for f in PLOT])
    assert np.array_equal(plot, want_plot)
    want_rest = np.concatenate([s.download(f) for f in RESTART])
    assert np.array_equal(rest, want_rest)
    s.close()


def test_output_is_a_snapshot_while_the_loop_goes_on():
    s = solver((24, 8, 10))
    s.solve_nse(1)
    before = np.concatenate([s.download(f) for f in RESTART])
    rest = pinned_like(s.output_array(_abi.OUTPUT_RESTART))
    t = s.output_begin(_abi.OUTPUT_RESTART, rest)
    s.solve_nse(2)                 # queued behind the packing, overlaps the copy
    s.output_wait(t)
    assert np.array_equal(rest, before)
    after = np.concatenate([s.download(f) for f in RESTART])
    assert not np.array_equal(after, before)
    # the same set again: the new packing waits for the old copy, tickets differ
    t2 = s.output_begin(_abi.OUTPUT_RESTART, rest)
    assert t2 != t
    s.output_wait(t2)
    assert np.array_equal(rest, after)
    with pytest.raises(nimgpu.NimError) as e:
        s.output_wait(t)           # overtaken by t2
    assert e.value.status == _abi.NIM_ERR_STATE
    s.close()


def test_output_arguments():
    s = solver()
    lib = _abi.gpu_lib()
    assert lib.nim_gpu_output_bytes(s._h, 7) == _abi.NIM_ERR_BAD_ARG
    small = np.empty(3, dtype=np.float32)
    with pytest.raises(nimgpu.NimError) as e:
        s.output_begin(_abi.OUTPUT_PLOT, small)
    assert e.value.status == _abi.NIM_ERR_BAD_ARG
    s.close()
