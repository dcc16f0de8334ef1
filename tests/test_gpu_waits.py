"""Bounded device waits.  The TMA-staged sweeps wait on mbarriers for their
bulk copies; every such wait gives up after a bounded number of tries,
marks the step NIM_ERR_TIMEOUT and stops it instead of hanging the GPU.
nim_gpu_selftest_wait_timeout runs that wait on an mbarrier no copy will
complete (no fault, nothing in flight) and reports the status the device
recorded; afterwards the context must still step normally."""
import pytest

import nimgpu
from nimgpu import _abi, config

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_the_context_stays_usable():
    case = config.small_case(16, 6, 6)
    s = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params())
    s.initialize_nse()
    s.add_temperature_noise(case.noise, case.seed)
    assert s.lib.nim_gpu_selftest_wait_timeout(s._h, 1000) == _abi.NIM_ERR_TIMEOUT
    assert s.lib.nim_gpu_selftest_wait_timeout(s._h, 0) == _abi.NIM_ERR_BAD_ARG
    recs = s.solve_nse(2)
    assert all(r.status == _abi.NIM_OK and r.iters > 1 for r in recs)
    s.close()
