"""The device exp of the NIM coefficients (nim_gpu_selftest_exp, through the
C ABI) against the host libm's exp, bit for bit: 1e8 arguments dense in the
exponential branch's range |Pe| in [1e-2, 50] (nim.f90:190-194), plus the
full range and random bit patterns."""
import sys
from pathlib import Path

import numpy as np
import pytest

from nimgpu import _abi

sys.path.insert(0, str(Path(__file__).resolve().parent))
import _exp_harness as H  # noqa: E402

pytestmark = pytest.mark.gpu

CHUNK = 10_000_000


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    return H.build(tmp_path_factory.mktemp("exp"))


def device_exp(x: np.ndarray) -> np.ndarray:
    y = np.empty_like(x)
    st = _abi.gpu_lib().nim_gpu_selftest_exp(H.ptr(x), H.ptr(y), x.size)
    assert st == _abi.NIM_OK, _abi.strerror(st)
    return y


def same_bits(a: np.ndarray, b: np.ndarray) -> int:
    """Count of elements whose bits differ (NaN against NaN counts as equal)."""
    diff = a.view(np.uint64) != b.view(np.uint64)
    diff &= ~(np.isnan(a) & np.isnan(b))
    return int(diff.sum())


@pytest.mark.parametrize("kind,lo,hi,chunks", [
    (0, 1e-2, 50.0, 10),     # 1e8 arguments in the NIM exponential range
    (0, 1e-20, 745.0, 1),
    (0, 500.0, 745.0, 1),
    (1, 1.0, 2.0, 1),        # random bit patterns
])
def test_device_exp_equals_libm(harness, kind, lo, hi, chunks):
    bad = 0
    for c in range(chunks):
        x = H.args(harness, CHUNK, 7 + 1000 * c + kind, kind, lo, hi)
        bad += same_bits(device_exp(x), H.libm_exp(harness, x))
    assert bad == 0


def test_selftest_exp_checks_arguments():
    lib = _abi.gpu_lib()
    assert lib.nim_gpu_selftest_exp(None, None, 0) == _abi.NIM_OK
    assert lib.nim_gpu_selftest_exp(None, None, 5) == _abi.NIM_ERR_BAD_ARG
    assert lib.nim_gpu_selftest_exp(None, None, -1) == _abi.NIM_ERR_BAD_ARG
