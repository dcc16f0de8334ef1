"""The temperature's NIM coefficients of one direction on the device
(nim_gpu_selftest_nim_coef, through the C ABI): the float form of the FP32
phase of the mixed path against the FP64 form of the FP64 path
(nim.f90:334-464), and the FP64 form against the exact functions.

The float form evaluates all six coefficients from one Bernoulli series for
|2u/k| <= 2 and from the exponential form above, so it carries no
cancellation at small cell Reynolds numbers (the FP64 formulas in float lose
most of their digits just above |2u/k| = v_limit).  Bound: 2e-6 relative,
with coefficients 3 and 4 (u/(k(e^-x - 1)), u/(k(1 - e^x))) measured against
the larger of the two, since one of them is exponentially small for large
|x| and float rounds x itself."""
import ctypes as C

import numpy as np
import pytest

from nimgpu import _abi

pytestmark = pytest.mark.gpu

V_LIMIT = 1e-2


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def device_coef(u: np.ndarray, k: np.ndarray, precision: int) -> np.ndarray:
    u = np.ascontiguousarray(u, dtype=np.float64)
    k = np.ascontiguousarray(k, dtype=np.float64)
    A = np.empty(6 * u.size)
    st = _abi.gpu_lib().nim_gpu_selftest_nim_coef(ptr(u), ptr(k), u.size, precision, V_LIMIT, ptr(A))
    assert st == _abi.NIM_OK, _abi.strerror(st)
    return A.reshape(-1, 6).T


def exact(u: np.ndarray, k: np.ndarray) -> np.ndarray:
    """The coefficients in double through expm1 (no cancellation), for
    |2u/k| >= 0.05."""
    x = 2 * u / k
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        em, emn = np.expm1(x), np.expm1(-x)
        A4 = np.where(x > 0, (-k + u * (emn + 2) / (-emn)) / (u * u), (-k + u * (em + 2) / em) / (u * u))
        A5 = np.where(x > 0, 1 / (-emn) - 1 / x, (em + 1) / em - 1 / x)
        return np.array([2 / (k * emn) + 1 / u, 2 / (k * em) - 1 / u, u / (k * emn), -u / (k * em), A4, A5])


def cases():
    x = np.geomspace(1e-7, 1e3, 200_001)
    x = np.concatenate([x, -x, [0.0, 2.0, -2.0, V_LIMIT, -V_LIMIT]])
    out = []
    for kk in (1e-3, 0.7, 50.0):
        out.append((x * kk / 2, np.full_like(x, kk)))
    return out


def rel_err(got, want):
    err = np.abs(got - want)
    scale = np.abs(want).copy()
    pair = np.maximum(np.abs(want[2]), np.abs(want[3]))
    scale[2], scale[3] = pair, pair
    return err / np.maximum(scale, 1e-300)


@pytest.mark.parametrize("case", range(3))
def test_float_form_tracks_fp64_form(case):
    u, k = cases()[case]
    a64 = device_coef(u, k, _abi.PRECISION_FP64)
    a32 = device_coef(u, k, _abi.PRECISION_MIXED)
    assert np.isfinite(a64).all() and np.isfinite(a32).all()
    # float's own range: the exponentially small member of the 3/4 pair
    # underflows in float beyond |x| ~ 87 (checked against its partner)
    e = rel_err(a32, a64)
    assert e.max() <= 2e-6, (e.max(axis=1), np.unravel_index(e.argmax(), e.shape))


def test_fp64_form_matches_exact_functions():
    for u, k in cases():
        x = 2 * u / k
        sel = np.abs(x) >= 0.05
        a64 = device_coef(u[sel], k[sel], _abi.PRECISION_FP64)
        e = rel_err(a64, exact(u[sel], k[sel]))
        assert e.max() <= 1e-9, e.max(axis=1)


def test_zero_velocity_gives_the_series_limits():
    k = np.array([0.25, 2.0])
    for prec in (_abi.PRECISION_FP64, _abi.PRECISION_MIXED):
        A = device_coef(np.zeros(2), k, prec)
        want = np.array([-1 / k, -1 / k, [-0.5, -0.5], [-0.5, -0.5], 1 / (3 * k), [0.5, 0.5]])
        np.testing.assert_allclose(A, want, rtol=1e-7)


def test_selftest_nim_coef_checks_arguments():
    lib = _abi.gpu_lib()
    assert lib.nim_gpu_selftest_nim_coef(None, None, 0, _abi.PRECISION_FP64, V_LIMIT, None) == _abi.NIM_OK
    assert lib.nim_gpu_selftest_nim_coef(None, None, 3, _abi.PRECISION_FP64, V_LIMIT, None) == _abi.NIM_ERR_BAD_ARG
    one = np.ones(1)
    assert lib.nim_gpu_selftest_nim_coef(ptr(one), ptr(one), 1, 7, V_LIMIT, ptr(np.ones(6))) == _abi.NIM_ERR_BAD_ARG
