"""Parity at the benchmark sizes over whole runs, against the oracle's
recorded histories (tests/golden/scale_*.json, made by
tests/golden/make_scale_golden.py: the oracle takes minutes to hours per
run on the CPU).

* the parallel order (the kernels' order) on the 48x48x32 cylinder for all
  200 steps of its run and on the 128x128x96 cylinder for 20 steps: the same
  iteration count and the same find_error maxima every step, the fields
  bit-identical to the oracle's at the recorded steps, the steady-state
  maxima exactly, and the Nusselt numbers to 1e-12 and the dilatation to
  1e-10 relative (the GPU sums them in another order);
* the reference's own Gauss-Seidel order (NIM_SCHEDULE_REFERENCE) on the
  48x48x32 cylinder against the sequential oracle: the same per-step
  history and bit-identical fields.

Every step runs to the reference tolerances (1e-6 for u, v, w, T; 5e-3 for
p), so these are the runs a user of the reference makes."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GOLDEN = Path(__file__).resolve().parent / "golden"
FIELDS = {"faces_u": _abi.FACES_U, "faces_v": _abi.FACES_V, "faces_w": _abi.FACES_W, "faces_p": _abi.FACES_P,
          "faces_T": _abi.FACES_T, "meshes_u": _abi.MESHES_U, "meshes_v": _abi.MESHES_V,
          "meshes_w": _abi.MESHES_W, "meshes_T": _abi.MESHES_T, "meshes_p": _abi.MESHES_P}
EXACT = ("iters", "err_u", "err_v", "err_w", "err_p", "err_T", "dudt_max", "dTdt_max", "time")
# sums the device forms in another order than the oracle: the wall integrals
# of find_Nu2 (a few thousand terms) to 1e-12; evaluate_D's root of a sum
# of one squared residual per cell (1.6 M at 128x128x96) to 1e-10
CLOSE = {"nu_outer": 1e-12, "nu_inner": 1e-12, "area_outer": 1e-12, "area_inner": 1e-12, "dilatation": 1e-10}


def load(name):
    path = GOLDEN / name
    return json.loads(path.read_text())


def sample_index(n, k):
    return np.linspace(0, n - 1, min(k, n)).astype(np.int64)


def check_fields(solver, want: dict, step: int):
    for name, f in FIELDS.items():
        w = want[name]
        a = solver.download(f)
        assert a.size == w["n"], name
        if hashlib.sha256(a.tobytes()).hexdigest() == w["sha256"]:
            continue
        s = np.asarray(w["samples"])
        got = a[sample_index(a.size, len(s))]
        err = np.abs(got - s).max() / max(w["max_abs"], 1e-300)
        pytest.fail(f"step {step}: {name} differs from the oracle's bits (sampled max rel. error {err:.3e})")


def run_and_compare(golden: dict, schedule: int):
    case = config.CASES[golden["case"]]
    steps = golden["steps"]
    solver = nimgpu.NimSolver(nimgpu.Mesh(case.mesh_params()), case.params(schedule=schedule))
    solver.initialize_nse()
    solver.add_temperature_noise(case.noise, case.seed)
    per = golden["per_step"]
    for s in range(1, steps + 1):
        r = solver.solve_nse(1)[0]
        assert r.status == _abi.NIM_OK, (s, _abi.strerror(r.status))
        for k in EXACT:
            assert getattr(r, k) == per[k][s - 1], (s, k, getattr(r, k), per[k][s - 1])
        for k, rtol in CLOSE.items():
            want = per[k][s - 1]
            assert abs(getattr(r, k) - want) <= rtol * abs(want) + 1e-300, (s, k, getattr(r, k), want)
        if str(s) in golden["fields"]:
            check_fields(solver, golden["fields"][str(s)], s)
    solver.close()


@pytest.mark.parametrize("name", ["scale_c1_parallel_200.json", "scale_c2_parallel_20.json"])
def test_benchmark_runs_match_parallel_oracle(name):
    run_and_compare(load(name), _abi.SCHEDULE_PARALLEL)


def test_reference_order_matches_sequential_oracle():
    run_and_compare(load("scale_c1_sequential_200.json"), _abi.SCHEDULE_REFERENCE)
