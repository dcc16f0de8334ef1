#!/usr/bin/env python
"""Generate the benchmark-size step histories in tests/golden/ from the CPU
oracle (test infrastructure: the checker, never the product).

The 48x48x32 (c1) and 128x128x96 (c2) cylinders take minutes to hours per
run on the CPU, too long to repeat inside a test, so the oracle's history is
recorded once here and the GPU tests compare against it:

    python tests/golden/make_scale_golden.py c1 200 parallel   # ~25 min, 8 threads
    python tests/golden/make_scale_golden.py c2 20 parallel    # ~50 min
    python tests/golden/make_scale_golden.py c1 200 sequential # ~45 min, 1 thread

Each file holds, per step, the oracle's iteration count and the statistics
the reference prints (nse.f90:169-171, 2793-2794) as exact float reprs, and
at a few checkpoint steps a summary of every state field: the SHA-256 of
its bytes, sum, sum of squares, max |x| and a strided sample.  The inputs are
the seeded synthetic cases of nimgpu.config (same mesh builder, parameters,
noise seed), so the GPU side rebuilds them exactly.
"""
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "nim-conv22-shared_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import nimgpu  # noqa: E402
from nimgpu import _abi, config  # noqa: E402
import oracle as O  # noqa: E402

FIELDS = {"faces_u": _abi.FACES_U, "faces_v": _abi.FACES_V, "faces_w": _abi.FACES_W, "faces_p": _abi.FACES_P,
          "faces_T": _abi.FACES_T, "meshes_u": _abi.MESHES_U, "meshes_v": _abi.MESHES_V,
          "meshes_w": _abi.MESHES_W, "meshes_T": _abi.MESHES_T, "meshes_p": _abi.MESHES_P}
STATS = ("iters", "err_u", "err_v", "err_w", "err_p", "err_T", "dilatation", "dudt_max", "dTdt_max",
         "nu_outer", "nu_inner", "area_outer", "area_inner", "time")
NSAMPLE = 256


def field_size(mesh, f):
    return mesh.nface if f <= _abi.FACES_T else mesh.nmesh


def sample_index(n: int) -> np.ndarray:
    return np.linspace(0, n - 1, min(NSAMPLE, n)).astype(np.int64)


def summarize(v: np.ndarray) -> dict:
    """What the GPU test compares: exact hash, norms and a strided sample."""
    idx = sample_index(v.size)
    return {"sha256": hashlib.sha256(np.ascontiguousarray(v, dtype=np.float64).tobytes()).hexdigest(),
            "n": int(v.size), "sum": float(v.sum()), "sumsq": float(np.dot(v, v)),
            "max_abs": float(np.abs(v).max()), "mean": float(v.mean()),
            "samples": [float(x) for x in v[idx]]}


def checkpoints(steps: int):
    return sorted({1, min(steps, 10), steps})


def main():
    name, steps, sched = sys.argv[1], int(sys.argv[2]), sys.argv[3]
    schedule = {"parallel": O.PARALLEL, "sequential": O.SEQUENTIAL}[sched]
    threads = int(sys.argv[4]) if len(sys.argv) > 4 else (8 if schedule == O.PARALLEL else 1)
    case = config.CASES[name]
    mesh = nimgpu.Mesh(case.mesh_params())
    params = case.params()
    ref = O.Oracle(mesh, params, schedule=schedule, threads=threads)
    ref.init()
    nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, case.noise, case.seed)
    rec = {"case": name, "schedule": sched, "steps": steps, "cells": case.ncells,
           "per_step": {k: [] for k in STATS}, "fields": {}}
    t0 = time.time()
    for s in range(1, steps + 1):
        st, so = ref.step(1)
        if st != 0:
            raise SystemExit(f"oracle step {s}: status {st}")
        for k in STATS:
            rec["per_step"][k].append(getattr(so[0], k))
        if s in checkpoints(steps):
            rec["fields"][str(s)] = {fn: summarize(ref.get(f, field_size(mesh, f))) for fn, f in FIELDS.items()}
        print(f"step {s}: {so[0].iters} iterations, Nu_hot {so[0].nu_inner!r}, {time.time() - t0:.0f} s",
              flush=True)
    rec["oracle_seconds"] = time.time() - t0
    out = HERE / f"scale_{name}_{sched}_{steps}.json"
    out.write_text(json.dumps(rec, separators=(",", ":")) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
