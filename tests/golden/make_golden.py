#!/usr/bin/env python
"""Generate the golden fixtures in tests/golden/ from the CPU oracle.

The reference ships no tests, fixtures or outputs and cannot be built here
(no Fortran compiler), so these fixtures pin the oracle itself: any change
to its arithmetic shows up as a diff.  Re-run after a deliberate change:

    python tests/golden/make_golden.py
"""
import json
import sys
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
          "meshes_w": _abi.MESHES_W, "meshes_T": _abi.MESHES_T}
STATS = ("iters", "err_u", "err_v", "err_w", "err_p", "err_T", "dilatation", "dudt_max", "dTdt_max",
         "nu_outer", "nu_inner", "area_outer", "area_inner", "time")


def summary(get, mesh):
    out = {}
    for name, f in FIELDS.items():
        n = mesh.nface if f <= _abi.FACES_T else mesh.nmesh
        v = get(f, n)
        idx = np.linspace(0, n - 1, 16).astype(int)
        out[name] = {"sum": float(v.sum()), "abs_sum": float(np.abs(v).sum()), "max_abs": float(np.abs(v).max()),
                     "idx": idx.tolist(), "samples": v[idx].tolist()}
    return out


def run(name, mesh_params, params, steps, noise=None):
    mesh = nimgpu.Mesh(mesh_params)
    res = {"name": name, "steps": steps}
    for label, sched in (("sequential", O.SEQUENTIAL), ("parallel", O.PARALLEL)):
        o = O.Oracle(mesh, params, schedule=sched)
        o.init()
        if noise:
            nimgpu.apply_temperature_noise(o.get, o.set, mesh, *noise)
        st, recs = o.step(steps)
        assert st == 0
        res[label] = {"stats": [{k: getattr(r, k) for k in STATS} for r in recs],
                      "fields": summary(o.get, mesh)}
    return res


def main():
    cases = [
        run("reference_36x6x12", config.reference_mesh(), config.reference_params(), 3),
    ]
    sc = config.small_case(16, 6, 6)
    cases.append(run("tanh_16x6x6", sc.mesh_params(), sc.params(), 3, noise=(sc.noise, sc.seed)))
    # nim_formulation = 1 (nim.f90:17-157, nse.f90:330-828)
    cases.append(run("formulation1_16x6x6", sc.mesh_params(), sc.params(formulation=1), 3,
                     noise=(sc.noise, sc.seed)))
    (HERE / "oracle_golden.json").write_text(json.dumps(cases, indent=1))
    print("wrote", HERE / "oracle_golden.json")


if __name__ == "__main__":
    main()
