"""Parity at the benchmark sizes: the GPU against the oracle's parallel
order (the kernels' order; multithreaded, thread-count independent) on the
48x48x32 and 128x128x96 cylinders of the benchmark geometry, whole steps to
the reference tolerances.  Same iteration count per step; fields and Nusselt
numbers to 1e-9 (CUDA's and glibc's exp differ in the last bit, amplified by
the exponential form of the NIM coefficients near |Pe| = v_limit)."""
import os

import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config
import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

STATE = [
    _abi.FACES_U, _abi.FACES_V, _abi.FACES_W, _abi.FACES_P, _abi.FACES_T,
    _abi.MESHES_U, _abi.MESHES_V, _abi.MESHES_W, _abi.MESHES_T, _abi.MESHES_P,
]


@pytest.mark.parametrize("name,steps", [("c1", 3), ("c2", 1)])
def test_benchmark_sizes_match_parallel_oracle(name, steps):
    case = config.CASES[name]
    mesh = nimgpu.Mesh(case.mesh_params())
    gpu = nimgpu.NimSolver(mesh, case.params())
    gpu.initialize_nse()
    gpu.add_temperature_noise(case.noise, case.seed)
    ref = O.Oracle(mesh, case.params(), schedule=O.PARALLEL, threads=os.cpu_count() or 1)
    ref.init()
    nimgpu.apply_temperature_noise(ref.get, ref.set, mesh, case.noise, case.seed)
    sg = gpu.solve_nse(steps)
    st, so = ref.step(steps)
    assert st == 0
    assert [a.iters for a in sg] == [b.iters for b in so]
    for a, b in zip(sg, so):
        assert abs(a.nu_inner - b.nu_inner) <= 1e-9 * abs(b.nu_inner)
        assert abs(a.nu_outer - b.nu_outer) <= 1e-9 * abs(b.nu_outer) + 1e-14
        assert abs(a.dilatation - b.dilatation) <= 1e-8 * abs(b.dilatation)
    for f in STATE:
        a = gpu.download(f)
        b = ref.get(f, a.size)
        if f == _abi.FACES_P:
            a, b = a - a.mean(), b - b.mean()
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), f
    gpu.close()
