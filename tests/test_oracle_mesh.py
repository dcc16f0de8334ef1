"""The oracle's own mesh (create_hollow, deform_nodes and
fill_global_geometry followed loop by loop) against the library's
closed-form host mesh builder: the same arrays to the bit, for the
reference geometry and the benchmark geometry, so the CPU reference arm can
build its input without the product libraries."""
import numpy as np
import pytest

import nimgpu
from nimgpu import _abi, config
import oracle as O

ARRAYS = ("node_xyz", "meshes_nodes", "meshes_faces", "meshes_neighbors", "faces_bc", "bcs_faces",
          "bcs_faces_id", "bcs_faces_position", "bcs_faces_mesh_num")


@pytest.mark.parametrize("mp", [
    config.reference_mesh(),
    config.reference_mesh(n_theta=12, n_r=5, n_z=4),
    config.CASES["c1"].mesh_params(),
    config.small_case(15, 10, 9).mesh_params(),
    config.reference_mesh(n_theta=24, n_r=6, n_z=5, cluster=_abi.CLUSTER_NONE, hexagon=0),
])
def test_oracle_mesh_equals_library_mesh(mp):
    a, b = O.OracleMesh(mp), nimgpu.Mesh(mp)
    for name in ARRAYS:
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert (a.nnode, a.nmesh, a.nface, a.nbcface) == (b.nnode, b.nmesh, b.nface, b.nbcface)


def test_oracle_noise_equals_library_noise():
    case = config.small_case(12, 6, 6)
    mp = case.mesh_params()
    a, b = O.temperature_noise(O.OracleMesh(mp), 1e-6, 7), nimgpu.temperature_noise(nimgpu.Mesh(mp), 1e-6, 7)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
