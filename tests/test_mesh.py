"""Host mesh builder: the arrays of create_hollow + link_mesh +
fill_global_arrays for the structured O-grid."""
import numpy as np
import pytest

import nimgpu
from nimgpu import config

MATH_PI = 3.14159265359


@pytest.fixture(scope="module")
def ref():
    return nimgpu.Mesh(config.reference_mesh())


def test_sizes_follow_parameters_f90(ref):
    n1, n2, n3 = 36, 6, 12
    assert ref.nmesh == n1 * n2 * n3
    assert ref.nface == 3 * n1 * n2 * n3 + n1 * n3 + n1 * n2          # parameters.f90:117
    assert ref.nnode == n1 * (n2 + 1) * (n3 + 1)                      # parameters.f90:119
    assert ref.nbcface == 2 * n1 * n2 + 2 * n1 * n3


def test_faces_are_numbered_in_bc_order(ref):
    n1, n2, n3 = 36, 6, 12
    nint = ref.nface - 2 * n1 * n2 - 2 * n1 * n3
    assert np.all(ref.faces_bc[:nint] == 1)
    ids = ref.faces_bc[nint:]
    assert np.all(ids[: n1 * n2] == 2) and np.all(ids[n1 * n2: 2 * n1 * n2] == 3)
    assert np.all(ids[2 * n1 * n2: 2 * n1 * n2 + n1 * n3] == 4) and np.all(ids[2 * n1 * n2 + n1 * n3:] == 5)
    assert np.array_equal(ref.bcs_faces, np.arange(nint + 1, ref.nface + 1))
    # positions: bottom 5, top 6, inner 1, outer 2 (fill_global_arrays)
    pos = ref.bcs_faces_position
    assert set(pos[: n1 * n2]) == {5} and set(pos[n1 * n2: 2 * n1 * n2]) == {6}
    assert set(pos[2 * n1 * n2: 2 * n1 * n2 + n1 * n3]) == {1} and set(pos[2 * n1 * n2 + n1 * n3:]) == {2}
    for b in range(ref.nbcface):
        m = ref.bcs_faces_mesh_num[b] - 1
        assert ref.meshes_faces[m, pos[b] - 1] == ref.bcs_faces[b]
        assert ref.meshes_neighbors[m, pos[b] - 1] == 0


def test_every_face_has_one_or_two_cells(ref):
    count = np.bincount(ref.meshes_faces.ravel(), minlength=ref.nface + 1)[1:]
    assert np.all(count[ref.faces_bc == 1] == 2)
    assert np.all(count[ref.faces_bc != 1] == 1)


def test_neighbours_are_symmetric(ref):
    opp = [1, 0, 3, 2, 5, 4]
    for c in range(ref.nmesh):
        for p in range(6):
            nb = ref.meshes_neighbors[c, p]
            if nb:
                assert ref.meshes_neighbors[nb - 1, opp[p]] == c + 1
                assert ref.meshes_faces[nb - 1, opp[p]] == ref.meshes_faces[c, p]


def _centre(mesh, c, nodes):
    return mesh.node_xyz[mesh.meshes_nodes[c, nodes] - 1].mean(axis=0)


def test_local_axes_are_r_theta_z(ref):
    """link_mesh's frame: xi1 outward (face 2 outside face 1), xi2
    counter-clockwise (face 4 ahead of face 3), xi3 up (face 6 above 5).
    Faces via their corner nodes (create_mesh.f90:326-349 drawing)."""
    f1, f2 = [0, 3, 4, 7], [1, 2, 5, 6]
    f3, f4 = [0, 1, 4, 5], [2, 3, 6, 7]
    f5, f6 = [0, 1, 2, 3], [4, 5, 6, 7]
    for c in range(ref.nmesh):
        a, b = _centre(ref, c, f1), _centre(ref, c, f2)
        assert np.hypot(*b[:2]) > np.hypot(*a[:2])
        a, b = _centre(ref, c, f3), _centre(ref, c, f4)
        assert a[0] * b[1] - a[1] * b[0] > 0
        a, b = _centre(ref, c, f5), _centre(ref, c, f6)
        assert b[2] > a[2]


def test_hexagon_and_outer_wall(ref):
    n1, n2, n3 = 36, 6, 12
    xyz = ref.node_xyz.reshape(n3 + 1, n2 + 1, n1, 3)
    R_i = MATH_PI / 3
    inner = np.hypot(xyz[:, 0, :, 0], xyz[:, 0, :, 1])
    outer = np.hypot(xyz[:, -1, :, 0], xyz[:, -1, :, 1])
    assert np.allclose(outer, 2.0, rtol=0, atol=1e-12)
    assert inner.max() <= R_i * (1 + 1e-12)
    # the 6 corners sit on multiples of 60 degrees and keep their radius
    corners = inner[:, ::6]
    assert np.allclose(corners, R_i, rtol=0, atol=1e-12)
    # edge points lie on the straight edges: apothem = R_i*cos(30 deg)
    assert inner.min() >= R_i * np.cos(np.pi / 6) * (1 - 1e-9)
    z = xyz[..., 2]
    assert np.allclose(z[0], 0.0) and np.allclose(z[-1], 2.0)


def test_tanh_case_geometry():
    case = config.small_case(24, 8, 6)
    m = nimgpu.Mesh(case.mesh_params())
    xyz = m.node_xyz.reshape(7, 9, 24, 3)
    r = np.hypot(xyz[0, :, 12, 0], xyz[0, :, 12, 1])  # ray at 180 degrees (a hexagon corner)
    assert r[0] == pytest.approx(0.2, abs=1e-12) and r[-1] == pytest.approx(0.5, abs=1e-12)
    d = np.diff(r)
    assert d[0] < d[4] and d[-1] < d[4]   # clustered toward both walls


def test_bad_sizes_are_refused():
    with pytest.raises(nimgpu.NimError):
        nimgpu.Mesh(config.reference_mesh(n_theta=4))
