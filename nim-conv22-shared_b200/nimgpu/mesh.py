"""Host mesh: numpy arrays in the reference layout plus the nim_mesh_desc
that points at them (include/nim_gpu.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi


class Mesh:
    """Arrays of create_hollow + prepare_mesh + fill_global_arrays for one
    structured O-grid, built by libnim_host.so (include/nim_mesh.h).

    Index arrays are 1-based and column-major like the Fortran globals:
    meshes_faces has shape (nmesh, 6) in C order == (6, NMESH) column-major.
    """

    def __init__(self, mp: _abi.MeshParams):
        lib = _abi.host_lib()
        nn, nm, nf, nb = (C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32())
        st = lib.nim_mesh_sizes(C.byref(mp), C.byref(nn), C.byref(nm), C.byref(nf), C.byref(nb))
        if st != 0:
            raise _abi.NimError(st, "nim_mesh_sizes", "bad mesh parameters")
        self.params = mp
        self.n_theta, self.n_r, self.n_z = mp.n_theta, mp.n_r, mp.n_z
        self.nnode, self.nmesh, self.nface, self.nbcface = nn.value, nm.value, nf.value, nb.value
        self.node_xyz = np.zeros((self.nnode, 3), dtype=np.float64)
        self.meshes_nodes = np.zeros((self.nmesh, 8), dtype=np.int32)
        self.meshes_faces = np.zeros((self.nmesh, 6), dtype=np.int32)
        self.meshes_neighbors = np.zeros((self.nmesh, 6), dtype=np.int32)
        self.faces_bc = np.zeros(self.nface, dtype=np.int32)
        self.bcs_faces = np.zeros(self.nbcface, dtype=np.int32)
        self.bcs_faces_id = np.zeros(self.nbcface, dtype=np.int32)
        self.bcs_faces_position = np.zeros(self.nbcface, dtype=np.int32)
        self.bcs_faces_mesh_num = np.zeros(self.nbcface, dtype=np.int32)
        st = lib.nim_mesh_build(
            C.byref(mp), _dp(self.node_xyz), _ip(self.meshes_nodes), _ip(self.meshes_faces),
            _ip(self.meshes_neighbors), _ip(self.faces_bc), _ip(self.bcs_faces),
            _ip(self.bcs_faces_id), _ip(self.bcs_faces_position), _ip(self.bcs_faces_mesh_num))
        if st != 0:
            raise _abi.NimError(st, "nim_mesh_build")
        self.desc = self.make_desc()

    def make_desc(self) -> _abi.MeshDesc:
        d = _abi.MeshDesc()
        d.n_theta, d.n_r, d.n_z = self.n_theta, self.n_r, self.n_z
        d.nnode, d.nmesh, d.nface, d.nbcface = self.nnode, self.nmesh, self.nface, self.nbcface
        d.node_xyz = _dp(self.node_xyz)
        d.meshes_nodes = _ip(self.meshes_nodes)
        d.meshes_faces = _ip(self.meshes_faces)
        d.meshes_neighbors = _ip(self.meshes_neighbors)
        d.faces_bc = _ip(self.faces_bc)
        d.bcs_faces = _ip(self.bcs_faces)
        d.bcs_faces_id = _ip(self.bcs_faces_id)
        d.bcs_faces_position = _ip(self.bcs_faces_position)
        d.bcs_faces_mesh_num = _ip(self.bcs_faces_mesh_num)
        return d

    @property
    def interior_faces(self) -> np.ndarray:
        """Boolean mask of faces with BC id 1 (interior)."""
        return self.faces_bc == 1


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def temperature_noise(mesh: Mesh, amp: float, seed: int):
    """Seeded U(-amp, amp) perturbation of the initial temperature: one value
    per cell and one per face (boundary faces keep their Dirichlet values).
    Returns (cell_noise[nmesh], face_noise[nface])."""
    rng = np.random.default_rng(seed)
    cells = rng.uniform(-amp, amp, size=mesh.nmesh)
    faces = rng.uniform(-amp, amp, size=mesh.nface)
    faces[~mesh.interior_faces] = 0.0
    return cells, faces


def apply_temperature_noise(get, set_, mesh: Mesh, amp: float, seed: int):
    """Add the seeded noise to an initialised solver through its
    download/upload pair (get(field, n) -> array, set_(field, array))."""
    if amp == 0.0:
        return
    cells, faces = temperature_noise(mesh, amp, seed)
    fT = get(_abi.FACES_T, mesh.nface) + faces
    set_(_abi.FACES_T, fT)
    for fld in (_abi.MESHES_T, _abi.MESHES_T_OLD, _abi.MESHES_TT):
        set_(fld, get(fld, mesh.nmesh) + cells)
