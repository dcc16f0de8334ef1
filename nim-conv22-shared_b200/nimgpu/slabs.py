"""z-slab decomposition of one enclosure over the C ABI (include/nim_gpu.h,
nim_slab_layout / nim_slab_halo / nim_gpu_create_slab / nim_slab_step).

The n_z cell planes split into contiguous slabs; a slab context holds its
own planes plus the two nearest planes of each neighbour slab (its halo).
nim_slab_step advances a group of slab contexts on one device with a halo
exchange after the velocity, pressure and temperature parts of every pass.
This module maps the reference-layout arrays of the whole mesh to and from
the slab contexts' structured layout, so a host can scatter a restart over
the slabs and gather their owned planes back.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .mesh import Mesh, temperature_noise


def slab_layout(n_z: int, nslab: int, s: int) -> tuple[int, int, int, int]:
    """(first plane held, one past the last held, first owned, one past the
    last owned) of slab s, global plane numbers."""
    out = (C.c_int32 * 4)()
    _abi.check(_abi.gpu_lib().nim_slab_layout(n_z, nslab, s, out), "nim_slab_layout")
    return tuple(out)


def slab_halo(n_theta: int, n_r: int, n_z: int, nslab: int, s: int, side: int):
    """(recv, send) element spans of slab s's exchange with its neighbour
    below (side 0) or above (side 1): four (offset, count) pairs each, for
    the cells and the r, theta and z faces of the slab context's arrays."""
    recv, send = (C.c_int64 * 8)(), (C.c_int64 * 8)()
    _abi.check(_abi.gpu_lib().nim_slab_halo(n_theta, n_r, n_z, nslab, s, side, recv, send), "nim_slab_halo")
    pairs = lambda a: [(a[2 * t], a[2 * t + 1]) for t in range(4)]
    return pairs(recv), pairs(send)


def slab_sizes(n_theta: int, n_r: int, held: int) -> tuple[int, int]:
    """(cells, faces) of a slab context holding `held` planes."""
    pl = n_theta * n_r
    return pl * held, n_theta * (n_r + 1) * held + pl * held + pl * (held + 1)


def structured_faces(mesh: Mesh) -> np.ndarray:
    """For every face of the whole mesh in the library's structured order
    (radial, theta, then axial blocks; cell c = i + n_theta*(j + n_r*k)),
    its 0-based reference face number (meshes_faces, link_mesh order)."""
    NT, NR, NZ = mesh.n_theta, mesh.n_r, mesh.n_z
    c = np.arange(mesh.nmesh, dtype=np.int64)
    i, k = c % NT, c // (NT * NR)
    offT = NT * (NR + 1) * NZ
    offZ = offT + NT * NR * NZ
    ip = np.where(i == NT - 1, 0, i + 1)
    sf = np.stack([c + NT * k, c + NT * k + NT, offT + c, offT + c - i + ip, offZ + c, offZ + c + NT * NR], axis=1)
    ref = np.full(mesh.nface, -1, dtype=np.int64)
    ref[sf.ravel()] = mesh.meshes_faces.astype(np.int64).ravel() - 1
    if (ref < 0).any():
        raise ValueError("mesh is not the structured O-grid")
    return ref


def slab_face_planes(mesh: Mesh, lo: int, hi: int):
    """For the faces of a slab context holding planes [lo, hi): the whole
    mesh's structured face index of each, and the plane that owns it (its
    cell plane for r and theta faces, the plane above for an axial face,
    n_z for the top wall)."""
    NT, NR, NZ = mesh.n_theta, mesh.n_r, mesh.n_z
    held, pl, rb = hi - lo, NT * NR, NT * (NR + 1)
    offT, offZ = rb * NZ, rb * NZ + pl * NZ
    r = np.arange(rb * held, dtype=np.int64) + rb * lo
    t = np.arange(pl * held, dtype=np.int64) + pl * lo
    z = np.arange(pl * (held + 1), dtype=np.int64) + pl * lo
    glob = np.concatenate([r, offT + t, offZ + z])
    plane = np.concatenate([r // rb, t // pl, z // pl])
    return glob, plane


class SlabGroup:
    """nslab z-slab contexts of one mesh on the current device, advanced
    together (nim_slab_step).  Without the CUDA library or a GPU the
    constructor raises."""

    def __init__(self, mesh: Mesh, params: _abi.Params, nslab: int):
        self.lib = _abi.gpu_lib()
        self.mesh, self.params, self.nslab = mesh, params, nslab
        self.layout = [slab_layout(mesh.n_z, nslab, s) for s in range(nslab)]
        self._ref = structured_faces(mesh)
        self._h = []
        try:
            for s in range(nslab):
                h = C.c_void_p()
                _abi.check(self.lib.nim_gpu_create_slab(C.byref(mesh.desc), C.byref(params), nslab, s, C.byref(h)),
                           "nim_gpu_create_slab")
                self._h.append(h)
        except Exception:
            self.close()
            raise

    # -- lifetime
    def close(self):
        for h in self._h:
            if h:
                self.lib.nim_gpu_destroy(h)
        self._h = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's call sites
    def initialize_nse(self):
        for h in self._h:
            _abi.check(self.lib.nim_gpu_init(h), "nim_gpu_init")

    def solve_nse(self, nsteps: int, raise_on_error: bool = True):
        """nsteps of the time loop over the group; returns the group's
        per-step records."""
        n = self.nslab
        handles = (C.c_void_p * n)(*[h.value for h in self._h])
        per = (_abi.StepStats * max(nsteps, 1))()
        done = C.c_int32()
        st = self.lib.nim_slab_step(n, handles, nsteps, per, C.byref(done))
        if raise_on_error:
            _abi.check(st, "nim_slab_step")
        return [per[k] for k in range(done.value)]

    def set_graph_iters(self, n: int):
        for h in self._h:
            _abi.check(self.lib.nim_gpu_set_graph_iters(h, n), "nim_gpu_set_graph_iters")

    # -- host copies in the slab's structured layout
    def _sizes(self, s: int):
        lo, hi = self.layout[s][:2]
        return slab_sizes(self.mesh.n_theta, self.mesh.n_r, hi - lo)

    def download(self, s: int, field: int) -> np.ndarray:
        nc, nf = self._sizes(s)
        out = np.empty(nf if field <= _abi.FACES_T else nc, dtype=np.float64)
        _abi.check(self.lib.nim_gpu_download(self._h[s], field, out.ctypes.data_as(C.POINTER(C.c_double)), out.size),
                   "nim_gpu_download")
        return out

    def upload(self, s: int, field: int, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64)
        _abi.check(self.lib.nim_gpu_upload(self._h[s], field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
                   "nim_gpu_upload")

    # -- whole-mesh arrays (reference layout) to and from the slabs
    def scatter(self, field: int, values: np.ndarray):
        """Upload the held part of a whole-mesh field to every slab."""
        pl = self.mesh.n_theta * self.mesh.n_r
        for s, (lo, hi, _, _) in enumerate(self.layout):
            if field <= _abi.FACES_T:
                glob, _ = slab_face_planes(self.mesh, lo, hi)
                self.upload(s, field, values[self._ref[glob]])
            else:
                self.upload(s, field, values[lo * pl:hi * pl])

    def gather(self, field: int) -> np.ndarray:
        """A whole-mesh field in the reference layout from the slabs' owned
        planes."""
        m = self.mesh
        pl = m.n_theta * m.n_r
        if field > _abi.FACES_T:
            out = np.empty(m.nmesh, dtype=np.float64)
            for s, (lo, _, olo, ohi) in enumerate(self.layout):
                out[olo * pl:ohi * pl] = self.download(s, field)[(olo - lo) * pl:(ohi - lo) * pl]
            return out
        out = np.full(m.nface, np.nan, dtype=np.float64)
        for s, (lo, hi, olo, ohi) in enumerate(self.layout):
            glob, plane = slab_face_planes(m, lo, hi)
            top = ohi + (1 if s == self.nslab - 1 else 0)
            keep = (plane >= olo) & (plane < top)
            out[self._ref[glob[keep]]] = self.download(s, field)[keep]
        return out

    def add_temperature_noise(self, amp: float, seed: int):
        """nimgpu.apply_temperature_noise for the group: the whole mesh's
        seeded noise added to every slab's held planes."""
        if amp == 0.0:
            return
        cells, faces = temperature_noise(self.mesh, amp, seed)
        pl = self.mesh.n_theta * self.mesh.n_r
        for s, (lo, hi, _, _) in enumerate(self.layout):
            glob, _ = slab_face_planes(self.mesh, lo, hi)
            self.upload(s, _abi.FACES_T, self.download(s, _abi.FACES_T) + faces[self._ref[glob]])
            for fld in (_abi.MESHES_T, _abi.MESHES_T_OLD, _abi.MESHES_TT):
                self.upload(s, fld, self.download(s, fld) + cells[lo * pl:hi * pl])
