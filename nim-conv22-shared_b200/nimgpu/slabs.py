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
import math

import numpy as np

from . import _abi
from .mesh import Mesh, temperature_noise


def slab_layout(n_z: int, nslab: int, s: int, lib=None) -> tuple[int, int, int, int]:
    """(first plane held, one past the last held, first owned, one past the
    last owned) of slab s, global plane numbers."""
    out = (C.c_int32 * 4)()
    _abi.check((lib or _abi.gpu_lib()).nim_slab_layout(n_z, nslab, s, out), "nim_slab_layout")
    return tuple(out)


def slab_halo(n_theta: int, n_r: int, n_z: int, nslab: int, s: int, side: int, lib=None):
    """(recv, send) element spans of slab s's exchange with its neighbour
    below (side 0) or above (side 1): four (offset, count) pairs each, for
    the cells and the r, theta and z faces of the slab context's arrays."""
    recv, send = (C.c_int64 * 8)(), (C.c_int64 * 8)()
    _abi.check((lib or _abi.gpu_lib()).nim_slab_halo(n_theta, n_r, n_z, nslab, s, side, recv, send),
               "nim_slab_halo")
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


class _Slabs:
    """Slab contexts of one mesh held by this process (slab numbers in
    `slabs`), with the host copies between the whole mesh's reference
    layout and the slabs' structured layout."""

    def __init__(self, mesh: Mesh, params: _abi.Params, nslab: int, slabs, lib=None):
        self.lib = lib or _abi.gpu_lib()
        self.mesh, self.params, self.nslab = mesh, params, nslab
        self.slabs = list(slabs)
        self.layout = {s: slab_layout(mesh.n_z, nslab, s, self.lib) for s in self.slabs}
        self._ref = structured_faces(mesh)
        self._h = []
        try:
            for s in self.slabs:
                h = C.c_void_p()
                _abi.check(self.lib.nim_gpu_create_slab(C.byref(mesh.desc), C.byref(params), nslab, s, C.byref(h)),
                           "nim_gpu_create_slab")
                self._h.append(h)
        except Exception:
            self.close()
            raise

    def _handle(self, s: int):
        return self._h[self.slabs.index(s)]

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

    def initialize_nse(self):
        for h in self._h:
            _abi.check(self.lib.nim_gpu_init(h), "nim_gpu_init")

    def set_graph_iters(self, n: int):
        for h in self._h:
            _abi.check(self.lib.nim_gpu_set_graph_iters(h, n), "nim_gpu_set_graph_iters")

    # -- host copies in a slab's structured layout
    def _sizes(self, s: int):
        lo, hi = self.layout[s][:2]
        return slab_sizes(self.mesh.n_theta, self.mesh.n_r, hi - lo)

    def field_size(self, s: int, field: int) -> int:
        """Doubles of `field` in slab s's context (its held planes)."""
        nc, nf = self._sizes(s)
        return nf if field <= _abi.FACES_T else nc

    def download(self, s: int, field: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.field_size(s, field), dtype=np.float64)
        _abi.check(self.lib.nim_gpu_download(self._handle(s), field, out.ctypes.data_as(C.POINTER(C.c_double)),
                                             out.size), "nim_gpu_download")
        return out

    def upload(self, s: int, field: int, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64)
        _abi.check(self.lib.nim_gpu_upload(self._handle(s), field, a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
                   "nim_gpu_upload")

    # -- whole-mesh arrays (reference layout) to and from the slabs
    def scatter(self, field: int, values: np.ndarray):
        """Upload the held part of a whole-mesh field to every slab here."""
        pl = self.mesh.n_theta * self.mesh.n_r
        for s in self.slabs:
            lo, hi = self.layout[s][:2]
            if field <= _abi.FACES_T:
                glob, _ = slab_face_planes(self.mesh, lo, hi)
                self.upload(s, field, values[self._ref[glob]])
            else:
                self.upload(s, field, values[lo * pl:hi * pl])

    def gather(self, field: int) -> np.ndarray:
        """A whole-mesh field in the reference layout from the owned planes
        of the slabs here (NaN where another process's slab owns it)."""
        m = self.mesh
        pl = m.n_theta * m.n_r
        if field > _abi.FACES_T:
            out = np.full(m.nmesh, np.nan, dtype=np.float64)
            for s in self.slabs:
                lo, _, olo, ohi = self.layout[s]
                out[olo * pl:ohi * pl] = self.download(s, field)[(olo - lo) * pl:(ohi - lo) * pl]
            return out
        out = np.full(m.nface, np.nan, dtype=np.float64)
        for s in self.slabs:
            lo, hi, olo, ohi = self.layout[s]
            glob, plane = slab_face_planes(m, lo, hi)
            top = ohi + (1 if s == self.nslab - 1 else 0)
            keep = (plane >= olo) & (plane < top)
            out[self._ref[glob[keep]]] = self.download(s, field)[keep]
        return out

    def add_temperature_noise(self, amp: float, seed: int):
        """nimgpu.apply_temperature_noise for slabs: the whole mesh's seeded
        noise added to every slab's held planes."""
        if amp == 0.0:
            return
        cells, faces = temperature_noise(self.mesh, amp, seed)
        pl = self.mesh.n_theta * self.mesh.n_r
        for s in self.slabs:
            lo, hi = self.layout[s][:2]
            glob, _ = slab_face_planes(self.mesh, lo, hi)
            self.upload(s, _abi.FACES_T, self.download(s, _abi.FACES_T) + faces[self._ref[glob]])
            for fld in (_abi.MESHES_T, _abi.MESHES_T_OLD, _abi.MESHES_TT):
                self.upload(s, fld, self.download(s, fld) + cells[lo * pl:hi * pl])


class SlabGroup(_Slabs):
    """All nslab z-slab contexts of one mesh on the current device, advanced
    together (nim_slab_step).  Without the CUDA library or a GPU the
    constructor raises."""

    def __init__(self, mesh: Mesh, params: _abi.Params, nslab: int):
        super().__init__(mesh, params, nslab, range(nslab))

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


# exchange sets of nim_slab_arrays
HALO_VELOCITY, HALO_PRESSURE, HALO_TEMPERATURE, HALO_STATE = 1, 2, 4, 8


def exchange_packed(send: dict, recv: dict, rank: int, group=None):
    """One halo exchange over torch.distributed: per side with a neighbour
    (0 below, 1 above), the packed payload send[side] goes to that
    neighbour and its payload lands in recv[side] (NCCL for device tensors,
    ordered on the current CUDA stream; gloo for host tensors)."""
    import torch.distributed as dist
    ops = []
    for side in sorted(send):
        peer = rank - 1 if side == 0 else rank + 1
        ops.append(dist.P2POp(dist.isend, send[side], peer, group))
        ops.append(dist.P2POp(dist.irecv, recv[side], peer, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def _device_tensor(ptr: int, n: int, typestr: str, device):
    """A torch tensor over n elements of device memory the library owns."""
    import torch

    class _View:
        pass

    v = _View()
    v.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                  "strides": None, "version": 3}
    return torch.as_tensor(v, device=device)


class SlabRank(_Slabs):
    """This process's slab of a mesh split over the ranks of a
    torch.distributed group, one GPU per rank (rank r holds slab r, bottom to
    top).  solve_nse drives the pieces of nim_slab_step: each part of a pass
    on the context's stream, then the halo exchange over the group (packed
    by nim_slab_pack, one message per neighbour: exchange_packed), the
    maxima's all-reduce before every pass end, and the
    step-end sums reduced over the group.

    Every rank takes the same collective steps in the same order: the stop
    decision of each pass comes from maxima all-reduced over the group, so
    every rank reads the same `done` and leaves the loop after the same
    pass.  `lib` and `device` exist for testing the control flow on the CPU
    (a stand-in for the library's slab entry points and CPU tensors over a
    gloo group); by default the CUDA library and the current GPU."""

    def __init__(self, mesh: Mesh, params: _abi.Params, group=None, lib=None, device=None):
        import torch
        import torch.distributed as dist
        self._dist, self._group = dist, group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        super().__init__(mesh, params, self.world, [self.rank], lib=lib)
        h = self._h[0]
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.stream = (torch.cuda.ExternalStream(int(self.lib.nim_gpu_stream(h)), device=self.device)
                       if self.device.type == "cuda" else None)
        self.plans = {}
        if self.rank > 0:
            self.plans[0] = slab_halo(mesh.n_theta, mesh.n_r, mesh.n_z, self.world, self.rank, 0, self.lib)
        if self.rank < self.world - 1:
            self.plans[1] = slab_halo(mesh.n_theta, mesh.n_r, mesh.n_z, self.world, self.rank, 1, self.lib)
        # packed send / receive buffers per exchange set and side
        self._send, self._recv = {}, {}
        for st in (HALO_VELOCITY, HALO_PRESSURE, HALO_TEMPERATURE, HALO_STATE):
            self._send[st], self._recv[st] = {}, {}
            for side in self.plans:
                n = int(self.lib.nim_slab_pack_doubles(h, st, side))
                if n < 0:
                    _abi.check(n, "nim_slab_pack_doubles")
                self._send[st][side] = torch.empty(n, dtype=torch.float64, device=self.device)
                self._recv[st][side] = torch.empty(n, dtype=torch.float64, device=self.device)
        slots = C.c_void_p()
        _abi.check(self.lib.nim_slab_maxima(h, C.byref(slots)), "nim_slab_maxima")
        self._maxima = (_device_tensor(slots.value, 24, "<i8", self.device) if self.device.type == "cuda"
                        else torch.frombuffer((C.c_int64 * 24).from_address(slots.value), dtype=torch.int64))
        self._step, self._time = 1, params.DT

    def _on_stream(self):
        """The context's stream as torch's current stream (CUDA), so the
        collectives are ordered with the library's kernels."""
        import contextlib
        import torch
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def close(self):
        self._send, self._recv, self._maxima = {}, {}, None
        super().close()

    def _exchange(self, what: int):
        """Pack each side on the context's stream, one message per
        neighbour, unpack after it lands."""
        import torch
        if self.world == 1:
            return
        h, send, recv = self._h[0], self._send[what], self._recv[what]
        for side, buf in send.items():
            _abi.check(self.lib.nim_slab_pack(h, what, side, C.c_void_p(buf.data_ptr())), "nim_slab_pack")
        with self._on_stream():
            exchange_packed(send, recv, self.rank, self._group)
        for side, buf in recv.items():
            _abi.check(self.lib.nim_slab_unpack(h, what, side, C.c_void_p(buf.data_ptr())), "nim_slab_unpack")

    def _merge(self):
        with self._on_stream():
            self._dist.all_reduce(self._maxima, op=self._dist.ReduceOp.MAX, group=self._group)

    def _reduce(self, values, op):
        import torch
        t = torch.tensor(values, dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=op, group=self._group)
        return t.tolist()

    def initialize_nse(self):
        super().initialize_nse()
        self._step, self._time = 1, self.params.DT

    def solve_nse(self, nsteps: int, passes_per_check: int = 4, raise_on_error: bool = True):
        """nsteps of the time loop; every rank returns the same records."""
        lib, h, R = self.lib, self._h[0], self._dist.ReduceOp
        recs = []
        self._exchange(HALO_STATE)
        for _ in range(nsteps):
            _abi.check(lib.nim_gpu_begin_step(h), "nim_gpu_begin_step")
            state, err = (C.c_int32 * 3)(), (C.c_double * 5)()
            while True:
                for _ in range(passes_per_check):
                    for part, what in ((0, HALO_VELOCITY), (1, HALO_PRESSURE), (2, HALO_TEMPERATURE)):
                        _abi.check(lib.nim_slab_part(h, part), "nim_slab_part")
                        self._exchange(what)
                    self._merge()
                    _abi.check(lib.nim_slab_part(h, 3), "nim_slab_part")
                _abi.check(lib.nim_slab_loop_state(h, state, err), "nim_slab_loop_state")
                if state[0]:
                    break
            a3 = (C.c_double * 3)()
            _abi.check(lib.nim_slab_after_loop(h, a3), "nim_slab_after_loop")
            (dsum,) = self._reduce([a3[0]], R.SUM)
            dudt, dTdt = self._reduce([a3[1], a3[2]], R.MAX)
            r = _abi.StepStats()
            r.step, r.iters, r.status = self._step, state[1], state[2]
            r.err_u, r.err_v, r.err_w, r.err_p, r.err_T = err
            r.dilatation = math.sqrt(dsum / self.mesh.nmesh)
            r.dudt_max, r.dTdt_max = dudt, dTdt
            p = self.params
            if r.status != _abi.NIM_OK or (p.check_steady and dudt < p.dudt_epsilon and dTdt < p.dudt_epsilon):
                r.steady = int(r.status == _abi.NIM_OK)
                recs.append(r)
                break
            s4 = (C.c_double * 4)()
            _abi.check(lib.nim_slab_end_step(h, s4), "nim_slab_end_step")
            sum1, sumA1, sum2, sumA2 = self._reduce(list(s4), R.SUM)
            self._time = self._time + 2 * p.DT
            r.nu_outer = -(sum1 / sumA1 * p.R_o)
            r.nu_inner = -(sum2 / sumA2 * p.R_i)
            r.area_outer, r.area_inner, r.time = sumA1, sumA2, self._time
            self._step += 1
            recs.append(r)
        if raise_on_error and recs and recs[-1].status != _abi.NIM_OK:
            _abi.check(recs[-1].status, "SlabRank.solve_nse")
        return recs
