"""nimgpu.SlabRank's control flow (one process per GPU, the z-slab path of
bench.py --gpus N) run by 2 and 3 gloo ranks on the CPU, with a stand-in for
the library's slab entry points: every part of a pass, the packed halo
exchange with each neighbour, the all-reduce of the find_error maxima before
each pass end, the polling of the loop state and the step-end reductions.

The stand-in gives each rank a different rate of convergence, so only the
all-reduced maxima can make the ranks stop together: every rank must leave
the loop after the same pass (the slowest rank's), receive each halo
payload from the right neighbour and side, and return the same per-step
records, whose sums are the group's."""
import ctypes as C
import math
import os
import socket
import struct
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
TOL = 1e-6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _value(b: int) -> float:
    return struct.unpack("<d", struct.pack("<q", b))[0]


class FakeSlabLib:
    """The slab entry points of include/nim_gpu.h as SlabRank calls them,
    over a toy iteration: rank r's change after pass n is 0.5^n (r+1), so
    the ranks would stop on different passes on their own."""

    def __init__(self, rank: int):
        self.rank = rank
        self.max = (C.c_int64 * 24)()
        self.done = 0
        self.passes = 0
        self.parts = []
        self.bad_payloads = []
        self.exchanges = 0
        self.last_err = [0.0] * 5

    # -- layout and contexts
    def nim_slab_layout(self, n_z, nslab, s, out):
        base, extra = divmod(n_z, nslab)
        olo = s * base + min(s, extra)
        ohi = olo + base + (1 if s < extra else 0)
        out[0], out[1], out[2], out[3] = max(olo - 2, 0), min(ohi + 2, n_z), olo, ohi
        return 0

    def nim_slab_halo(self, n_theta, n_r, n_z, nslab, s, side, recv, send):
        for t in range(8):
            recv[t] = send[t] = t
        return 0

    def nim_gpu_create_slab(self, mesh, params, nslab, s, h):
        h._obj.value = 1000 + s
        return 0

    def nim_gpu_init(self, h):
        return 0

    def nim_gpu_destroy(self, h):
        return None

    def nim_slab_pack_doubles(self, h, what, side):
        return 4 + what

    def nim_slab_maxima(self, h, slots):
        slots._obj.value = C.addressof(self.max)
        return 0

    # -- one step
    def nim_gpu_begin_step(self, h):
        self.done, self.passes = 0, 0
        return 0

    def _change(self, n: int) -> float:
        return 0.5 ** n * (self.rank + 1)

    def nim_slab_part(self, h, part):
        self.parts.append(part)
        if self.done:
            return 0
        if part == 0:  # the sweeps record this rank's changes
            e = self._change(self.passes + 1)
            for q in range(5):
                self.max[q] = _bits(e)
        elif part == 3:  # the pass end reads the group's maxima
            self.passes += 1
            self.last_err = [_value(self.max[q]) for q in range(5)]
            if max(self.last_err) < TOL:
                self.done = 1
        return 0

    def _view(self, buf, n):
        return (C.c_double * n).from_address(buf.value)

    def nim_slab_pack(self, h, what, side, buf):
        v = self._view(buf, 4 + what)
        v[0], v[1], v[2], v[3] = self.rank, side, what, self.passes
        return 0

    def nim_slab_unpack(self, h, what, side, buf):
        v = self._view(buf, 4 + what)
        peer = self.rank - 1 if side == 0 else self.rank + 1
        if (v[0], v[1], v[2], v[3]) != (peer, 1 - side, what, self.passes):
            self.bad_payloads.append((what, side, tuple(v[:4])))
        self.exchanges += 1
        return 0

    def nim_slab_loop_state(self, h, state, err):
        state[0], state[1], state[2] = self.done, self.passes, 0
        for q in range(5):
            err[q] = self.last_err[q]
        return 0

    def nim_slab_after_loop(self, h, out):
        out[0], out[1], out[2] = float(self.rank + 1), 0.1 * self.rank, 0.2 * self.rank
        return 0

    def nim_slab_end_step(self, h, out):
        out[0], out[1], out[2], out[3] = 1.0 * (self.rank + 1), 2.0, 3.0 * (self.rank + 1), 4.0
        return 0


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT / "nim-conv22-shared_b200"))
    import datetime

    from nimgpu import config
    from nimgpu.slabs import SlabRank

    class _Mesh:  # the few attributes SlabRank reads
        n_theta, n_r, n_z = 8, 4, 12
        nmesh = 8 * 4 * 12
        nface = 3 * nmesh + 8 * 12 + 8 * 4
        meshes_faces = None

        def __init__(self):
            from nimgpu import _abi
            self.desc = _abi.MeshDesc()

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import nimgpu.slabs as S
        S.structured_faces = lambda mesh: None  # no real mesh behind the stand-in
        lib = FakeSlabLib(rank)
        params = config.small_case().params()
        r = SlabRank(_Mesh(), params, lib=lib, device=torch.device("cpu"))
        r.initialize_nse()
        recs = r.solve_nse(2)
        out[rank] = {
            "recs": [(x.step, x.iters, x.status, x.err_u, x.dilatation, x.dudt_max, x.dTdt_max, x.nu_outer,
                      x.nu_inner, x.area_outer, x.area_inner, x.time) for x in recs],
            "bad": lib.bad_payloads, "exchanges": lib.exchanges, "parts": len(lib.parts),
        }
        r.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_rank_control_flow(world):
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == list(range(world))
    recs = [res[r]["recs"] for r in range(world)]
    assert all(x == recs[0] for x in recs), recs          # the same records on every rank
    # the slowest rank (the last) decides: 0.5^n world < TOL
    slow = float(world)
    want_iters = next(n for n in range(1, 200) if 0.5 ** n * slow < TOL)
    assert [x[1] for x in recs[0]] == [want_iters, want_iters]
    assert recs[0][0][3] == 0.5 ** want_iters * slow       # err_u: the group's maximum
    nmesh = 8 * 4 * 12
    dsum = sum(range(1, world + 1))
    assert recs[0][0][4] == pytest.approx(math.sqrt(dsum / nmesh))
    assert recs[0][0][5] == pytest.approx(0.1 * (world - 1)) and recs[0][0][6] == pytest.approx(0.2 * (world - 1))
    # Nusselt numbers from the summed wall integrals
    s1, a1, s2, a2 = float(dsum), 2.0 * world, 3.0 * dsum, 4.0 * world
    assert recs[0][0][7] == pytest.approx(-(s1 / a1 * 0.5))
    assert recs[0][0][9] == a1 and recs[0][0][10] == a2
    for r in range(world):
        assert res[r]["bad"] == []                      # every payload from the right neighbour
        neighbours = (r > 0) + (r < world - 1)
        assert res[r]["exchanges"] > 0 and res[r]["exchanges"] % neighbours == 0
    # every rank queued the same number of parts (the same collective sequence)
    assert len({res[r]["parts"] for r in range(world)}) == 1
