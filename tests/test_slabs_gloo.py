"""The halo exchange of z-slabs over torch.distributed
(nimgpu.exchange_packed), run by 2 and 3 gloo ranks on the CPU: each rank
holds one slab's arrays (a cell and a face array per field, both face
halves) filled with their whole-mesh identity and its halo wiped, packs
each side in the order nim_slab_pack uses, exchanges one message per
neighbour and unpacks: every element is whole again.  The same function
moves the device-packed payloads over NCCL between one process per GPU."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _slab_arrays(NT, NR, NZ, nslab, s, nfields):
    """(want, have) lists of (tensor, is_face) for slab s: the whole-mesh
    identity of every element, and the same with the halo wiped (NaN)."""
    from nimgpu.slabs import slab_layout
    lo, hi, olo, ohi = slab_layout(NZ, nslab, s)
    pl, rb, held = NT * NR, NT * (NR + 1), hi - lo
    offT, offZ = rb * NZ, rb * NZ + pl * NZ
    cells = np.arange(pl * held) + pl * lo
    faces = np.concatenate([np.arange(rb * held) + rb * lo, offT + np.arange(pl * held) + pl * lo,
                            offZ + np.arange(pl * (held + 1)) + pl * lo]).astype(np.float64)
    lt, lz = rb * held, rb * held + pl * held
    cw, fw = cells.astype(np.float64), faces.copy()
    for k in range(lo, hi):
        if not olo <= k < ohi:
            l = k - lo
            cw[l * pl:(l + 1) * pl] = np.nan
            fw[rb * l:rb * (l + 1)] = np.nan
            fw[lt + l * pl:lt + (l + 1) * pl] = np.nan
    for k in range(lo, hi + 1):  # axial rows between two planes neither owned
        if not (olo <= k < ohi or olo <= k - 1 < ohi):
            fw[lz + (k - lo) * pl:lz + (k - lo + 1) * pl] = np.nan
    want, have = [], []
    for q in range(nfields):
        base = 1e7 * q
        want += [(torch.from_numpy(cells + base), False), (torch.from_numpy(np.concatenate([faces, faces + 0.5]) + base), True)]
        have += [(torch.from_numpy(cw + base), False), (torch.from_numpy(np.concatenate([fw, fw + 0.5]) + base), True)]
    return want, have, faces.size


def _rank(rank, world, port, dims, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT / "nim-conv22-shared_b200"))
    from nimgpu.slabs import exchange_packed, slab_halo
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        NT, NR, NZ = dims
        want, have, nf = _slab_arrays(NT, NR, NZ, world, rank, 3)
        plans = {}
        if rank > 0:
            plans[0] = slab_halo(NT, NR, NZ, world, rank, 0)
        if rank < world - 1:
            plans[1] = slab_halo(NT, NR, NZ, world, rank, 1)

        def views(side, send):
            # nim_slab_pack's order: each array; a face array's spans 1..3 of
            # its first half, then of its second
            recv_sp, send_sp = plans[side]
            sp = send_sp if send else recv_sp
            out = []
            for a, face in have:
                for base, t in ([(h * nf, t) for h in (0, 1) for t in (1, 2, 3)] if face else [(0, 0)]):
                    o, n = sp[t]
                    out.append(a[base + o:base + o + n])
            return out

        send = {side: torch.cat(views(side, True)) for side in plans}
        recv = {side: torch.empty_like(send[side]) for side in plans}
        exchange_packed(send, recv, rank)
        for side in plans:
            off = 0
            for v in views(side, False):
                v.copy_(recv[side][off:off + v.numel()])
                off += v.numel()
        out[rank] = all(torch.equal(w, h) for (w, _), (h, _) in zip(want, have))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims", [(2, (12, 6, 6)), (3, (10, 4, 11))])
def test_exchange_over_gloo(world, dims):
    if not (ROOT / "nim-conv22-shared_b200" / "lib" / "libnimgpu.so").exists():
        pytest.skip("libnimgpu.so not built")
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), dims, out), nprocs=world, join=True)
        res = dict(out)
    assert res == {r: True for r in range(world)}
