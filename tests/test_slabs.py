"""z-slab plan of the C ABI (nim_slab_layout, nim_slab_halo): every plane
owned once, halos of two planes from the neighbour, and exchange spans that
carry exactly the neighbour's copies of the halo planes.  Pure host
functions of libnimgpu.so: no GPU needed."""
import numpy as np
import pytest

from nimgpu import _abi
from nimgpu.slabs import slab_halo, slab_layout, slab_sizes


@pytest.fixture(scope="module", autouse=True)
def gpu_lib():
    if not _abi.gpu_lib_path().exists():
        pytest.skip("libnimgpu.so not built (needs nvcc: __graft_entry__.build())")


def test_layout_owns_every_plane_once():
    for n_z in range(3, 70):
        for nslab in range(1, n_z // 2 + 1):
            lay = [slab_layout(n_z, nslab, s) for s in range(nslab)]
            assert lay[0][2] == 0 and lay[-1][3] == n_z
            sizes = [ohi - olo for _, _, olo, ohi in lay]
            assert min(sizes) >= 2 and max(sizes) - min(sizes) <= 1
            for s, (lo, hi, olo, ohi) in enumerate(lay):
                assert lo == max(0, olo - 2) and hi == min(n_z, ohi + 2)
                if s:
                    assert olo == lay[s - 1][3]


@pytest.mark.parametrize("args", [(3, 2, 0), (8, 0, 0), (8, 2, 2), (8, 2, -1), (9, 5, 0), (2, 1, 0)])
def test_layout_rejects(args):
    with pytest.raises(_abi.NimError):
        slab_layout(*args)


@pytest.mark.parametrize("dims,nslab", [((12, 6, 6), 3), ((16, 12, 12), 5), ((15, 7, 13), 2), ((8, 3, 9), 4)])
def test_halo_spans_in_bounds_and_matched(dims, nslab):
    NT, NR, NZ = dims
    pl, rb = NT * NR, NT * (NR + 1)
    for s in range(nslab):
        lo, hi, olo, ohi = slab_layout(NZ, nslab, s)
        nc, nf = slab_sizes(NT, NR, hi - lo)
        held = hi - lo
        offT, offZ = rb * held, rb * held + pl * held
        for side in (0, 1):
            if (side == 0 and s == 0) or (side == 1 and s == nslab - 1):
                with pytest.raises(_abi.NimError):
                    slab_halo(NT, NR, NZ, nslab, s, side)
                continue
            recv, send = slab_halo(NT, NR, NZ, nslab, s, side)
            bounds = [(0, nc), (0, offT), (offT, offZ), (offZ, nf)]
            for spans in (recv, send):
                for (o, n), (b0, b1) in zip(spans, bounds):
                    assert n > 0 and b0 <= o and o + n <= b1
            # the halo is the neighbour's, the sent planes are this slab's own
            g_recv, g_send = recv[0][0] // pl + lo, send[0][0] // pl + lo
            if side == 0:
                assert (g_recv, g_send) == (olo - 2, olo)
            else:
                assert (g_recv, g_send) == (ohi, ohi - 2)
            if side == 1:
                r2, s2 = slab_halo(NT, NR, NZ, nslab, s + 1, 0)
                assert [n for _, n in send] == [n for _, n in r2]
                assert [n for _, n in recv] == [n for _, n in s2]


def _global_planes(NT, NR, NZ, lo, hi):
    """Global identity of each element of a slab's cell and face arrays:
    cells and faces numbered in the whole mesh's structured order."""
    pl, rb = NT * NR, NT * (NR + 1)
    held = hi - lo
    cells = np.arange(pl * held) + pl * lo
    offT, offZ = rb * NZ, rb * NZ + pl * NZ
    faces = np.concatenate([np.arange(rb * held) + rb * lo, offT + np.arange(pl * held) + pl * lo,
                            offZ + np.arange(pl * (held + 1)) + pl * lo])
    return cells.astype(np.float64), faces.astype(np.float64)


@pytest.mark.parametrize("dims,nslab", [((12, 6, 6), 3), ((16, 12, 12), 5), ((15, 7, 13), 2), ((10, 4, 23), 6)])
def test_exchange_restores_every_halo(dims, nslab):
    """Slab arrays filled with their whole-mesh identity, halos wiped, then
    the exchange nim_slab_step issues (per cut: the lower slab's sent
    planes into the upper's receive spans and back, both face halves):
    every element is whole again."""
    NT, NR, NZ = dims
    lay = [slab_layout(NZ, nslab, s) for s in range(nslab)]
    pl, rb = NT * NR, NT * (NR + 1)
    want, have = [], []
    for s, (lo, hi, olo, ohi) in enumerate(lay):
        c, f = _global_planes(NT, NR, NZ, lo, hi)
        want.append((c, np.concatenate([f, f])))
        cw, fw = c.copy(), f.copy()
        held = hi - lo
        offT, offZ = rb * held, rb * held + pl * held
        for k in [k for k in range(lo, hi) if not olo <= k < ohi]:
            l = k - lo
            cw[l * pl:(l + 1) * pl] = np.nan
            fw[rb * l:rb * (l + 1)] = np.nan
            fw[offT + l * pl:offT + (l + 1) * pl] = np.nan
        # an axial face row k lies between planes k-1 and k: the slab
        # computes it itself when either is owned (the cut faces)
        for k in range(lo, hi + 1):
            if not (olo <= k < ohi or olo <= k - 1 < ohi):
                l = k - lo
                fw[offZ + l * pl:offZ + (l + 1) * pl] = np.nan
        have.append((cw, np.concatenate([fw, fw])))
    nfs = [slab_sizes(NT, NR, hi - lo)[1] for lo, hi, _, _ in lay]

    def copy(a, sa, b, rb_):
        (ca, fa), (cb, fb) = have[a], have[b]
        (o, n), (p, m) = sa[0], rb_[0]
        assert n == m
        cb[p:p + n] = ca[o:o + n]
        for h in (0, 1):
            for t in (1, 2, 3):
                (o, n), (p, m) = sa[t], rb_[t]
                assert n == m
                fb[h * nfs[b] + p:h * nfs[b] + p + n] = fa[h * nfs[a] + o:h * nfs[a] + o + n]

    for s in range(nslab - 1):
        r_up, s_up = slab_halo(NT, NR, NZ, nslab, s, 1)
        r_dn, s_dn = slab_halo(NT, NR, NZ, nslab, s + 1, 0)
        copy(s, s_up, s + 1, r_dn)
        copy(s + 1, s_dn, s, r_up)
    for (wc, wf), (hc, hf) in zip(want, have):
        assert np.array_equal(wc, hc) and np.array_equal(wf, hf)
