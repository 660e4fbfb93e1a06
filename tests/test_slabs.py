"""Host logic of the slab decomposition (dspw.slabs), on CPU: the split of a
domain's layers, slab bounds that reproduce the domain's cell size exactly
(the kernels derive it from the bounds), the halo faces, and the layer
exchange between ranks as real gloo processes (two and three ranks, periodic
and walled)."""
import os
import socket

import numpy as np
import pytest

from dspw import make_desc
from dspw.capi import BC
from dspw.slabs import exchange_layers, layer_ranges, split


def test_layer_ranges_cover_the_domain():
    for n in (6, 7, 31, 2048):
        for k in (1, 2, 3, 5):
            if n < k:
                continue
            r = layer_ranges(n, k)
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [hi - lo for lo, hi in r]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("bounds", [(0.0, 1.0), (0.0, 2 * np.pi), (-5.0, 5.0), (-0.37, 1.91)])
@pytest.mark.parametrize("n,k", [(2048, 3), (100, 7), (37, 4), (12, 2)])
def test_slabs_keep_the_cell_size(bounds, n, k):
    """Each slab carries the domain's cell sizes (descriptor cell_size), since
    its own bounds over its own cell count need not round to them."""
    d = make_desc(nx=16, ny=n, nz=1, y=bounds, x=(0.0, 0.3))
    h = [(d.xmax - d.xmin) / d.nx, (d.ymax - d.ymin) / d.ny, (d.zmax - d.zmin) / d.nz]
    for s, lo, hi in split(d, k):
        assert list(s.cell_size) == h             # bit for bit
        assert s.ny == hi - lo and abs(s.ymin - (d.ymin + lo * h[1])) <= 1e-12 * max(1.0, abs(d.ymin))
        assert (s.nx, s.nz) == (d.nx, d.nz) and (s.xmin, s.xmax) == (d.xmin, d.xmax)


def test_halo_faces():
    per = make_desc(nx=8, ny=12, nz=1, bc="periodic")
    sl = split(per, 3)
    assert all(s.bc[2] == BC["halo"] and s.bc[3] == BC["halo"] for s, _, _ in sl)
    assert all(s.bc[0] == BC["periodic"] for s, _, _ in sl)
    walled = make_desc(nx=8, ny=1, nz=10, bc=["periodic", "periodic", "wall", "wall", "neumann", "wall"])
    sl = split(walled, 3)
    assert [(s.bc[4], s.bc[5]) for s, _, _ in sl] == [(BC["neumann"], BC["halo"]), (BC["halo"], BC["halo"]),
                                                      (BC["halo"], BC["wall"])]
    # one slab of a walled domain is the domain itself
    s, lo, hi = split(walled, 1)[0]
    assert list(s.bc) == list(walled.bc) and (lo, hi) == (0, 10)
    # eno 3 needs three layers per slab
    with pytest.raises(ValueError):
        split(make_desc(recon="eno3", nx=8, ny=8, nz=1), 3)
    split(make_desc(recon="eno3", nx=8, ny=9, nz=1), 3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, periodic, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ncomp, count = 4, 6
        # boundary layers carry (rank, side, component) so every halo shows its source
        send_lo = [torch.full((count,), 100.0 * rank + 10 * 0 + c) for c in range(ncomp)]
        send_hi = [torch.full((count,), 100.0 * rank + 10 * 1 + c) for c in range(ncomp)]
        recv_lo = [torch.full((count,), -1.0) for _ in range(ncomp)]
        recv_hi = [torch.full((count,), -1.0) for _ in range(ncomp)]
        exchange_layers(send_lo, send_hi, recv_lo, recv_hi, rank, world, periodic)
        q.put((rank, [t[0].item() for t in recv_lo], [t[0].item() for t in recv_hi]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_layer_exchange_over_gloo(world, periodic):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, periodic, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        rank, lo, hi = q.get(timeout=120)
        got[rank] = (lo, hi)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        lo, hi = got[r]
        down = r - 1 if r > 0 else (world - 1 if periodic else None)
        up = r + 1 if r + 1 < world else (0 if periodic else None)
        # the lower halo holds the lower neighbour's top layers, the upper halo
        # the upper neighbour's bottom layers; outer faces stay untouched
        assert lo == ([100.0 * down + 10 + c for c in range(4)] if down is not None else [-1.0] * 4), (r, lo)
        assert hi == ([100.0 * up + c for c in range(4)] if up is not None else [-1.0] * 4), (r, hi)
