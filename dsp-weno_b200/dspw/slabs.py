"""Slab decomposition of one problem along its last swept direction.

The layers of that direction (y rows of a 2-D problem, z planes of a 3-D one,
x cells of a 1-D one; the outermost direction in memory) are cut into slabs of
contiguous layers.  Every slab is a problem of its own whose faces towards its
neighbours are ``halo`` faces (DSPW_BC_HALO): their ghost layers (2, or 3 for
eno 3) are stored beside the interior and, before every stage, filled with the
neighbours' boundary layers of the state that stage reads.  The outer faces
keep the domain's boundary conditions; a periodic domain wraps the first and
the last slab around.  Every slab takes the same dt, the minimum over the
slabs of the CFL step (the domain's own CFL step), clipped to the time stamps
as a single problem's.  A face flux then sees the stencil it sees in the
undivided problem, so the slabs reproduce it bit for bit.

Two transports move the layers:

* ``LocalSlabs``: every slab in this process, one handle each (one GPU):
  device-to-device copies.
* ``DistSlabs``: one slab per rank of a ``torch.distributed`` group (NCCL over
  NVLink / NVSwitch on a multi-GPU node): point-to-point sends and receives in
  two phases (upwards, then downwards), the dt by an all-reduce(min).

The reference has no decomposition (its solver is serial); this is the
structured-grid sharding of its stage loop (enflo/src/fv.cc:1262-1313): the
halo exchange stands where apply_bc fills ghost layers (fv.cc:121-361).
"""
from __future__ import annotations

import numpy as np

from .capi import BC, RECON, Desc, Solver, nvar

_AXIS = ("x", "y", "z")


def problem_dim(d: Desc) -> int:
    return 3 if d.nz > 1 else (2 if d.ny > 1 else 1)


def ghost_width(d: Desc) -> int:
    return 3 if d.recon == RECON["eno3"] else 2


def layer_ranges(n: int, nslab: int) -> list[tuple[int, int]]:
    """Layers [lo, hi) of each slab: as even as possible, the first n % nslab
    slabs one layer longer."""
    base, extra = divmod(n, nslab)
    out, lo = [], 0
    for s in range(nslab):
        hi = lo + base + (1 if s < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def split(desc: Desc, nslab: int) -> list[tuple[Desc, int, int]]:
    """(slab descriptor, first layer, end layer) of each slab of `desc`."""
    dim = problem_dim(desc)
    D = dim - 1
    n = (desc.nx, desc.ny, desc.nz)[D]
    ng = ghost_width(desc)
    if nslab < 1 or n < nslab * ng:
        raise ValueError(f"{n} layers cannot make {nslab} slabs of at least {ng} layers")
    lo_b = (desc.xmin, desc.ymin, desc.zmin)[D]
    hi_b = (desc.xmax, desc.ymax, desc.zmax)[D]
    h = (hi_b - lo_b) / n
    periodic = desc.bc[2 * D] == BC["periodic"]
    cell = [(desc.xmax - desc.xmin) / desc.nx, (desc.ymax - desc.ymin) / desc.ny, (desc.zmax - desc.zmin) / desc.nz]
    out = []
    for s, (lo, hi) in enumerate(layer_ranges(n, nslab)):
        d = Desc.from_buffer_copy(desc)
        setattr(d, "n" + _AXIS[D], hi - lo)
        setattr(d, _AXIS[D] + "min", lo_b + lo * h)
        setattr(d, _AXIS[D] + "max", lo_b + hi * h)
        # the slab keeps the domain's cell sizes exactly (descriptor cell_size)
        for k in range(3):
            if d.cell_size[k] <= 0.0:
                d.cell_size[k] = cell[k]
        if nslab > 1 or periodic:
            if s > 0 or periodic:
                d.bc[2 * D] = BC["halo"]
            if s < nslab - 1 or periodic:
                d.bc[2 * D + 1] = BC["halo"]
        out.append((d, lo, hi))
    return out


class _DeviceSpan:
    """A span of device memory seen by torch without a copy."""

    def __init__(self, ptr: int, count: int, elem_bytes: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8" if elem_bytes == 8 else "<f4",
                                         "data": (int(ptr), False), "version": 3}


def layer_tensors(view, device):
    """Per component: the torch tensors (send_lo, send_hi, recv_lo, recv_hi)
    over a slab's halo view, on `device`, sharing its memory."""
    import torch
    out = {k: [] for k in ("send_lo", "send_hi", "recv_lo", "recv_hi")}
    for c in range(view.ncomp):
        for k in out:
            ptr = getattr(view, k) + c * view.comp_stride * view.elem_bytes
            out[k].append(torch.as_tensor(_DeviceSpan(ptr, view.count, view.elem_bytes), device=device))
    return out


def exchange_layers(send_lo, send_hi, recv_lo, recv_hi, rank: int, world: int, periodic: bool, group=None):
    """Fill this rank's halo layers from its neighbours' boundary layers.

    Each argument lists one tensor per component.  The first and the last rank
    of a non-periodic domain skip their outer face.  Phase 1 moves layers upwards (a rank's send_hi into the upper
    neighbour's recv_lo), phase 2 downwards; within a phase each pair of ranks
    exchanges at most one message per component, issued in component order
    on both sides, so sends and receives pair up also when the two
    neighbours are the same rank (two slabs, periodic)."""
    import torch.distributed as dist
    up = rank + 1 if rank + 1 < world else (0 if periodic else None)
    down = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    for send, recv, to, frm in ((send_hi, recv_lo, up, down), (send_lo, recv_hi, down, up)):
        ops = []
        if to is not None:
            ops += [dist.P2POp(dist.isend, t, to, group) for t in send]
        if frm is not None:
            ops += [dist.P2POp(dist.irecv, t, frm, group) for t in recv]
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()


def connect(sol: Solver, rank: int, world: int, group=None):
    """Connect a one-slab handle to its neighbours over NCCL (dspw_slab_connect):
    rank 0 makes the NCCL id and the group hands it to every rank.  The
    handle's steps then exchange halo layers and reduce the CFL speed on the
    GPU, inside its step graph."""
    import ctypes

    from .capi import check, lib
    buf = ctypes.create_string_buffer(128)
    if rank == 0:
        check(lib().dspw_nccl_id(buf), "dspw_nccl_id")
    raw = buf.raw
    if world > 1:
        import torch.distributed as dist
        obj = [raw]
        dist.broadcast_object_list(obj, src=0, group=group)
        raw = obj[0]
    check(lib().dspw_slab_connect(sol.h, raw, int(rank), int(world)), "dspw_slab_connect")


class _SlabsBase:
    def upload_prim(self, prim):
        """prim: the domain's primitive planes (nvar, nz, ny, nx)."""
        for sol, lo, hi in self._mine():
            sol.upload_prim(np.ascontiguousarray(self._take(prim, lo, hi)))

    def _take(self, a, lo, hi):
        D = self.D
        sl = [slice(None)] * 4
        sl[3 - D] = slice(lo, hi)
        return a[tuple(sl)]

    def step(self, n=1):
        """n steps: the common dt, then for every stage the halo exchange of the
        stage's input state and the stage on every slab."""
        for _ in range(int(n)):
            dt = self.dt()
            for rk in range(self.nrk):
                self.exchange(rk)
                for sol, _, _ in self._mine():
                    sol.stage(rk, dt)


class LocalSlabs(_SlabsBase):
    """Every slab of `desc` in this process, one handle each, on one GPU."""

    def __init__(self, desc: Desc, nslab: int):
        import torch
        self.D = problem_dim(desc) - 1
        self.periodic = desc.bc[2 * self.D] == BC["periodic"]
        self.parts = [(Solver(d), lo, hi) for d, lo, hi in split(desc, nslab)]
        self.shape = (nvar(desc), desc.nz, desc.ny, desc.nx)
        self.nrk = {0: 1, 1: 3}.get(desc.time_scheme, 4)
        self.device = torch.device("cuda", torch.cuda.current_device())

    def _mine(self):
        return self.parts

    def dt(self) -> float:
        return min(sol.compute_dt() for sol, _, _ in self.parts)

    def exchange(self, rk: int):
        import torch
        k = len(self.parts)
        if k == 1 and not self.periodic:
            return
        views = [layer_tensors(sol.halo_view(0, rk), self.device) for sol, _, _ in self.parts]
        for s in range(k):
            up = s + 1 if s + 1 < k else (0 if self.periodic else None)
            if up is None:
                continue
            for c in range(len(views[s]["send_hi"])):
                views[up]["recv_lo"][c].copy_(views[s]["send_hi"][c])
                views[s]["recv_hi"][c].copy_(views[up]["send_lo"][c])
        torch.cuda.current_stream().synchronize()

    def prim(self) -> np.ndarray:
        return self._gather(lambda sol: sol.prim())

    def cons(self) -> np.ndarray:
        return self._gather(lambda sol: sol.cons())

    def _gather(self, get):
        out = np.empty(self.shape)
        for sol, lo, hi in self.parts:
            self._take(out, lo, hi)[...] = get(sol)
        return out

    def globals(self):
        return [sol.globals() for sol, _, _ in self.parts]


class DistSlabs(_SlabsBase):
    """Slab `rank` of `desc` split over the `world` ranks of a torch.distributed
    group: with NCCL the layers move GPU to GPU; with gloo they are staged
    through host memory (ranks that share a GPU, or checks without NCCL).
    Every rank's kernels have finished before its exchange starts: no kernel
    waits on another rank."""

    def __init__(self, desc: Desc, rank: int, world: int, group=None, device_exchange=False):
        import torch
        self.D = problem_dim(desc) - 1
        self.periodic = desc.bc[2 * self.D] == BC["periodic"]
        self.rank, self.world, self.group = rank, world, group
        d, lo, hi = split(desc, world)[rank]
        self.sol, self.lo, self.hi = Solver(d), lo, hi
        self.nrk = {0: 1, 1: 3}.get(desc.time_scheme, 4)
        self.device = torch.device("cuda", torch.cuda.current_device())
        # device_exchange: the library's NCCL path (halo layers and dt on the
        # GPU inside the step graph, no host round trip per stage)
        self.device_exchange = bool(device_exchange)
        if self.device_exchange:
            connect(self.sol, rank, world, group)

    def step(self, n=1):
        if self.device_exchange:
            self.sol.step(n)
        else:
            super().step(n)

    def _mine(self):
        return [(self.sol, self.lo, self.hi)]

    def _host_staged(self) -> bool:
        import torch.distributed as dist
        return dist.get_backend(self.group) != "nccl"

    def dt(self) -> float:
        import torch
        import torch.distributed as dist
        dev = "cpu" if self._host_staged() else self.device
        t = torch.tensor([self.sol.compute_dt()], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t.item())

    def exchange(self, rk: int):
        import torch
        v = layer_tensors(self.sol.halo_view(0, rk), self.device)
        if self.world == 1:
            if self.periodic:
                for c in range(len(v["send_hi"])):
                    v["recv_lo"][c].copy_(v["send_hi"][c])
                    v["recv_hi"][c].copy_(v["send_lo"][c])
        elif self._host_staged():
            h = {k: [t.cpu() for t in v[k]] for k in v}
            exchange_layers(h["send_lo"], h["send_hi"], h["recv_lo"], h["recv_hi"], self.rank, self.world,
                            self.periodic, self.group)
            has_down = self.rank > 0 or self.periodic
            has_up = self.rank + 1 < self.world or self.periodic
            for c in range(len(v["recv_lo"])):
                if has_down:
                    v["recv_lo"][c].copy_(h["recv_lo"][c])
                if has_up:
                    v["recv_hi"][c].copy_(h["recv_hi"][c])
        else:
            exchange_layers(v["send_lo"], v["send_hi"], v["recv_lo"], v["recv_hi"], self.rank, self.world,
                            self.periodic, self.group)
        torch.cuda.current_stream().synchronize()

    def local_cons(self) -> np.ndarray:
        return self.sol.cons()


__all__ = ["split", "layer_ranges", "exchange_layers", "layer_tensors", "connect", "LocalSlabs", "DistSlabs"]
