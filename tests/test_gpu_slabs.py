"""Slab decomposition on the GPU (dspw.slabs.LocalSlabs): one problem cut into
slabs along its last swept direction, halo layers exchanged before every stage,
one dt for all slabs.  Every slab face then sees the stencil it sees in the
undivided problem, so the slabs reproduce the undivided run bit for bit: 2-D
and 3-D, FP64 and the FP32 + BF16 network form (specialised cooperative y / z
sweeps), eno 3 (three halo layers), walls and neumann faces at the outer
ends, periodic wrap (also between two slabs and within one), 1-D slabs along
x, and a scalar law."""
import numpy as np
import pytest

from _common import net
from dspw import Solver, make_desc
from dspw.slabs import LocalSlabs

pytestmark = pytest.mark.gpu


def state(nv, nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    if nv == 1:
        return (0.5 + np.sin(2 * np.pi * X) + 0.2 * rng.standard_normal(X.shape))[None]
    p = np.zeros((5, nz, ny, nx))
    p[0] = 1.0 + 0.3 * np.sin(2 * np.pi * (X + 2 * Y + Z)) + 0.05 * rng.standard_normal(X.shape)
    p[1] = 0.4 * np.cos(2 * np.pi * (X - Y))
    p[2] = 0.3 * np.sin(2 * np.pi * (X + Z)) * (ny > 1)
    p[3] = 0.2 * np.cos(2 * np.pi * (Y + Z)) * (nz > 1)
    p[4] = 1.0 + 0.2 * np.cos(2 * np.pi * (X + Y - Z)) + 0.02 * rng.standard_normal(X.shape)
    return p


def undivided(d, p0, nsteps, nrk):
    """The domain as one problem, stepped by the same host loop (CFL dt of the
    state, then the stages)."""
    s = Solver(d)
    s.upload_prim(p0)
    for _ in range(nsteps):
        dt = s.compute_dt()
        for rk in range(nrk):
            s.stage(rk, dt)
    return s


CASES = {
    "kh2d_fp64_3slabs": (dict(flux="kepes_tecno4_roe", recon="sp_weno", nx=40, ny=36, nz=1), 3),
    "kh2d_fp32_dl_4slabs": (dict(flux="kepes_tecno4_roe", recon="sp_weno_dl", nx=48, ny=32, nz=1,
                                 precision="fp32_bf16"), 4),
    "wall2d_roe_2slabs": (dict(flux="roe_tecno_roe", recon="sp_wenoc", nx=24, ny=20, nz=1, ec1_fix=True,
                               bc=["wall", "neumann", "wall", "neumann", "periodic", "periodic"]), 2),
    "periodic2d_2slabs": (dict(flux="kepes_tecno4_rusanov", recon="minmod", nx=16, ny=10, nz=1), 2),
    "periodic2d_1slab": (dict(flux="kepes_tecno4_roe", recon="sp_weno", nx=16, ny=10, nz=1), 1),
    "euler3d_eno3_3slabs": (dict(flux="kepes_tecno4_roe", recon="eno3", nx=12, ny=9, nz=11,
                                 bc=["periodic", "periodic", "wall", "wall", "neumann", "wall"]), 3),
    "euler3d_fp32_dl_2slabs": (dict(flux="kepes_tecno4_roe", recon="sp_weno_dl", nx=16, ny=12, nz=10,
                                    precision="fp32_bf16"), 2),
    "shu1d_5slabs": (dict(flux="kepes_tecno4_roe", recon="sp_weno_dl", nx=150, ny=1, nz=1, bc="neumann"), 5),
    "burgers1d_3slabs": (dict(model="burgers", flux="bur_tecno4", recon="sp_wenoc", nx=90, ny=1, nz=1,
                              x=(-np.pi, np.pi)), 3),
    "kh2d_rk4_3slabs": (dict(flux="kepes_tecno4_roe", recon="sp_weno", nx=24, ny=18, nz=1, time_scheme="rk4"), 3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_slabs_reproduce_the_undivided_problem(name):
    kw, nslab = CASES[name]
    kw = dict(kw)
    d = make_desc(network=net(), cfl=0.4, final_time=10.0, **kw)
    nv = 1 if kw.get("model") == "burgers" else 5
    p0 = state(nv, d.nx, d.ny, d.nz, seed=len(name))
    nrk = {"rk4": 4}.get(kw.get("time_scheme", "ssprk3"), 3)
    nsteps = 6
    ref = undivided(d, p0, nsteps, nrk)
    sl = LocalSlabs(d, nslab)
    sl.upload_prim(p0)
    sl.step(nsteps)
    a, b = sl.cons(), ref.cons()
    assert np.all(np.isfinite(a))
    assert np.array_equal(a, b), (name, float(np.max(np.abs(a - b))))
    for g in sl.globals():
        assert g.iter == nsteps and g.time == ref.globals().time
    for sol, _, _ in sl.parts:
        st = sol.status()
        assert st.code == 0 and st.nonfinite_cells == 0


def test_slab_handles_refuse_the_diagnostics():
    d = make_desc(nx=16, ny=12, nz=1)
    sl = LocalSlabs(d, 2)
    from dspw.capi import lib
    assert lib().dspw_diag_enable(sl.parts[0][0].h, 8) == 6


def _dist_rank(rank, world, port, name, q):
    import os
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from dspw.slabs import DistSlabs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        kw, _ = CASES[name]
        d = make_desc(network=net(), cfl=0.4, final_time=10.0, **dict(kw))
        nv = 1 if kw.get("model") == "burgers" else 5
        p0 = state(nv, d.nx, d.ny, d.nz, seed=len(name))
        sl = DistSlabs(d, rank, world)
        sl.upload_prim(p0)
        sl.step(6)
        q.put((rank, sl.lo, sl.hi, sl.local_cons()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("kh2d_fp64_3slabs", 2), ("euler3d_eno3_3slabs", 3)])
def test_rank_slabs_reproduce_the_undivided_problem(name, world):
    """DistSlabs as `world` processes sharing this GPU, layers and dt over gloo
    (host-staged): the ranks' slabs together equal the undivided run bit for
    bit.  The NCCL transport differs only in moving the layers GPU to GPU."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_dist_rank, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    parts = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    kw, _ = CASES[name]
    d = make_desc(network=net(), cfl=0.4, final_time=10.0, **dict(kw))
    p0 = state(5, d.nx, d.ny, d.nz, seed=len(name))
    ref = undivided(d, p0, 6, 3).cons()
    D = 2 if d.nz > 1 else 1
    for rank, lo, hi, local in parts:
        want = ref[:, lo:hi] if D == 2 else ref[:, :, lo:hi]
        assert np.array_equal(local, want), (name, rank)


@pytest.mark.parametrize("name", ["kh2d_fp64_3slabs", "kh2d_fp32_dl_4slabs", "euler3d_eno3_3slabs",
                                  "burgers1d_3slabs", "kh2d_rk4_3slabs"])
def test_nccl_slab_in_the_step_graph(name):
    """One slab connected over NCCL (dspw_slab_connect, one rank): a periodic
    domain's slab sends its boundary layers to itself and receives them as
    its halo, and all-reduces its CFL speed, inside the step graph; a walled
    domain's slab has no halo faces and only reduces.  Both equal the
    undivided problem's own graph steps bit for bit, and so do stages issued
    one by one (dspw_stage with the dt of the graph's rule)."""
    from dspw.slabs import connect, split
    kw, _ = CASES[name]
    d = make_desc(network=net(), cfl=0.4, final_time=10.0, **dict(kw))
    nv = 1 if kw.get("model") == "burgers" else 5
    p0 = state(nv, d.nx, d.ny, d.nz, seed=len(name))
    ref = Solver(d)
    ref.upload_prim(p0)
    ref.step(5)
    sd, lo, hi = split(d, 1)[0]
    s = Solver(sd)
    s.upload_prim(p0)
    connect(s, 0, 1)
    s.step(3)
    nrk = {"rk4": 4}.get(kw.get("time_scheme", "ssprk3"), 3)
    for _ in range(2):
        for rk in range(nrk):
            s.stage(rk, 0.0)
    assert np.array_equal(s.cons(), ref.cons()), name
    assert s.globals().time == ref.globals().time and s.globals().iter == 5
