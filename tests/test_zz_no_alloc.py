"""dspw_globals_noalloc: the global sums of a state the caller owns, computed
without any device allocation (for callers that cannot call cudaMalloc, e.g. a
driver that keeps all device memory in its own pool).  Checked against
dspw_globals on the same state, twice in a row, because every call reuses the
library's one fixed scratch array.  This file is collected last on purpose.
"""
import ctypes
import math

import numpy as np
import pytest

from dspw import Solver, capi, make_desc
from dspw.slabs import split

pytestmark = pytest.mark.gpu


def _state(nx, ny, nz=1, scalar=False):
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    if scalar:
        return (0.5 + 0.4 * np.sin(2 * np.pi * X)).reshape(1, nz, ny, nx)
    p = np.zeros((5, nz, ny, nx))
    p[0] = 1.0 + 0.3 * np.sin(2 * np.pi * (X + Y + Z))
    p[1] = 0.4 * np.cos(2 * np.pi * X)
    if ny > 1:
        p[2] = -0.2 * np.sin(2 * np.pi * Y)
    if nz > 1:
        p[3] = 0.1 * np.cos(2 * np.pi * Z)
    p[4] = 1.0 + 0.1 * np.cos(2 * np.pi * (X - Y))
    return p


def _slab_desc(precision):
    """The middle slab of a 3-slab cut of a 2-D domain whose bounds over its
    cell count do not round to the domain's cell size (descriptor cell_size)."""
    dom = make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=40, ny=37, nz=1,
                    x=(-0.37, 1.91), y=(-0.37, 1.91), precision=precision)
    d, lo, hi = split(dom, 3)[1]
    return d


# (name, descriptor builder): two calls in a row per case, different sizes and
# component layouts (nv = 1, 3, 4, 5)
CASES = {
    "euler2d": lambda pr: [make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=96, ny=80, nz=1,
                                     precision=pr),
                           make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=300, ny=7, nz=1,
                                     precision=pr)],
    "burgers1d": lambda pr: [make_desc(model="burgers", flux="bur_tecno4", recon="sp_weno", nx=500,
                                       x=(-math.pi, math.pi), precision=pr),
                             make_desc(model="burgers", flux="bur_tecno4", recon="sp_weno", nx=77,
                                       x=(-math.pi, math.pi), precision=pr)],
    "euler1d": lambda pr: [make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=400, x=(-5, 5),
                                     precision=pr),
                           make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=123, x=(-5, 5),
                                     precision=pr)],
    "euler3d": lambda pr: [make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=20, ny=18, nz=16,
                                     precision=pr),
                           make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=9, ny=12, nz=10,
                                     precision=pr)],
    "slab2d": lambda pr: [_slab_desc(pr), _slab_desc(pr)],
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "fp32_bf16"])
def test_globals_noalloc_matches_globals_twice(case, precision):
    import torch

    lib = capi.lib()
    for call, d in enumerate(CASES[case](precision)):
        s = Solver(d)
        s.upload_prim(_state(d.nx, d.ny, d.nz, scalar=d.model <= 1))
        if case != "slab2d":   # a slab's halo layers are the caller's: no steps
            s.step(2)
        ref = s.globals()
        ptr, stride, eb = ctypes.c_void_p(), ctypes.c_longlong(), ctypes.c_int()
        capi.check(lib.dspw_device_state(s.h, 0, ctypes.byref(ptr), ctypes.byref(stride), ctypes.byref(eb)),
                   "dspw_device_state")
        out = torch.full((7,), float("nan"), dtype=torch.float64, device="cuda")
        s.sync()
        capi.check(lib.dspw_globals_noalloc(ctypes.byref(d), ptr, stride.value, eb.value,
                                            ctypes.c_void_p(out.data_ptr()), s.stream_ptr()), "dspw_globals_noalloc")
        s.sync()
        got = out.cpu().numpy()
        want = np.array([ref.total_entropy, ref.kinetic_energy] + list(ref.conserved))
        scale = np.abs(want) + np.max(np.abs(want))
        # dspw_globals evaluates the pressure of an FP32 state in FP32 before the
        # log; this entry point evaluates it in FP64 from the same FP32 values
        rtol = 1e-12 if precision == "fp64" else 1e-5
        assert np.all(np.abs(got - want) <= rtol * scale), (case, call, got, want)


def test_globals_noalloc_rejects_bad_arguments():
    import torch

    lib = capi.lib()
    out = torch.zeros(7, dtype=torch.float64, device="cuda")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    d = make_desc(model="euler", nx=4096, ny=4097, nz=1)   # above 16,777,216 cells
    rc = lib.dspw_globals_noalloc(ctypes.byref(d), ctypes.c_void_p(buf.data_ptr()), 4096 * 4097, 8,
                                  ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1   # DSPW_ERR_ARG
    d = make_desc(model="euler", nx=4, ny=4, nz=1)
    d.model = 7      # no such model
    rc = lib.dspw_globals_noalloc(ctypes.byref(d), ctypes.c_void_p(buf.data_ptr()), 16, 8,
                                  ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
