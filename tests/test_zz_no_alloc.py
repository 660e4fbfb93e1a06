"""dspw_globals_noalloc: the global sums of a state the caller owns, computed
without any device allocation (for callers that cannot call cudaMalloc, e.g. a
driver that keeps all device memory in its own pool).  Checked against
dspw_globals on the same state, twice in a row, because every call reuses the
library's one fixed scratch array.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from dspw import Solver, capi, make_desc

pytestmark = pytest.mark.gpu


def _state(nx, ny):
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    p = np.zeros((5, 1, ny, nx))
    p[0, 0] = 1.0 + 0.3 * np.sin(2 * np.pi * (X + Y))
    p[1, 0] = 0.4 * np.cos(2 * np.pi * X)
    p[2, 0] = -0.2 * np.sin(2 * np.pi * Y)
    p[4, 0] = 1.0 + 0.1 * np.cos(2 * np.pi * (X - Y))
    return p


@pytest.mark.parametrize("precision", ["fp64", "fp32_bf16"])
def test_globals_noalloc_matches_globals_twice(precision):
    import torch

    lib = capi.lib()
    for call, (nx, ny) in enumerate(((96, 80), (300, 7))):   # two calls in a row, different sizes
        d = make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=nx, ny=ny, nz=1,
                      precision=precision)
        s = Solver(d)
        s.upload_prim(_state(nx, ny))
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
        assert np.all(np.abs(got - want) <= rtol * scale), (call, got, want)


def test_globals_noalloc_rejects_oversize_state():
    import torch

    lib = capi.lib()
    d = make_desc(model="euler", nx=4096, ny=4097, nz=1)   # above 16,777,216 cells
    out = torch.zeros(7, dtype=torch.float64, device="cuda")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.dspw_globals_noalloc(ctypes.byref(d), ctypes.c_void_p(buf.data_ptr()), 4096 * 4097, 8,
                                  ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1   # DSPW_ERR_ARG
