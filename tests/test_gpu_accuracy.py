"""Accuracy of the FP32 + BF16-network form against the FP64 forms.

* Shu-Osher (1-D Euler, transmissive BCs, t = 1.8): the reference solution is
  the FP64 SP-WENO run at Nx = 12800, cell-averaged to the coarse grid.  The
  FP32 DSP-WENO L1 density error must stay within 1.5x of the FP64 DSP-WENO
  error (and of the FP64 plain SP-WENO error) at Nx = 400 and 800.
* Kelvin-Helmholtz 128^2 to t = 1.0: the FP32 DSP-WENO state is compared with
  the FP64 DSP-WENO state (no exact solution exists; the shear layer's
  instability amplifies any difference, so this is a report with a loose bound).
Every FP32 run must keep the sign property at every checked face (the FP64
form is the reference's unlimited network, whose violations are reported).
"""
import numpy as np
import pytest

from _common import net
from dspw import Solver, workloads as W

pytestmark = pytest.mark.gpu


def run(descs, prims):
    s = Solver(descs)
    for p, a in enumerate(prims):
        s.upload_prim(a, p)
    s.run(chunk=256)
    return s


@pytest.fixture(scope="module")
def shu_reference():
    d, p, _ = W.shu_osher(12800, "fp64", "sp_weno", net())
    s = run(d, p)
    assert abs(s.globals().time - 1.8) < 1e-12
    return s.prim()[0, 0, 0]


@pytest.mark.parametrize("nx", [400, 800])
def test_shu_osher_fp32_dl_error_within_1p5x_of_fp64(shu_reference, nx):
    ref = shu_reference.reshape(nx, -1).mean(axis=1)
    err = {}
    for prec, rec in (("fp64", "sp_weno"), ("fp64", "sp_weno_dl"), ("fp32_bf16", "sp_weno_dl")):
        d, p, _ = W.shu_osher(nx, prec, rec, net())
        s = run(d, p)
        st = s.status()
        assert st.code == 0 and st.sign_violations == 0
        err[(prec, rec)] = float(np.mean(np.abs(s.prim()[0, 0, 0] - ref)))
    e32 = err[("fp32_bf16", "sp_weno_dl")]
    print(f"Shu-Osher Nx={nx} L1(rho): fp64 sp_weno {err[('fp64', 'sp_weno')]:.4e}  "
          f"fp64 dl {err[('fp64', 'sp_weno_dl')]:.4e}  fp32 dl {e32:.4e}")
    assert e32 <= 1.5 * err[("fp64", "sp_weno_dl")]
    assert e32 <= 1.5 * err[("fp64", "sp_weno")]


def test_kh_fp32_dl_tracks_fp64_dl():
    out, viol = {}, {}
    for prec in ("fp64", "fp32_bf16"):
        d, p, _ = W.kh(128, prec, "sp_weno_dl", net(), final_time=1.0)
        s = run(d, p)
        st = s.status()
        assert st.code == 0
        viol[prec] = st.sign_violations
        assert abs(s.globals().time - 1.0) < 1e-12
        out[prec] = s.prim()[0, 0]
    # the FP64 form is the reference's network without a limiter and may break
    # the sign property; the FP32 form limits every face
    assert viol["fp32_bf16"] == 0
    print(f"KH 128^2 t=1: sign violations fp64 dl {viol['fp64']}, fp32 dl {viol['fp32_bf16']}")
    l1 = float(np.mean(np.abs(out["fp32_bf16"] - out["fp64"])))
    print(f"KH 128^2 t=1: L1(rho) fp32 dl - fp64 dl = {l1:.4e} (mean rho 1.5)")
    assert np.all(np.isfinite(out["fp32_bf16"])) and l1 < 0.05
