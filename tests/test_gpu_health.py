"""Device health reported by the stepping calls.

FV::run never looks at the state it produces (the reference detects no NaN).
Here every step's last stage counts non-finite and non-positive cells on the
device, and dspw_step / dspw_stage return the first such error after their
final synchronisation, so a caller that only steps still learns that the run
broke down.  The failures are made by plain arithmetic: valid states stepped
far beyond their stability limit overflow to Inf / NaN.  Nothing faults."""
import math

import numpy as np
import pytest

from dspw import DspwError, Solver, make_desc, workloads as W
from _common import net

pytestmark = pytest.mark.gpu

NONFINITE, NONPOSITIVE = 3, 4


def sin4(nx):
    x = -math.pi + (np.arange(nx) + 0.5) * (2 * math.pi / nx)
    return (np.sin(x) ** 4).reshape(1, 1, 1, nx)


@pytest.mark.parametrize("precision", ["fp64", "fp32_bf16"])
def test_step_returns_nonfinite_of_an_unstable_run(precision):
    """Linear advection at CFL 40 grows until it overflows: dspw_step returns
    DSPW_ERR_NONFINITE, the status counters agree, and after they are read a
    fresh upload steps cleanly again."""
    d = make_desc(model="linadv", flux="lin_tecno4", recon="sp_weno", nx=64, x=(-math.pi, math.pi),
                  cfl=40.0, final_time=1e9, precision=precision)
    s = Solver(d)
    s.upload_prim(sin4(64))
    code = 0
    for _ in range(200):
        try:
            s.step(5)
        except DspwError as e:
            code = e.code
            break
    assert code == NONFINITE
    st = s.status()
    assert st.code == NONFINITE and st.nonfinite_cells > 0
    # dspw_last_status cleared the word: a valid state at a stable CFL steps on
    d.cfl = 0.5
    s2 = Solver(d)
    s2.upload_prim(sin4(64))
    s2.step(5)
    assert s2.status().code == 0


def test_step_and_stage_return_euler_breakdown():
    """2-D Euler (Kelvin-Helmholtz) with a fixed dt 50 times the CFL step:
    density or pressure leaves the positive range or overflows, and both
    dspw_step and the last dspw_stage of a step report it."""
    (d,), (p,), _ = W.kh(32, "fp64", "sp_weno", net())
    dt = 50 * 0.4 / 32 / 2.37
    s = Solver(d)
    s.upload_prim(p)
    code = 0
    for _ in range(50):
        try:
            s.step(1, dt)
        except DspwError as e:
            code = e.code
            break
    assert code in (NONFINITE, NONPOSITIVE)
    assert s.status().code == code
    s = Solver(d)
    s.upload_prim(p)
    code = 0
    for _ in range(50):
        try:
            for rk in range(3):
                s.stage(rk, dt)
        except DspwError as e:
            code = e.code
            assert rk == 2   # the health epilogue runs in the stage that yields U^(n+1)
            break
    assert code in (NONFINITE, NONPOSITIVE)
