"""FP64 parity at the benchmark's grid sizes.

The golden runs pin the kernels on 16^2 to 32^2 grids.  The benchmark times
the specialised 2-D kepes_tecno4 kernels on 2048^2, where every y launch works
on 16-byte aligned cp.async tiles of 256 column groups and 69 segments per
column: these tests run that code on 512^2 and 2048^2 Kelvin-Helmholtz states
(seeded noise, periodic) in the FP64 plain form with SP-WENO and with the
DSP-WENO network, and compare every cell with the CPU oracle (the reference's
arithmetic restated in C) after a fixed number of steps of a fixed dt, at
1e-12 of the component's scale.  The oracle runs in spawned worker processes,
in parallel."""
import concurrent.futures as cf
import multiprocessing as mp

import numpy as np
import pytest

from _common import net, oracle_kh_cons
from dspw import Solver, workloads as W

pytestmark = pytest.mark.gpu

# (grid, reconstruction, steps); dt is 0.9 x the CFL 0.4 step of the initial
# state (max |u| + c = 0.5 + sqrt(1.4 * 2.5) = 2.37)
CASES = [(512, "sp_weno", 3), (512, "sp_weno_dl", 3), (2048, "sp_weno", 1), (2048, "sp_weno_dl", 1)]
RTOL = 1e-12


def dt_of(n):
    return 0.9 * 0.4 * (1.0 / n) / 2.37


@pytest.fixture(scope="module")
def oracle_states():
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=len(CASES), mp_context=ctx) as ex:
        futs = {c: ex.submit(oracle_kh_cons, c[0], c[1], c[2], dt_of(c[0])) for c in CASES}
        return {c: f.result() for c, f in futs.items()}


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"kh{c[0]}_{c[1]}")
def test_kh_fp64_matches_oracle_at_bench_size(case, oracle_states):
    n, recon, steps = case
    (d,), (p,), _ = W.kh(n, "fp64", recon, net(), seed=12345)
    s = Solver(d)
    s.upload_prim(p)
    s.step(steps, dt_of(n))
    got = s.cons()[[0, 1, 2, 4]]
    ref = oracle_states[case][[0, 1, 2, 4]]
    assert got.shape == ref.shape == (4, 1, n, n)
    for c in range(4):
        scale = np.max(np.abs(ref[c]))
        err = np.abs(got[c] - ref[c])
        bad = err > RTOL * (np.abs(ref[c]) + scale)
        assert not bad.any(), (f"kh{n} {recon} comp {c}: {int(bad.sum())} of {bad.size} cells off, max "
                               f"{np.max(err) / scale:.3e} of the scale")
    st = s.status()
    assert st.code == 0 and st.nonfinite_cells == 0 and st.faces_checked > 0
    g = s.globals()
    assert g.iter == steps and abs(g.time - steps * dt_of(n)) <= 1e-15 * steps
