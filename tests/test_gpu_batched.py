"""Batched problems of uneven size and different models in one handle: the
isentropic-vortex OOC mesh list plus many independent 1-D Burgers problems
(the composition of the batched workload, at reduced sizes), advanced together
by ``dspw_run`` (one launch per sweep direction over the flat task index, one
CUDA graph per step), each problem with its own dt, time and finish.

* FP64 plain form: every checked problem's final state equals the oracle's run
  of that problem alone (1e-12 per cell), and each problem ends at its own
  final time;
* FP32 + BF16 DSP-WENO form: every problem finishes, no sign violations, and
  the L1 density difference to the FP64 oracle's DSP-WENO run stays small;
* OOC: the vortex levels of the batch converge at third order or better.
"""
import math

import numpy as np
import pytest

import oracle as O
from _common import net
from dspw import Solver, workloads as W
from test_gpu_parity import assert_state_close

pytestmark = pytest.mark.gpu

LEVELS = (16, 32, 64)
VORTEX_T = 1.0


def small_batch(precision, recon, nburgers=24, seed=11):
    return W.batched(precision, recon, net(), levels=LEVELS, nburgers=nburgers, burgers_nx=(100, 400), seed=seed,
                     vortex_time=VORTEX_T, burgers_time=0.5)


def run_batch(descs, prims):
    s = Solver(descs)
    for p, a in enumerate(prims):
        s.upload_prim(a, p)
    steps = s.run(chunk=64)
    return s, steps


def oracle_final(d, prim):
    o = O.Oracle(d)
    o.set_prim(prim)
    o.step(1 << 30)
    return o


def test_batch_fp64_matches_oracle_per_problem():
    descs, prims, _ = small_batch("fp64", "sp_weno")
    s, _ = run_batch(descs, prims)
    st = s.status()
    assert st.code == 0 and st.sign_violations == 0
    picks = list(range(len(LEVELS))) + [len(LEVELS), len(LEVELS) + 7, len(descs) - 1]
    for p in picks:
        o = oracle_final(descs[p], prims[p])
        t, it, _ = o.time()
        g = s.globals(p)
        assert g.iter == it and abs(g.time - t) <= 1e-12 * t and abs(t - descs[p].final_time) <= 1e-12 * t
        assert_state_close(s.cons(p), o.cons(), what=f"problem {p}")


def test_batch_fp32_dl_completes_and_tracks_fp64():
    descs, prims, _ = small_batch("fp32_bf16", "sp_weno_dl")
    s, _ = run_batch(descs, prims)
    st = s.status()
    assert st.code == 0 and st.nonfinite_cells == 0 and st.nonpositive_cells == 0
    assert st.sign_violations == 0 and st.faces_checked > 0
    d64, _, _ = small_batch("fp64", "sp_weno_dl")
    for p in range(len(descs)):
        g = s.globals(p)
        assert abs(g.time - descs[p].final_time) <= 1e-12 * descs[p].final_time, p
    for p in (0, len(LEVELS) - 1, len(LEVELS), len(descs) - 1):
        ref = oracle_final(d64[p], prims[p]).prim()[0]
        got = s.prim(p)[0]
        l1 = np.mean(np.abs(got - ref)) / np.mean(np.abs(ref))
        assert l1 < 2e-3, (p, l1)


def test_vortex_ooc_in_batch():
    descs, prims, _ = small_batch("fp64", "sp_weno", nburgers=4)
    s, _ = run_batch(descs, prims)
    errs = []
    for p, n in enumerate(LEVELS):
        g = s.globals(p)
        exact = W.vortex_exact_density(n, g.time)
        errs.append(s.errors(exact, comp=0, p=p)[0])
    rates = [math.log(errs[i - 1] / errs[i], 2) for i in range(1, len(errs))]
    assert errs[-1] < errs[0] and rates[-1] > 2.5, (errs, rates)
