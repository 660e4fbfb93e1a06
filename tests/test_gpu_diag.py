"""Per-step diagnostics on the GPU (dspw_diag_*): the rows of total entropy,
KE, KE dissipation (pressure and viscous-stress parts), enstrophy and residual
norms that the reference's FV::run computes every step (compute_global,
compute_residual_norm, find_vorticity).

* FP64: every row of every golden case equals the reference's row
  (``diag.npz``, produced by the reference's own functions) to rounding: the
  device sums in another order than the reference's loops.
* The recording does not change the solution (bit-identical state).
* Batched problems record one row each per step, equal to their single runs.
* FP32: rows track the FP64 ones.
* The ring: dspw_step drains it every ``capacity`` steps; stages issued one by
  one do not, and the rows they overwrite are counted as dropped.
"""
import numpy as np
import pytest

import oracle as O
from _common import desc_from_cfg, load, run_cases
from dspw import Solver
from dspw.capi import DIAG_COLS, DIAG_NAMES

pytestmark = pytest.mark.gpu

DIAG = [c for c in run_cases() if f"{c[0]}|rows" in load("diag.npz")]
# relative tolerance against the column's scale (sums of O(N) terms in another order)
RTOL = 1e-11


def _solver(case, precision=None, capacity=64):
    name, kind, cfg, nsteps, fixed_dt = case
    p0 = load("runs.npz")[f"{name}|prim0"]
    _, nz, ny, nx = p0.shape
    over = {} if precision is None else {"precision": precision}
    d = desc_from_cfg(cfg, nx, ny, nz, **over)
    s = Solver(d)
    s.upload_prim(p0)
    if capacity:
        s.diag_enable(capacity)
    return s, d, p0


def assert_rows_close(got, ref, rtol=RTOL, what=""):
    assert got.shape == ref.shape, (what, got.shape, ref.shape)
    np.testing.assert_array_equal(got[:, 0], ref[:, 0], err_msg=f"{what} iter")
    for c in range(1, DIAG_COLS):
        scale = np.max(np.abs(ref[:, c]))
        tol = rtol * max(scale, 1e-300)
        err = np.max(np.abs(got[:, c] - ref[:, c]))
        assert err <= tol, f"{what} column {DIAG_NAMES[c]}: max |diff| {err:.3e} > {tol:.3e} (scale {scale:.3e})"


@pytest.mark.parametrize("case", DIAG, ids=lambda c: c[0])
def test_rows_match_reference(case):
    name, kind, cfg, nsteps, fixed_dt = case
    ref = load("diag.npz")[f"{name}|rows"]
    s, _, _ = _solver(case)
    s.step(len(ref), fixed_dt)
    got, dropped = s.diag_rows()
    assert dropped == 0
    assert_rows_close(got, ref, what=name)
    # read rows are removed
    again, _ = s.diag_rows()
    assert again.shape == (0, DIAG_COLS)


@pytest.mark.parametrize("name", ["kh_sp_weno_dl", "tgv_ns", "burgers_wall_dl"])
def test_recording_leaves_solution_unchanged(name):
    case = next(c for c in DIAG if c[0] == name)
    a, _, _ = _solver(case, capacity=8)
    b, _, _ = _solver(case, capacity=0)
    for s in (a, b):
        s.step(5, case[4])
    np.testing.assert_array_equal(a.cons(), b.cons())
    assert a.globals().time == b.globals().time


def test_batch_rows_equal_single_runs():
    names = ["kh_sp_weno", "wall2d", "burgers_wenoc", "tgv_ns_kep", "shuosher_sp_weno"]
    cases = [next(c for c in DIAG if c[0] == n) for n in names]
    g = load("runs.npz")
    descs, prims = [], []
    for name, kind, cfg, nsteps, fixed_dt in cases:
        p0 = g[f"{name}|prim0"]
        _, nz, ny, nx = p0.shape
        descs.append(desc_from_cfg(cfg, nx, ny, nz))
        prims.append(p0)
    # mixed models cannot share a handle with an NS problem; split by viscosity
    groups = [[i for i, c in enumerate(cases) if c[2].get("model") in ("ns_es", "ns_kep")],
              [i for i, c in enumerate(cases) if c[2].get("model") not in ("ns_es", "ns_kep")]]
    for grp in groups:
        s = Solver([descs[i] for i in grp])
        for q, i in enumerate(grp):
            s.upload_prim(prims[i], q)
        s.diag_enable(16)
        s.step(4)
        for q, i in enumerate(grp):
            got, _ = s.diag_rows(q)
            ref = load("diag.npz")[f"{cases[i][0]}|rows"][:4]
            assert_rows_close(got, ref, what=f"batch {cases[i][0]}")


@pytest.mark.parametrize("name", ["kh_sp_weno_dl", "tgv_ns", "shuosher_sp_weno", "burgers_wenoc"])
def test_fp32_rows_track_fp64(name):
    case = next(c for c in DIAG if c[0] == name)
    ref = load("diag.npz")[f"{name}|rows"]
    s, _, _ = _solver(case, precision="fp32_bf16")
    s.step(len(ref), case[4])
    got, _ = s.diag_rows()
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got[:, 0], ref[:, 0])
    # time (the CFL dt of an FP32 state), entropy and KE to FP32 rounding and
    # the reconstruction difference; the dissipation rates and residual norms
    # are differences of fluxes: on the KH shear layer the FP32 form's limited
    # BF16 network (the FP64 form runs the reference's unlimited one) moves
    # them by several percent (measured 5.5e-2 and 7.6e-2 after 6 steps), on
    # smooth flows by 1e-2 at most
    bad = []
    for c, tol in ((1, 1e-5), (2, 5e-5), (3, 1e-4), (4, 0.1), (5, 0.05), (6, 1e-3), (7, 0.1), (11, 0.1)):
        scale = np.max(np.abs(ref[:, c]))
        if scale == 0:
            continue
        err = np.max(np.abs(got[:, c] - ref[:, c])) / scale
        print(f"{name} {DIAG_NAMES[c]}: relative error {err:.2e} (bound {tol:.0e})")
        if err > tol:
            bad.append((DIAG_NAMES[c], err))
    assert not bad, (name, bad)


def test_ring_drains_and_counts_drops():
    case = next(c for c in DIAG if c[0] == "shuosher_sp_weno")
    s, d, p0 = _solver(case, capacity=4)
    s.step(10)                           # drained every 4 steps
    rows, dropped = s.diag_rows()
    assert rows.shape[0] == 10 and dropped == 0
    np.testing.assert_array_equal(rows[:, 0], np.arange(10))
    # the oracle's rows of the same 10 steps
    o = O.Oracle(d)
    o.set_prim(p0)
    assert_rows_close(rows, o.step_diag(10), what="oracle 10 steps")
    # single stages do not drain: 6 steps into a ring of 4 keep the newest 4
    import ctypes as C
    from dspw.capi import lib
    for _ in range(6):
        for rk in range(3):
            assert lib().dspw_stage(s.h, rk, C.c_double(0.0)) == 0
    rows, dropped = s.diag_rows()
    assert dropped == 2
    np.testing.assert_array_equal(rows[:, 0], np.arange(12, 16))
    # disabling stops the recording
    s.diag_enable(0)
    s.step(2)
    rows, _ = s.diag_rows()
    assert rows.shape[0] == 0


def test_diagnostics_and_globals_are_bitwise_reproducible():
    """The device sums run in a fixed order (block partials, then a fixed
    fold), so two runs of the same batch give the same bits: a 2-D Euler
    problem beside uneven Burgers problems, whose cells make blocks straddle
    problem boundaries."""
    from dspw import make_desc, workloads as W

    def run():
        (dk,), (pk,), _ = W.kh(96, "fp64", "sp_weno", None)
        descs, prims = [dk], [pk]
        rng = np.random.default_rng(7)
        for nx in (100, 257, 3001, 5, 640):
            descs.append(make_desc(model="burgers", flux="bur_tecno4", recon="sp_weno", nx=nx, x=(-np.pi, np.pi),
                                   final_time=1e9))
            prims.append(W.burgers_fourier(nx, rng))
        s = Solver(descs)
        for k, p in enumerate(prims):
            s.upload_prim(p, k)
        s.diag_enable(16)
        s.step(6)
        rows = [s.diag_rows(k)[0] for k in range(len(descs))]
        g = [s.globals(k) for k in range(len(descs))]
        return rows, [(x.total_entropy, x.kinetic_energy, tuple(x.conserved)) for x in g]

    r1, g1 = run()
    r2, g2 = run()
    for a, b in zip(r1, r2):
        assert a.shape[0] == 6 and np.array_equal(a, b)
    assert g1 == g2
