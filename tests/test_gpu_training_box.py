"""The network's training box and what the retrained network gains over plain
SP-WENO (the method without it).

The reference applies its network to every stencil
(enflo/src/reconstruct.cc:138-157).  Here a network can carry the box of the
inputs it was fitted on (descriptor nn_use_box / nn_feat_lo / nn_feat_hi,
filled from dspw_trainer_box after training); in the FP32 form a stencil whose
five network inputs fall outside that box is reconstructed by plain SP-WENO.
The reference's own training data is not in its repository, so the box the
GPU trainer records is the only definition of the training range."""
import numpy as np
import pytest

import oracle as O
from _common import net
from dspw import Solver, Trainer, make_desc, set_training_box, workloads as W, xavier_network
from dspw.capi import reconstruct_batch

pytestmark = pytest.mark.gpu


def _stencils(rng, n):
    x = rng.uniform(0, 2 * np.pi, (n, 1)) + rng.uniform(0.01, 0.6, (n, 1)) * np.arange(4)[None, :]
    u = np.sin(x) * rng.uniform(0.5, 3.0, (n, 1))
    u[n // 2:] = rng.normal(0, 1, (n - n // 2, 4))
    # no near-flat middle jumps: those take the network's own guard, not the box
    keep = np.abs(u[:, 2] - u[:, 1]) > 1e-3 * np.max(np.abs(u), axis=1)
    return u[keep]


def test_stencils_outside_the_box_take_sp_weno():
    rng = np.random.default_rng(31)
    u = _stencils(rng, 40000)
    feats = np.array([O.nn_features(s)[0] for s in u])
    lo, hi = np.quantile(feats, 0.15, axis=0), np.quantile(feats, 0.85, axis=0)
    d_nn = make_desc(recon="sp_weno_dl", precision="fp32_bf16", network=net())
    d_box = set_training_box(make_desc(recon="sp_weno_dl", precision="fp32_bf16", network=net()), lo, hi)
    d_sp = make_desc(recon="sp_weno", precision="fp32_bf16")
    l_nn, r_nn, _ = reconstruct_batch(d_nn, u)
    l_box, r_box, _ = reconstruct_batch(d_box, u)
    l_sp, r_sp, _ = reconstruct_batch(d_sp, u)
    # FP32 features on the device vs FP64 here: keep clear of the box faces
    m = 1e-3 * (hi - lo)
    inside = np.all((feats >= lo + m) & (feats <= hi - m), axis=1)
    outside = np.any((feats < lo - m) | (feats > hi + m), axis=1)
    assert inside.sum() > 200 and outside.sum() > 1000, (inside.sum(), outside.sum())
    scale = np.max(np.abs(u), axis=1)
    tol = 1e-6 * scale
    # inside: the network's reconstruction, as without a box
    assert np.all(np.abs(l_box - l_nn)[inside] <= tol[inside])
    assert np.all(np.abs(r_box - r_nn)[inside] <= tol[inside])
    # outside: plain SP-WENO's
    assert np.all(np.abs(l_box - l_sp)[outside] <= tol[outside])
    assert np.all(np.abs(r_box - r_sp)[outside] <= tol[outside])
    # and the two methods really differ there (the test would be empty otherwise)
    assert np.mean(np.abs(l_nn - l_sp)[outside] > 1e-4 * scale[outside]) > 0.3


def test_solver_with_the_trainer_box():
    """The box recorded by the trainer goes into the descriptor; a solver run
    with it is healthy, and a box that excludes every stencil turns the FP32
    DSP-WENO solver into the FP32 SP-WENO one."""
    W0, b0 = net()
    tr = Trainer((W0, b0), batch=4096, bf16=True)
    (d,), (p,), _ = W.kh(64, "fp64", "sp_weno", None)
    s = Solver(d)
    s.upload_prim(p)
    s.step(20)
    assert tr.collect(s, 200000) > 10000
    lo, hi = tr.box()
    _, fmax = tr.info()
    assert np.all(lo <= hi) and np.allclose(np.maximum(np.abs(lo), np.abs(hi)), fmax)
    assert -1.0 <= lo[0] and hi[1] <= 1.0 and lo[2] >= 0.0   # tanh features, absolute jumps
    (dd,), _, _ = W.kh(64, "fp32_bf16", "sp_weno_dl", (W0, b0))
    sb = Solver(set_training_box(dd, lo, hi))
    sb.upload_prim(p)
    sb.step(20)
    st = sb.status()
    assert st.code == 0 and st.sign_violations == 0
    # a box that holds every input: the same bits as no box at all
    (dw,), _, _ = W.kh(64, "fp32_bf16", "sp_weno_dl", (W0, b0))
    sw = Solver(set_training_box(dw, [-10.0] * 5, [10.0] * 5))
    sw.upload_prim(p)
    sw.step(20)
    (dn,), _, _ = W.kh(64, "fp32_bf16", "sp_weno_dl", (W0, b0))
    sn = Solver(dn)
    sn.upload_prim(p)
    sn.step(20)
    assert np.array_equal(sw.cons(), sn.cons())
    # an empty box: no face reaches the network's limiter, and the solution is
    # the FP32 SP-WENO one except at the no-jump faces, where the network path
    # keeps the reference's DSP-WENO guard (a zero jump below 4 FP32 ulps of
    # the values) and SP-WENO its own (below 1e-13)
    (de,), _, _ = W.kh(64, "fp32_bf16", "sp_weno_dl", (W0, b0))
    se = Solver(set_training_box(de, [9.0] * 5, [9.0] * 5))
    se.upload_prim(p)
    se.step(20)
    assert se.status().limiter_acts == 0
    (ds,), _, _ = W.kh(64, "fp32_bf16", "sp_weno", None)
    ss = Solver(ds)
    ss.upload_prim(p)
    ss.step(20)
    a, b, c = se.cons(), ss.cons(), sn.cons()
    d_sp, d_nn = np.max(np.abs(a - b)), np.max(np.abs(c - b))
    print(f"empty box vs SP-WENO {d_sp:.3e}, network vs SP-WENO {d_nn:.3e}")
    assert d_sp <= 5e-3 * np.max(np.abs(b))


def _collect(tr, max_pairs):
    """(stencil, plain SP-WENO interface value) pairs of GPU solver runs of the
    linear advection (config 1), Shu-Osher (config 2) and Kelvin-Helmholtz
    (config 3) problems."""
    total = 0
    nx = 400
    x = -np.pi + (np.arange(nx) + 0.5) * 2 * np.pi / nx
    s = Solver(make_desc(model="linadv", flux="lin_tecno4", recon="sp_weno", nx=nx, x=(-np.pi, np.pi), cfl=0.5,
                         final_time=0.5))
    s.upload_prim((np.sin(x) ** 4).reshape(1, 1, 1, nx))
    for _ in range(3):
        total += tr.collect(s, max_pairs // 9)
        s.step(10)
    (d,), (p,), _ = W.shu_osher(800, "fp64", "sp_weno", None)
    s = Solver(d)
    s.upload_prim(p)
    for _ in range(3):
        s.step(60)
        total += tr.collect(s, max_pairs // 9)
    (d,), (p,), _ = W.kh(128, "fp64", "sp_weno", None)
    s = Solver(d)
    s.upload_prim(p)
    for _ in range(3):
        s.step(40)
        total += tr.collect(s, max_pairs // 9)
    return total


def _linadv_l1(recon, network=None):
    nx = 200
    x = -np.pi + (np.arange(nx) + 0.5) * 2 * np.pi / nx
    d = make_desc(model="linadv", flux="lin_tecno4", recon=recon, nx=nx, x=(-np.pi, np.pi), cfl=0.5,
                  final_time=0.5, t_stamps=5, network=network)
    s = Solver(d)
    s.upload_prim((np.sin(x) ** 4).reshape(1, 1, 1, nx))
    s.run(chunk=32)
    return float(s.errors(np.sin(x - s.globals().time) ** 4)[0])


def _shu_osher_l1(ref, recon, network=None, n=400):
    (d,), (p,), _ = W.shu_osher(n, "fp64", recon, network)
    s = Solver(d)
    s.upload_prim(p)
    s.run(chunk=256)
    return float(np.mean(np.abs(s.prim()[0, 0, 0] - ref.reshape(n, -1).mean(axis=1))))


def test_retrained_network_against_plain_sp_weno():
    """The gain of the retrained network over the method without it.  Plain
    SP-WENO produced the training targets, so on held-out pairs it is the
    judge: its own error there is zero, and the network's held-out loss says
    how closely it follows SP-WENO.  On the solutions the comparison is made
    against exact (config 1) and converged (Shu-Osher, a 6400-cell FP64
    SP-WENO run averaged to 400 cells) references.  Asserted: the network
    learns (its held-out loss falls below the untrained network's) and its
    solutions stay within a factor of SP-WENO's; which method is more accurate
    is printed and recorded, whichever it is."""
    W0, b0 = xavier_network(6008)
    tr = Trainer((W0, b0), batch=8192, bf16=True, collect_stride=3)
    n = _collect(tr, 300000)
    assert n > 50000, n
    for _ in range(150):
        tr.epoch()
    W1, b1 = tr.params()
    held_untrained = Trainer((W0, b0), bf16=False, collect_stride=7)
    held_trained = Trainer((W1, b1), bf16=False, collect_stride=7)
    assert _collect(held_untrained, 60000) == _collect(held_trained, 60000)
    lu, lt = held_untrained.eval(), held_trained.eval()
    assert lt < lu, (lt, lu)
    c1_sp, c1_nn = _linadv_l1("sp_weno"), _linadv_l1("sp_weno_dl", (W1, b1))
    (d,), (p,), _ = W.shu_osher(6400, "fp64", "sp_weno", None)
    s = Solver(d)
    s.upload_prim(p)
    s.run(chunk=256)
    ref = s.prim()[0, 0, 0]
    so_sp, so_nn = _shu_osher_l1(ref, "sp_weno"), _shu_osher_l1(ref, "sp_weno_dl", (W1, b1))
    so_ship = _shu_osher_l1(ref, "sp_weno_dl", net())
    for v in (c1_sp, c1_nn, so_sp, so_nn, so_ship):
        assert np.isfinite(v)
    assert c1_nn < 3 * c1_sp and so_nn < 3 * so_sp
    print(f"held-out loss against SP-WENO targets: SP-WENO 0, untrained {lu:.3e}, retrained {lt:.3e}")
    print(f"config-1 L1 (exact): SP-WENO {c1_sp:.4e}, retrained DSP-WENO {c1_nn:.4e} "
          f"({'network' if c1_nn < c1_sp else 'SP-WENO'} more accurate)")
    print(f"Shu-Osher Nx=400 L1(rho): SP-WENO {so_sp:.4e}, retrained DSP-WENO {so_nn:.4e}, "
          f"shipped DSP-WENO {so_ship:.4e} ({'network' if so_nn < so_sp else 'SP-WENO'} more accurate)")
