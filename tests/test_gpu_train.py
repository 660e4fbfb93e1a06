"""GPU training kernels (dsp-weno_b200/csrc/dspw_train.cu) against the torch
float64 restatement of the reference trainer, GPU data collection from plain
SP-WENO runs, and what the trained network gains over the network it started
from."""
import numpy as np
import pytest

from _common import net
from dspw import Solver, Trainer, make_desc, xavier_network
from trainer_oracle import TorchTrainer

pytestmark = pytest.mark.gpu


def _data(rng, n):
    x0 = rng.uniform(0, 2 * np.pi, (n, 1))
    dx = rng.uniform(0.02, 0.5, (n, 1))
    st = np.sin(x0 + dx * np.arange(4)) * rng.uniform(0.5, 2.0, (n, 1))
    st[: n // 5] = rng.normal(0, 1, (n // 5, 4))
    st[n // 5: n // 5 + 4] = st[n // 5: n // 5 + 4, 1:2]   # flat stencils (|u2-u1| = 0): excluded
    xf = x0 + 1.5 * dx   # exact interface value of the smooth part
    amp = np.linalg.norm(st, axis=1, keepdims=True) * 0 + 1
    tg = np.concatenate([np.sin(xf), np.sin(xf)], 1) * amp
    tg[: n // 5] = st[: n // 5, 1:3]
    return st, tg


def test_loss_and_gradients_match_torch_fp64():
    rng = np.random.default_rng(5)
    st, tg = _data(rng, 3000)
    W, b = xavier_network(6008)
    tr = Trainer((W, b), bf16=False)
    L, gw, gb = tr.loss_grad(st, tg)
    Lt, gwt, gbt = TorchTrainer(W, b).loss_grad(st, tg)
    assert abs(L - Lt) <= 1e-5 * abs(Lt)
    scale = max(np.max(np.abs(gwt)), np.max(np.abs(gbt)))
    assert np.max(np.abs(gw - gwt)) <= 2e-5 * scale, np.max(np.abs(gw - gwt)) / scale
    assert np.max(np.abs(gb - gbt)) <= 2e-5 * scale


def test_adam_steps_match_torch():
    rng = np.random.default_rng(6)
    st, tg = _data(rng, 1024)
    W, b = xavier_network(11)
    tr = Trainer((W, b), batch=1024, bf16=False)
    tr.set_data(st, tg)
    tt = TorchTrainer(W, b)
    for _ in range(5):
        lg = tr.epoch()
        lt = tt.step(st, tg)
        assert abs(lg - lt) <= 1e-4 * abs(lt)
    Wg, bg = tr.params()
    Wt, bt = tt.params()
    assert np.max(np.abs(Wg - Wt)) < 1e-5 and np.max(np.abs(bg - bt)) < 1e-5


def _collect(tr, max_pairs):
    """Stencils and plain SP-WENO targets from GPU solver runs: linear
    advection (config 1), Shu-Osher (config 2 IC), Kelvin-Helmholtz (config 3)."""
    total = 0
    nx = 400
    x = -np.pi + (np.arange(nx) + 0.5) * 2 * np.pi / nx
    s = Solver(make_desc(model="linadv", flux="lin_tecno4", recon="sp_weno", nx=nx, x=(-np.pi, np.pi), cfl=0.5,
                         final_time=0.5))
    s.upload_prim((np.sin(x) ** 4).reshape(1, 1, 1, nx))
    for _ in range(3):
        total += tr.collect(s, max_pairs // 9)
        s.step(10)
    nx = 800
    x = -5 + (np.arange(nx) + 0.5) * 10 / nx
    p = np.zeros((5, 1, 1, nx))
    p[0, 0, 0] = np.where(x < -4, 3.857143, 1 + 0.2 * np.sin(5 * x))
    p[1, 0, 0] = np.where(x < -4, 2.629369, 0.0)
    p[4, 0, 0] = np.where(x < -4, 10.33333, 1.0)
    s = Solver(make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=nx, x=(-5, 5), cfl=0.4,
                         final_time=1.8, bc=["neumann", "neumann", "periodic", "periodic", "periodic", "periodic"]))
    s.upload_prim(p)
    for _ in range(3):
        s.step(60)
        total += tr.collect(s, max_pairs // 9)
    n = 128
    xx = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(xx, xx)
    inner = np.abs(Y - 0.5) < 0.25
    p = np.zeros((5, 1, n, n))
    p[0, 0] = np.where(inner, 2.0, 1.0)
    p[1, 0] = np.where(inner, 0.5, -0.5)
    p[2, 0] = 0.01 * np.sin(4 * np.pi * X)
    p[4, 0] = 2.5
    s = Solver(make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=n, ny=n, cfl=0.4))
    s.upload_prim(p)
    for _ in range(3):
        s.step(40)
        total += tr.collect(s, max_pairs // 9)
    return total


def _linadv_l1(network):
    nx = 200
    x = -np.pi + (np.arange(nx) + 0.5) * 2 * np.pi / nx
    d = make_desc(model="linadv", flux="lin_tecno4", recon="sp_weno_dl", nx=nx, x=(-np.pi, np.pi), cfl=0.5,
                  final_time=0.5, t_stamps=5, network=network)
    s = Solver(d)
    s.upload_prim((np.sin(x) ** 4).reshape(1, 1, 1, nx))
    s.run(chunk=32)
    return s.errors(np.sin(x - s.globals().time) ** 4)[0]


def test_collect_train_and_gain():
    """Retrain from a random (Xavier, seed 6008) network on stencil/target pairs
    that plain SP-WENO runs produce on the GPU (config-1, -2 and -3 problems).
    The gain over the network it started from is measured the way the task
    defines it, with plain SP-WENO as the judge of the reconstruction error:
    the training loss halves and the error on held-out pairs of the same runs
    drops.  The config-1 L1 errors with both networks are printed; on this
    smooth problem DSP-WENO's feasible region shrinks with the stencil's jumps,
    so the network changes the L1 error by a few percent only."""
    import oracle as O
    W0, b0 = xavier_network(6008)
    tr = Trainer((W0, b0), batch=8192, bf16=True, collect_stride=3)
    n = _collect(tr, 300000)
    assert n > 50000, n
    ns, fmax = tr.info()
    assert ns == n and np.all(np.isfinite(fmax))
    losses = [tr.epoch() for _ in range(120)]
    assert losses[-1] < 0.5 * losses[0], losses[::20]
    W1, b1 = tr.params()
    # held-out pairs: other samples of the same runs (another sampling stride),
    # plain SP-WENO's interface values as the judge
    before = Trainer((W0, b0), bf16=False, collect_stride=7)
    after = Trainer((W1, b1), bf16=False, collect_stride=7)
    assert _collect(before, 60000) == _collect(after, 60000)
    l_before, l_after = before.eval(), after.eval()
    assert l_after < l_before, (l_after, l_before)
    # config-1 L1 with both networks (reported, not a pass criterion)
    l1_untrained = _linadv_l1((W0, b0))
    l1_trained = _linadv_l1((W1, b1))
    assert np.isfinite(l1_trained) and l1_trained < 2 * l1_untrained
    print(f"train loss {losses[0]:.3e} -> {losses[-1]:.3e}")
    print(f"gain: held-out loss {l_before:.3e} -> {l_after:.3e}; config-1 L1 {l1_untrained:.3e} -> {l1_trained:.3e}")


def test_retrain_on_two_million_pairs():
    """The retraining set of the north-star size: 2 M (stencil, SP-WENO target)
    pairs collected on the GPU from plain SP-WENO runs of the scalar, 1-D and
    2-D problems, trained with FP32 master weights, BF16 compute, Adam and
    batch 8192.  Epoch time is reported; the loss must fall."""
    import time
    from dspw import workloads as W

    W0, b0 = xavier_network(6008)
    tr = Trainer((W0, b0), batch=8192, bf16=True, collect_stride=1)
    total = 0
    nx = 4000
    x = -np.pi + (np.arange(nx) + 0.5) * 2 * np.pi / nx
    s = Solver(make_desc(model="linadv", flux="lin_tecno4", recon="sp_weno", nx=nx, x=(-np.pi, np.pi), cfl=0.5,
                         final_time=0.5))
    s.upload_prim((np.sin(x) ** 4).reshape(1, 1, 1, nx))
    total += tr.collect(s, 100_000)
    d, p, _ = W.shu_osher(25600, "fp64", "sp_weno", None)
    s = Solver(d)
    s.upload_prim(p[0])
    for _ in range(4):
        s.step(200)
        total += tr.collect(s, 100_000)
    d, p, _ = W.kh(512, "fp64", "sp_weno", None)
    s = Solver(d)
    s.upload_prim(p[0])
    s.step(100)
    total += tr.collect(s, 2_000_000 - total)
    assert total >= 1_900_000, total
    losses, times = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        losses.append(tr.epoch())
        times.append(time.perf_counter() - t0)
    assert losses[-1] < losses[0], losses
    print(f"2M-pair retraining: {total} pairs, epoch {min(times) * 1e3:.1f} ms "
          f"({total / min(times) / 1e6:.1f} M samples/s), loss {losses[0]:.3e} -> {losses[-1]:.3e}")
