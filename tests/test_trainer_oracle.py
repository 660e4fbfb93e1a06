"""The torch restatement of the reference trainer (oracle/trainer_oracle.py):
its gradients agree with central finite differences of its own loss."""
import numpy as np

from _common import net
from dspw import xavier_network
from trainer_oracle import TorchTrainer


def test_torch_trainer_gradcheck():
    rng = np.random.default_rng(0)
    st = np.sin(rng.uniform(0, 6, (64, 1)) + rng.uniform(0.05, 0.4, (64, 1)) * np.arange(4))
    st[:8] = rng.normal(0, 1, (8, 4))
    tg = np.stack([st[:, 1] + 0.4 * (st[:, 2] - st[:, 1]), st[:, 2] - 0.4 * (st[:, 2] - st[:, 1])], 1)
    W, b = xavier_network(3)
    tt = TorchTrainer(W, b)
    L, gw, gb = tt.loss_grad(st, tg)
    h = 1e-6
    for (l, j, k) in [(0, 0, 0), (1, 2, 3), (2, 4, 1), (3, 1, 4)]:
        Wp = W.copy(); Wp[l, j, k] += h
        Wm = W.copy(); Wm[l, j, k] -= h
        fd = (TorchTrainer(Wp, b).loss(st, tg).item() - TorchTrainer(Wm, b).loss(st, tg).item()) / (2 * h)
        assert abs(fd - gw[l, j, k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
    assert np.isfinite(L) and L > 0


def test_torch_trainer_shipped_network_loss_finite():
    rng = np.random.default_rng(1)
    st = rng.normal(0, 1, (32, 4))
    tg = st[:, 1:3].copy()
    L, gw, gb = TorchTrainer(*net()).loss_grad(st, tg)
    assert np.isfinite(L) and np.all(np.isfinite(gw)) and np.all(np.isfinite(gb))
