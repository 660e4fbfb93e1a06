"""TEST INFRASTRUCTURE: float64 torch restatement of the reference trainer's
model and loss (DSP-WENO_trainer/DSP-WENO_network_trainer.py), the checker for
the GPU training kernels.

* MLP.forward (:63-91): 4 Linear layers 5->5 with ReLU between, softmax, convex
  combination of the vertex columns into C1/C2, weights (1-w1, w1, tw0, 1-tw0);
* inter_evaluation (:94-106) with sten = [[3/2,-1/2],[1/2,1/2],[-1/2,3/2]];
* loss = (MSE(left) + MSE(right)) / 2 (:404);
* torch.optim.Adam(lr, betas, weight_decay) (:353).

Features and vertices come from the oracle's restatement of the C++ forward's
preprocessing (or_nn_features), as the reference's data file carries them.
Samples with |u2 - u1| < 1e-15 (where the solver never calls the network)
contribute zero, and the means stay over the whole batch.
"""
from __future__ import annotations

import numpy as np

import oracle as O


def features(stencils):
    st = np.asarray(stencils, dtype=np.float64).reshape(-1, 4)
    n = len(st)
    F, VX, VY = np.zeros((n, 5)), np.zeros((n, 5)), np.zeros((n, 5))
    mask = np.zeros(n)
    for i in range(n):
        f, vx, vy = O.nn_features(st[i])
        ok = abs(st[i, 2] - st[i, 1]) >= 1e-15 and np.all(np.isfinite(f)) and np.all(np.isfinite(vx)) \
            and np.all(np.isfinite(vy))
        if ok:
            F[i], VX[i], VY[i], mask[i] = f, vx, vy, 1.0
    return F, VX, VY, mask


class TorchTrainer:
    def __init__(self, W, b, lr=1e-3, betas=(0.5, 0.9), weight_decay=1e-5, eps=1e-8):
        import torch
        self.torch = torch
        self.W = [torch.tensor(np.asarray(W[l], dtype=np.float64), requires_grad=True) for l in range(4)]
        self.b = [torch.tensor(np.asarray(b[l], dtype=np.float64), requires_grad=True) for l in range(4)]
        self.opt = torch.optim.Adam(self.W + self.b, lr=lr, betas=betas, weight_decay=weight_decay, eps=eps)

    def loss(self, stencils, targets):
        torch = self.torch
        F, VX, VY, mask = features(stencils)
        st = torch.tensor(np.asarray(stencils, dtype=np.float64).reshape(-1, 4))
        tg = torch.tensor(np.asarray(targets, dtype=np.float64).reshape(-1, 2))
        h = torch.tensor(F)
        for l in range(4):
            h = h @ self.W[l].T + self.b[l]
            if l < 3:
                h = torch.relu(h)
        s = torch.softmax(h, dim=1)
        C1 = (s * torch.tensor(VX)).sum(1)
        C2 = (s * torch.tensor(VY)).sum(1)
        w1 = 0.25 - 2 * C1
        tw0 = 0.25 - 2 * C2
        c = 0.5 * st[:, 1] + 0.5 * st[:, 2]
        bl = -0.5 * st[:, 0] + 1.5 * st[:, 1]
        br = 1.5 * st[:, 2] - 0.5 * st[:, 3]
        left = (1 - w1) * c + w1 * bl
        right = tw0 * br + (1 - tw0) * c
        m = torch.tensor(mask)
        n = len(mask)
        mse_l = ((left - tg[:, 0]) ** 2 * m).sum() / n
        mse_r = ((right - tg[:, 1]) ** 2 * m).sum() / n
        return (mse_l + mse_r) / 2

    def loss_grad(self, stencils, targets):
        for p in self.W + self.b:
            p.grad = None
        L = self.loss(stencils, targets)
        L.backward()
        gw = np.stack([p.grad.numpy() for p in self.W])
        gb = np.stack([p.grad.numpy() for p in self.b])
        return float(L.item()), gw, gb

    def step(self, stencils, targets):
        self.opt.zero_grad()
        L = self.loss(stencils, targets)
        L.backward()
        self.opt.step()
        return float(L.item())

    def params(self):
        return (np.stack([p.detach().numpy() for p in self.W]), np.stack([p.detach().numpy() for p in self.b]))
