"""Face-level parity of the GPU reconstruction (dspw_reconstruct_batch runs the
same device code as the stage kernels) against the oracle and the reference's
golden vectors: SP-WENO / SP-WENOc / corr2 and DSP-WENO in FP64 (1e-13
relative), and in the FP32 form with the BF16 tensor-core network (bounded by
BF16/FP32 rounding) including the exact sign property."""
import numpy as np
import pytest

import oracle as O
from _common import load, net
from dspw import make_desc
from dspw.capi import reconstruct_batch

pytestmark = pytest.mark.gpu


def stencils():
    g = load("recon.npz")
    return g


@pytest.mark.parametrize("recon,corr", [("sp_weno", 0), ("sp_wenoc", 1), ("sp_weno_corr2", 2)])
def test_sp_weno_fp64_golden(recon, corr):
    g = stencils()
    d = make_desc(recon=recon, precision="fp64")
    l, r, _ = reconstruct_batch(d, g["U"])
    for got, ref in ((l, g[f"spw{corr}_l"]), (r, g[f"spw{corr}_r"])):
        err = np.abs(got - ref) / (np.abs(ref) + 1e-300)
        assert np.max(np.where(np.abs(ref) > 1e-300, err, np.abs(got))) < 1e-13


def test_dsp_weno_fp64_golden():
    g = stencils()
    d = make_desc(recon="sp_weno_dl", precision="fp64", network=net())
    l, r, _ = reconstruct_batch(d, g["U"])
    m = g["nn_mask"]
    for got, ref in ((l, g["nn_l"]), (r, g["nn_r"])):
        scale = np.abs(ref[m]) + np.max(np.abs(g["U"][m]), axis=1) * 1e-3
        assert np.max(np.abs(got[m] - ref[m]) / scale) < 1e-12
    assert np.all(l[~m] == 0) and np.all(r[~m] == 0)


def _smooth_and_rough(rng, n):
    x = rng.uniform(0, 2 * np.pi, (n, 1)) + rng.uniform(0.005, 0.3, (n, 1)) * np.arange(4)[None, :]
    u = np.sin(x) * rng.uniform(0.5, 3.0, (n, 1))
    u[n // 2:] = rng.normal(0, 1, (n - n // 2, 4))
    return u


def test_sp_weno_fp32_close():
    rng = np.random.default_rng(1)
    u = _smooth_and_rough(rng, 20000)
    d = make_desc(recon="sp_weno", precision="fp32_bf16")
    l, r, _ = reconstruct_batch(d, u)
    lo = np.array([O.sp_weno(x, 0)[0] for x in u])
    ro = np.array([O.sp_weno(x, 0)[1] for x in u])
    scale = np.max(np.abs(u), axis=1)
    # FP32 rounding; far from region boundaries the weights agree
    assert np.median(np.abs(l - lo) / scale) < 1e-6
    assert np.quantile(np.abs(r - ro) / scale, 0.99) < 1e-4


def test_dsp_weno_fp32_bf16_close_and_sign_preserving():
    rng = np.random.default_rng(2)
    u = _smooth_and_rough(rng, 20000)
    d = make_desc(recon="sp_weno_dl", precision="fp32_bf16", network=net())
    l, r, acts = reconstruct_batch(d, u)
    d64 = make_desc(recon="sp_weno_dl", precision="fp64", network=net())
    lo = np.zeros(len(u)); ro = np.zeros(len(u))
    for i, x in enumerate(u):
        if abs(x[2] - x[1]) >= 1e-15:
            lo[i], ro[i] = O.nn_forward(d64, x)
    scale = np.max(np.abs(u), axis=1)
    errl = np.abs(l - lo) / scale
    errr = np.abs(r - ro) / scale
    # BF16 network (8-bit mantissa) moves the convex weights by ~1e-2 at most
    assert np.quantile(errl, 0.99) < 2e-2 and np.quantile(errr, 0.99) < 2e-2, (np.quantile(errl, 0.99), acts)
    # sign property holds exactly after the limiter
    jump_rec = r - l
    jump_cell = u[:, 2] - u[:, 1]
    assert np.sum(jump_rec * jump_cell < 0) == 0
    assert acts <= len(u) // 100
