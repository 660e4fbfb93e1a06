"""The network measurement kernels (libdspw_netbench.so): the sweep kernels'
mma.sync form and the tcgen05 form evaluate the shipped network on the same
inputs, and both agree with an FP64 evaluation of the same BF16-rounded
operands (FP32 accumulation in another order; a hidden activation whose FP32
value rounds to the other BF16 neighbour moves a logit by about 2^-8 of a
weight times an activation)."""
import numpy as np
import pytest

from _common import NET_FILE
from dspw import load_network_file
from dspw import netbench as NB

pytestmark = pytest.mark.gpu

NET = load_network_file(NET_FILE)


@pytest.mark.parametrize("form", list(NB.FORMS))
@pytest.mark.parametrize("ntile,reps,grid", [(40, 3, 0), (37, 2, 7), (1, 1, 1)])
def test_form_matches_fp64_evaluation(form, ntile, reps, grid):
    W, b = NET
    out, ms, used, _ = NB.run(form, W, b, ntile, reps, grid=grid)
    assert ms > 0
    if grid:
        assert used == min(grid, ntile)
    ref = NB.cpu_logits(W, b, np.arange(ntile * NB.TILE), reps)
    err = np.abs(out - ref) / np.maximum(np.abs(ref), 1.0)
    assert np.all(np.isfinite(out))
    assert err.max() < 2e-2, (form, float(err.max()))
    assert np.mean(err < 1e-5) > 0.99, (form, float(np.mean(err < 1e-5)))


def test_forms_agree():
    W, b = NET
    a, _, _, _ = NB.run("mma_sync", W, b, 50, 4)
    c, _, _, _ = NB.run("tcgen05", W, b, 50, 4)
    d = np.abs(a - c) / np.maximum(np.abs(a), 1.0)
    assert d.max() < 2e-2 and np.mean(d < 1e-5) > 0.99, (float(d.max()), float(np.mean(d < 1e-5)))
