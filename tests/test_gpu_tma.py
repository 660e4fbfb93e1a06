"""The tile variants of the specialised y / z sweeps against 8-column tiles
staged by per-thread cp.async copies: TMA staging (tile_staging 2) and narrow
tiles of 4 columns (tile_staging 3, k_sweep_narrow).  Every variant stages the
same rows and runs the same arithmetic per face and cell, so the FP64 cases
agree bit for bit and the FP32 ones to rounding: periodic wrap, walls and
neumann faces (whose ghost rows lie outside the tensor map and are patched
after the box load), partial last segments and partial column groups, several
problems per kernel class (tensor maps per problem), 3-D (the z sweep), FP64
and FP32 + BF16 DSP-WENO, a slab with halo faces, and the residual evaluation
of the tuner."""
import numpy as np
import pytest

from _common import net
from dspw import Solver, make_desc, workloads as W

pytestmark = pytest.mark.gpu


def _bump(nx, ny, nz=1):
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    p = np.zeros((5, nz, ny, nx))
    p[0] = 1.0 + 0.5 * np.exp(-40 * ((X - 0.4) ** 2 + (Y - 0.6) ** 2 + (Z - 0.5) ** 2))
    p[1] = 0.3
    p[2] = -0.2
    if nz > 1:
        p[3] = 0.1
    p[4] = 1.0 + 0.3 * np.exp(-30 * ((X - 0.5) ** 2 + (Y - 0.45) ** 2))
    return p


def _run(descs, prims, steps, staging):
    for d in descs:
        d.tile_staging = staging
    s = Solver(descs)
    for k, p in enumerate(prims):
        s.upload_prim(p, k)
    s.step(steps)
    return [s.cons(k) for k in range(len(descs))], s.status()


CASES = {
    "kh_periodic": lambda pr, rc: ([W.kh(64, pr, rc, net())[0][0]], [W.kh_prim(64)]),
    "walls_partial": lambda pr, rc: (
        [make_desc(model="euler", flux="kepes_tecno4_roe", recon=rc, nx=48, ny=70, precision=pr, network=net(),
                   bc=["wall", "wall", "wall", "neumann", "periodic", "periodic"])], [_bump(48, 70)]),
    "two_problems": lambda pr, rc: (
        [make_desc(model="euler", flux="kepes_tecno4_roe", recon=rc, nx=32, ny=40, precision=pr, network=net()),
         make_desc(model="euler", flux="kepes_tecno4_roe", recon=rc, nx=64, ny=33, precision=pr, network=net(),
                   bc=["periodic", "periodic", "wall", "wall", "periodic", "periodic"])],
        [_bump(32, 40), _bump(64, 33)]),
    "euler3d": lambda pr, rc: (
        [make_desc(model="euler", flux="kepes_tecno4_roe", recon=rc, nx=16, ny=24, nz=35, precision=pr,
                   network=net(), bc=["periodic", "periodic", "neumann", "wall", "wall", "neumann"])],
        [_bump(16, 24, 35)]),
    # nx = 30: the last column group of a row is partial for both widths
    # (TMA does not qualify; the narrow and wide tiles run plain loads there)
    "partial_groups": lambda pr, rc: (
        [make_desc(model="euler", flux="kepes_tecno4_roe", recon=rc, nx=30, ny=50, precision=pr, network=net(),
                   bc=["periodic", "periodic", "wall", "neumann", "periodic", "periodic"])], [_bump(30, 50)]),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision,recon", [("fp64", "sp_weno"), ("fp64", "sp_weno_dl"),
                                             ("fp32_bf16", "sp_weno_dl"), ("fp32_bf16", "sp_weno")])
@pytest.mark.parametrize("variant", [2, 3], ids=["tma", "narrow"])
def test_tile_variant_equals_cp_async(case, precision, recon, variant):
    d1, p1 = CASES[case](precision, recon)
    d2, p2 = CASES[case](precision, recon)
    a, sa = _run(d1, p1, 6, variant)   # TMA / narrow tiles
    b, sb = _run(d2, p2, 6, 1)         # 8-column tiles, cp.async
    for x, y in zip(a, b):
        if precision == "fp64":
            # IEEE arithmetic without contraction: the two kernels give the same bits
            assert np.array_equal(x, y), float(np.max(np.abs(x - y)))
        else:
            # FP32 with contraction: the two kernels are separate compilations
            # whose FMA choices may differ; an ulp that moves a stencil across a
            # reconstruction threshold can grow to ~1e-4 in a few steps
            scale = np.maximum(np.max(np.abs(y), axis=(1, 2, 3), keepdims=True), 1e-300)   # 2-D: w is 0
            rel = np.abs(x - y) / scale
            assert np.max(rel) < 1e-3 and np.mean(rel < 1e-6) > 0.95, (float(np.max(rel)), float(np.mean(rel < 1e-6)))
    assert sa.code == sb.code == 0
    assert sa.faces_checked == sb.faces_checked and sa.sign_violations == sb.sign_violations


def test_tile_variants_on_slabs_with_halo_faces():
    """Three slabs of a periodic 2-D domain stepped with their halo layers
    exchanged: the ghost rows are the stored halo layers beside each slab's
    interior, outside its tensor map.  Every variant gives the same bits."""
    from dspw.slabs import LocalSlabs
    out = []
    for staging in (2, 1, 3):
        dom = make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=32, ny=96)
        dom.tile_staging = staging
        sl = LocalSlabs(dom, 3)
        sl.upload_prim(_bump(32, 96))
        sl.step(3)
        out.append(sl.cons())
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[2], out[1])


def test_tuner_keeps_results_with_either_staging():
    """dspw_tune times the tile variants (tile_staging 0) and keeps the
    fastest; the state it leaves steps to the cp.async results."""
    (d,), (p,), _ = W.kh(128, "fp32_bf16", "sp_weno_dl", net())
    s = Solver(d)
    s.upload_prim(p)
    before, after = s.tune(reps=2)
    assert after <= before * 1.001
    s.step(3)
    (d2,), _, _ = W.kh(128, "fp32_bf16", "sp_weno_dl", net())
    d2.tile_staging = 1
    s2 = Solver(d2)
    s2.upload_prim(p)
    s2.step(3)
    a, b = s.cons(), s2.cons()
    # the same bits when the tuner kept cp.async; FP32 rounding for another variant
    assert np.max(np.abs(a - b)) <= 1e-3 * np.max(np.abs(b))
