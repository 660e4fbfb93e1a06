"""The reference's own enflo program with its time loop on the B200.

oracle/Makefile (target `patched`) copies the reference's enflo/src/fv.cc,
replaces FV::run's time loop by calls to libdspw.so (oracle/ref_patch: the
reference-side binding of include/dspw.h), and links it with the reference's
other sources and main.cc into oracle/_ref/enflo_dspw.  That binary reads a
param.in with the reference's own Parameter and fparser set-up, and here runs
golden cases to their step count; its final state (dumped at full precision)
must match the reference's own CPU run of the same param.in (runs.npz) at
1e-12, and it writes the reference's output files."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from _common import GOLDEN, load, run_cases
from dspw.paramfile import write_param

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]
BIN = REPO / "oracle" / "_ref" / "enflo_dspw"
CASES = ["kh_sp_weno_dl", "shuosher_sp_weno", "wall2d", "euler3d"]


@pytest.mark.parametrize("name", CASES)
def test_patched_reference_driver_matches_reference(name, tmp_path):
    if not BIN.exists():
        pytest.skip("oracle/_ref/enflo_dspw not built (make -C oracle patched needs the reference tree)")
    cases = {c[0]: c for c in run_cases()}
    _, kind, cfg, nsteps, fixed_dt = cases[name]
    assert kind == "E" and fixed_dt == 0.0
    cfg = dict(cfg)
    cfg["max_iter"] = nsteps
    if "net_file" in cfg:
        cfg["net_file"] = str(GOLDEN / "dsp_weno.txt")
    (tmp_path / "param.in").write_text(write_param(cfg))
    dump = tmp_path / "state.bin"
    env = dict(os.environ, DSPW_DUMP_STATE=str(dump))
    r = subprocess.run([str(BIN), "-i", "param.in"], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    g = load("runs.npz")
    ref = g[f"{name}|final"]
    raw = np.fromfile(dump, dtype=np.float64)
    t, it = raw[0], int(raw[1])
    got = raw[2:].reshape(ref.shape)
    tid = g[f"{name}|tid"]
    assert it == int(tid[1]) == nsteps
    assert abs(t - tid[0]) <= 1e-12 * abs(tid[0])
    for c in range(ref.shape[0]):
        scale = np.max(np.abs(ref[c]))
        err = np.abs(got[c] - ref[c])
        assert np.all(err <= 1e-12 * (np.abs(ref[c]) + scale)), (name, c, float(np.max(err)) / max(scale, 1e-300))
    # the reference's files: the solution at t = 0 and the per-step globals
    soln = next(tmp_path.glob("SOLN_FILES_*"))
    assert (soln / "sol0000.vtk").exists()
    rows = [ln for ln in (soln / "globals.dat").read_text().splitlines() if ln.strip()]
    assert len(rows) == nsteps
    assert abs(float(rows[0].split()[0])) == 0.0
