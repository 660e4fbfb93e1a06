"""The C++ command-line driver ``enflo_b200`` (drop-in for ``enflo -i param.in``
and ``enfloS -i param.in``, enflo/src/main.cc:12-29).

CPU tests: the param.in reader and expression evaluator, checked through
``--check`` (the descriptor the driver would create) and ``--dump-ic`` (the
initial state it would upload) against the initial states the reference's own
fparser-based setup produced for the golden runs (``runs.npz``, key
``<case>|prim0``).  The GPU test runs a three-level OOC study through the
driver and compares its ``l1_err.dat`` with the reference's errors
(``ooc.npz``).
"""
from __future__ import annotations

import json
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from dspw import capi
from dspw.paramfile import write_param
from _common import GOLDEN, NET_FILE, desc_from_cfg, load, run_cases

CLI = Path(capi.__file__).resolve().parents[1] / "enflo_b200"


def _need_cli():
    if not CLI.exists():
        pytest.fail("enflo_b200 is not built; run __graft_entry__.build()")


def _run(args, cwd, check=True):
    r = subprocess.run([str(CLI)] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError(f"enflo_b200 {args} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    return r


def _write(tmp_path, cfg, name="param.in"):
    cfg = dict(cfg)
    cfg["net_file"] = str(NET_FILE)
    p = tmp_path / name
    p.write_text(write_param(cfg))
    return p


@pytest.mark.parametrize("case", [c[0] for c in run_cases()])
def test_initial_state_matches_reference_setup(tmp_path, case):
    _need_cli()
    name, kind, cfg, _, _ = next(c for c in run_cases() if c[0] == case)
    p = _write(tmp_path, cfg)
    out = tmp_path / "ic.bin"
    _run(["-i", p, "--dump-ic", out], tmp_path)
    ref = load("runs.npz")[f"{name}|prim0"]
    got = np.fromfile(out, dtype=np.float64).reshape(ref.shape)
    scale = np.max(np.abs(ref.reshape(ref.shape[0], -1)), axis=1).reshape(-1, 1, 1, 1) + 1e-300
    assert np.max(np.abs(got - ref) / scale) <= 1e-14, case


@pytest.mark.parametrize("case", ["shuosher_sp_weno_dl", "linadv_sp_weno", "tgv_ns", "wall2d", "burgers_wall_dl",
                                  "wall2d_eno3", "linadv_wall_eno3"])
def test_descriptor_matches_python_side(tmp_path, case):
    _need_cli()
    name, kind, cfg, _, _ = next(c for c in run_cases() if c[0] == case)
    p = _write(tmp_path, cfg)
    got = json.loads(_run(["-i", p, "--check"], tmp_path).stdout)
    d = desc_from_cfg(cfg, cfg["Nx"], cfg.get("Ny", 2), cfg.get("Nz", 2))
    for key in ("model", "flux", "recon", "nx", "ny", "nz", "t_stamps"):
        assert got[key] == getattr(d, key), key
    assert got["bc"] == list(d.bc)
    assert got["xmin"] == d.xmin and got["xmax"] == d.xmax
    assert got["cfl"] == d.cfl and got["final_time"] == d.final_time
    if cfg["reconstruct"] == "sp_weno_dl":
        assert got["nn_w000"] == d.nn_w[0][0][0]
    assert got["levels"] == 1


HAND_WRITTEN = """
// a hand-written file: comments of every kind and ',' / ';' separators
grid
{
   x_min   -pi
   x_max   2*pi/2
   Nx_cell { 40,80;160 }
   y_min   0
   y_max   1
   Ny_cell { 2, 2, 2 }
   z_min   0
   z_max   1
   Nz_cell { 2 2 2 }
}
/* numerical scheme
   over two lines */
numeric
{
   time_scheme  ssprk3
   cfl          0.5      # trailing comment after a number
   max_iter     100000
   final_time   0.25
   min_residue  1.0e-6
   reconstruct  sp_wenoc
   net_file     none
}
material
{
   model  linadv
   vel    { 1.0 0.0 0.0 }
   flux   lin_tecno4
}
constants
{
   amp 0.75
   % width of the bump
   w   0.5
}
initial_condition
{
   amp*exp(-(x/w)^2) + (abs(x) < 1)*(x >= 0) - if(x > 2, 0.25, 0) + max(min(x, 0.1), -0.1)^2
}
exact_soln
{
   available  yes
   amp*exp(-((x-t)/w)^2)
}
boundary_condition
{
   xleft  { type periodic }
   xright { type periodic }
   yleft  { type periodic }
   yright { type periodic }
   zleft  { type periodic }
   zright { type periodic }
}
output
{
   OOC_study    yes
   problem_dim  1
   time_stamps  3
   output_path  .
}
"""


def test_hand_written_file(tmp_path):
    _need_cli()
    p = tmp_path / "param.in"
    p.write_text(HAND_WRITTEN)
    got = json.loads(_run(["-i", p, "--check"], tmp_path).stdout)
    assert got["levels"] == 3 and got["nx"] == 40 and got["recon"] == capi.RECON["sp_wenoc"]
    assert got["xmin"] == -math.pi and got["xmax"] == math.pi and got["t_stamps"] == 3
    out = tmp_path / "ic.bin"
    _run(["-i", p, "--dump-ic", out], tmp_path)
    u = np.fromfile(out).reshape(2, 2, 40)
    dx = 2 * math.pi / 40
    x = -math.pi + dx * (np.arange(40) + 0.5)
    want = (0.75 * np.exp(-(x / 0.5) ** 2) + ((np.abs(x) < 1) & (x >= 0)) - np.where(x > 2, 0.25, 0.0)
            + np.clip(x, -0.1, 0.1) ** 2)
    for k in range(2):
        for j in range(2):
            np.testing.assert_allclose(u[k, j], want, rtol=0, atol=1e-15)


@pytest.mark.parametrize("text,msg", [
    ("grid\n{\n x_minimum 0\n", "expecting x_min"),
    (HAND_WRITTEN.replace("Ny_cell { 2, 2, 2 }", "Ny_cell { 2, 2 }"), "same number of levels"),
    (HAND_WRITTEN.replace("lin_tecno4", "lin_upwind"), "unknown flux scheme"),
    (HAND_WRITTEN.replace("sp_wenoc", "weno5"), "reconstruction not supported"),
    (HAND_WRITTEN.replace("(x/w)^2", "(x/w)^^2"), "expression"),
    # expressions run to the end of the line, as Reader::getline reads them
    (HAND_WRITTEN.replace("x_max   2*pi/2", "x_max   2*pi/2   # comment"), "unexpected text"),
    (HAND_WRITTEN.replace("amp*exp(-((x-t)", "amp*expo(-((x-t)"), "unknown function"),
    (HAND_WRITTEN.replace("sp_wenoc", "sp_weno_dl").replace("net_file     none", "net_file     missing.txt"),
     "network file does not exist"),
], ids=["keyword", "levels", "flux", "recon", "syntax", "comment", "function", "network"])
def test_errors_are_reported(tmp_path, text, msg):
    _need_cli()
    p = tmp_path / "param.in"
    p.write_text(text)
    r = _run(["-i", p, "--check"], tmp_path, check=False)
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_eno_level(tmp_path):
    """'reconstruct eno <level>' carries its level (parameter.cc:178-184);
    levels 2 and 3 are built (eno_pw has coefficients for no other,
    limiter.h:88-94)."""
    _need_cli()
    p = tmp_path / "param.in"
    p.write_text(HAND_WRITTEN.replace("reconstruct  sp_wenoc", "reconstruct  eno 2"))
    got = json.loads(_run(["-i", p, "--check"], tmp_path).stdout)
    assert got["recon"] == capi.RECON["eno2"]
    p.write_text(HAND_WRITTEN.replace("reconstruct  sp_wenoc", "reconstruct  eno 3"))
    got = json.loads(_run(["-i", p, "--check"], tmp_path).stdout)
    assert got["recon"] == capi.RECON["eno3"]
    p.write_text(HAND_WRITTEN.replace("reconstruct  sp_wenoc", "reconstruct  eno 4"))
    r = _run(["-i", p, "--check"], tmp_path, check=False)
    assert r.returncode == 1 and "reconstruction not supported" in r.stderr


def test_usage(tmp_path):
    _need_cli()
    assert _run([], tmp_path, check=False).returncode == 2
    assert _run(["-i", tmp_path / "nope.in", "--check"], tmp_path, check=False).returncode == 1


def _read_table(path):
    rows = []
    for line in path.read_text().splitlines():
        f = line.split()
        if len(f) >= 4 and f[0].isdigit():
            rows.append((int(f[0]), float(f[3]), f[4] if len(f) > 4 else "-"))
    return rows


@pytest.mark.gpu
@pytest.mark.parametrize("recon", ["sp_weno", "sp_weno_dl"])
def test_ooc_study_through_driver(tmp_path, recon):
    """Three-level linear-advection OOC study (Nx = 100, 200, 400), errors
    against the reference's run of the same file."""
    _need_cli()
    cfg = dict(model="linadv", x=("-pi", "pi"), Nx=[100, 200, 400], Ny=[2, 2, 2], Nz=[2, 2, 2], cfl=0.5,
               final_time=0.5, reconstruct=recon, flux="lin_tecno4", ic="pow(sin(x),4)",
               exact="pow(sin(x-t),4)", bc="periodic", time_stamps=5, ooc=True)
    p = _write(tmp_path, cfg)
    _run(["-i", p], tmp_path)
    ref = load("ooc.npz")[recon]
    soln = tmp_path / f"SOLN_FILES_{recon}"
    for col, fname in enumerate(("l1_err.dat", "l2_err.dat", "linf_err.dat")):
        rows = _read_table(soln / fname)
        assert [r[0] for r in rows] == [100, 200, 400]
        for i, r in enumerate(rows):
            # the table carries 6 significant digits
            assert abs(r[1] - ref[i, col]) <= 5e-6 * ref[i, col], (fname, i, r, ref[i, col])
        rate = float(rows[2][2])
        # L1 converges at third order; L-inf is limited near the extrema of sin^4
        assert (2.5 < rate < 4.5) if col == 0 else (1.5 < rate < 4.5), (fname, rate)
    assert (soln / "globals.dat").exists()


def _numbers(path):
    return [[float(x) for x in line.split()] for line in path.read_text().splitlines() if line.strip()]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["kh_sp_weno", "tgv_ns", "wall2d", "burgers_wenoc"])
def test_globals_file_matches_reference_rows(tmp_path, name):
    """globals.dat in compute_global's layout (enflo/src/compute_global.cc:80-88,
    enflo_scalar/src_scalar/compute_global.cc:34-38), one row per step from the
    device diagnostics, against the reference's own rows of the same steps
    (``diag.npz``); the file carries 10 significant digits."""
    _need_cli()
    ref = load("diag.npz")[f"{name}|rows"]
    name_, kind, cfg, _, _ = next(c for c in run_cases() if c[0] == name)
    cfg = dict(cfg)
    cfg["max_iter"] = len(ref)
    cfg["ooc"] = False
    p = _write(tmp_path, cfg)
    r = _run(["-i", p], tmp_path)
    rows = _numbers(tmp_path / f"SOLN_FILES_{cfg['reconstruct']}" / "globals.dat")
    if kind == "S":
        # the state before the first step, then one row after every step
        assert len(rows) == len(ref) + 1 and len(rows[0]) == 3 and rows[0][0] == 0.0
        # sum u^2/2 vol of the initial state (the file's first row has 10 digits)
        g = load("runs.npz")
        ent0 = 0.5 * float(np.sum(g[f"{name}|prim0"] ** 2)) * float(np.prod(g[f"{name}|h"]))
        assert abs(rows[0][1] - ent0) <= 1e-9 * abs(ent0)
        got = np.array(rows[1:])
        want = np.stack([ref[:, 1], ref[:, 2], (ref[:, 2] - ent0) / ent0], axis=1)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("ITER =")]
        assert len(lines) == len(ref) and "RES = " in lines[0]
    else:
        assert len(rows) == len(ref) and all(len(x) == 7 for x in rows)
        got = np.array(rows)
        ent0 = ref[0, 2]
        want = np.stack([ref[:, 1], ref[:, 2], (ref[:, 2] - ent0) / abs(ent0), ref[:, 3], ref[:, 4], ref[:, 5],
                         ref[:, 6]], axis=1)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("ITER =")]
        assert len(lines) == len(ref)
        # ITER = n after the step and the mass residual norm of its last stage
        f = lines[-1].split()
        assert int(f[2]) == len(ref)
        assert abs(float(f[8]) - ref[-1, 7]) <= 1e-3 * ref[-1, 7]
    for c in range(got.shape[1]):
        scale = np.max(np.abs(want[:, c]))
        assert np.max(np.abs(got[:, c] - want[:, c])) <= 2e-9 * scale + 1e-300, (name, c, got[:, c], want[:, c])


def _output_cases():
    from make_golden import output_cases
    return output_cases()


def _compare_text(got, want, what, rtol):
    """Line-by-line comparison of a solution file: identical structure and
    words, numbers equal to `rtol` (the files print 6 significant digits)."""
    gl, wl = got.splitlines(), want.splitlines()
    assert len(gl) == len(wl), (what, len(gl), len(wl))
    for n, (a, b) in enumerate(zip(gl, wl)):
        if a == b:
            continue
        ta, tb = a.split(), b.split()
        assert len(ta) == len(tb), (what, n, a, b)
        for x, y in zip(ta, tb):
            if x == y:
                continue
            fx, fy = float(x), float(y)   # words must be identical; numbers may differ in the last digit
            assert abs(fx - fy) <= rtol * max(abs(fy), 1e-300) or abs(fx - fy) <= 1e-12, (what, n, a, b)


@pytest.mark.parametrize("case", _output_cases(), ids=lambda c: c[0])
def test_initial_solution_files_match_reference(tmp_path, case):
    """The t = 0 files of FV::output (sol0000.vtk, omg0000.vtk with the node
    vorticity, 1Dsol0000.dat) written by the driver's own writer, against the
    files the reference's writer produced for the same param.in."""
    _need_cli()
    name, kind, cfg = case
    gold = load("output.npz")
    cfg = dict(cfg)
    cfg["ooc"] = False
    p = _write(tmp_path, cfg)
    r = _run(["-i", p, "--output-ic"], tmp_path)
    soln = tmp_path / f"SOLN_FILES_{cfg['reconstruct']}"
    names = [k.split("|")[1] for k in gold.files if k.startswith(name + "|") and "0000" in k]
    assert names and "Saving solutions in" in r.stdout
    for fn in names:
        # the initial state is the same expression evaluation: only last-digit
        # differences of the 6-digit print are allowed
        _compare_text((soln / fn).read_text(), str(gold[f"{name}|{fn}"]), f"{name}/{fn}", rtol=2e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("case", _output_cases(), ids=lambda c: c[0])
def test_solution_files_at_time_stamps_match_reference(tmp_path, case):
    """A full run through the driver: the solution files at t = 0 and at every
    time stamp (from the device snapshots) against the reference's files."""
    _need_cli()
    name, kind, cfg = case
    gold = load("output.npz")
    cfg = dict(cfg)
    cfg["ooc"] = False
    p = _write(tmp_path, cfg)
    _run(["-i", p], tmp_path)
    soln = tmp_path / f"SOLN_FILES_{cfg['reconstruct']}"
    names = sorted(k.split("|")[1] for k in gold.files if k.startswith(name + "|"))
    # the numbered files of FV::output (the driver also writes sol_final.dat at full precision)
    got_names = sorted(f.name for f in soln.iterdir() if re.fullmatch(r"(sol|omg|1Dsol)\d{4}\.(vtk|dat)", f.name))
    assert got_names == names
    for fn in names:
        _compare_text((soln / fn).read_text(), str(gold[f"{name}|{fn}"]), f"{name}/{fn}", rtol=2e-5)
