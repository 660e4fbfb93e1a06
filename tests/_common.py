"""Shared helpers for the tests: fixture loading and param-dict -> dspw_desc."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from dspw.capi import make_desc, load_network_file

GOLDEN = Path(__file__).resolve().parent / "golden"
NET_FILE = GOLDEN / "dsp_weno.txt"


def net():
    return load_network_file(NET_FILE)


def _num(v):
    if isinstance(v, (int, float)):
        return float(v)
    return float(eval(str(v), {"__builtins__": {}}, {"pi": math.pi}))


def desc_from_cfg(cfg: dict, nx: int, ny: int, nz: int, **over):
    """dspw_desc equivalent to a param.in dict written by dspw.paramfile.write_param."""
    kw = dict(
        model=cfg["model"], flux=cfg["flux"], recon=cfg.get("reconstruct", "sp_weno").replace(" ", ""),
        nx=nx, ny=ny, nz=nz,
        x=tuple(_num(v) for v in cfg.get("x", (0, 1))),
        y=tuple(_num(v) for v in cfg.get("y", (0, 1))),
        z=tuple(_num(v) for v in cfg.get("z", (0, 1))),
        bc=cfg.get("bc", "periodic"), cfl=float(cfg["cfl"]), final_time=float(cfg["final_time"]),
        max_iter=int(cfg.get("max_iter", 50000)), t_stamps=int(cfg.get("time_stamps", 1)),
        ec1_fix=cfg.get("EC1_fix", "no") == "yes",
        gamma=float(cfg.get("gamma", 1.4)), gas_const=float(cfg.get("gas_const", 1.0)),
        prandtl=float(cfg.get("prandtl", 1.0)), mu_ref=float(cfg.get("mu_ref", 0.0)),
        lin_vel=tuple(cfg.get("vel", (1.0, 0.0, 0.0))), network=net(),
        time_scheme=cfg.get("time_scheme", "ssprk3"),
    )
    kw.update(over)
    return make_desc(**kw)


def load(name):
    return np.load(GOLDEN / name, allow_pickle=False)


def run_cases():
    from make_golden import run_cases as rc
    return rc()


def rel_err(a, b):
    a = np.asarray(a); b = np.asarray(b)
    scale = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / np.maximum(scale, np.max(np.abs(b)) * 1e-3 + 1e-300)))


def oracle_kh_cons(n, recon, steps, dt, seed=12345):
    """Conserved state of the CPU oracle after `steps` steps of size dt of the
    Kelvin-Helmholtz workload (FP64 plain form of recon) on an n x n grid.
    Runs in a worker process (spawned), so the larger grids proceed in
    parallel while the GPU side runs."""
    import oracle as O
    from dspw import workloads as W
    (d,), (p,), _ = W.kh(n, "fp64", recon, net(), seed=seed)
    o = O.Oracle(d)
    o.set_prim(p)
    o.step(steps, fixed_dt=dt)
    return o.cons()
