"""Small fixed workloads that launch one kind of kernel each, for profiler
captures of single kernels (no timing, no output beyond "ok"):

    python -m dspw.kernel_cases kh N PRECISION RECON STEPS   (run from dsp-weno_b200/)
    python -m dspw.kernel_cases kh_tuned N PRECISION RECON STEPS
                                               the same after dspw_tune (as the benchmark
                                               runs it); the profiler is started after the
                                               tuning (ncu --profile-from-start off)
    python -m dspw.kernel_cases burgers        4096 Burgers problems, k_sweep_scalar
    python -m dspw.kernel_cases tgv N PRECISION RECON STEPS  Navier-Stokes: k_entvars,
                                               k_visc_nodes, k_visc_update, the z sweep
    python -m dspw.kernel_cases diag           per-step diagnostics kernels on KH 1024^2
    python -m dspw.kernel_cases train          trainer kernels on 2 M collected pairs

The states are the seeded synthetic workloads of dspw.workloads."""
from __future__ import annotations

import sys
from pathlib import Path

from . import Solver, Trainer, load_network_file, xavier_network, workloads as W

NET_FILE = Path(__file__).resolve().parents[2] / "tests" / "golden" / "dsp_weno.txt"


def main(argv):
    net = load_network_file(NET_FILE)
    mode = argv[0]
    if mode in ("kh", "tgv", "kh_tuned"):
        n, prec, rec, steps = int(argv[1]), argv[2], argv[3], int(argv[4])
        d, p, _ = (W.tgv if mode == "tgv" else W.kh)(n, prec, rec, net)
        s = Solver(d)
        s.upload_prim(p[0])
        if mode == "kh_tuned":
            import torch

            s.tune(reps=3)
            s.sync()
            torch.cuda.profiler.start()
        s.step(steps)
        s.sync()
    elif mode == "burgers":
        d, p, _ = W.batched("fp32_bf16", "sp_weno_dl", net, levels=(), nburgers=4096)
        s = Solver(d)
        for k, a in enumerate(p):
            s.upload_prim(a, k)
        s.step(2)
        s.sync()
    elif mode == "diag":
        d, p, _ = W.kh(1024, "fp32_bf16", "sp_weno_dl", net)
        s = Solver(d)
        s.upload_prim(p[0])
        s.diag_enable(16)
        s.step(2)
    elif mode == "train":
        d, p, _ = W.kh(512, "fp64", "sp_weno", None)
        s = Solver(d)
        s.upload_prim(p[0])
        s.step(2)
        tr = Trainer(xavier_network(6008), batch=8192)
        tr.collect(s, 2_000_000)
        tr.epoch()
        tr.epoch()
    else:
        raise SystemExit(f"unknown case {mode}")
    print("ok")


if __name__ == "__main__":
    main(sys.argv[1:])
