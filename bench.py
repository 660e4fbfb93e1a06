"""Benchmark of the stage path: cell-updates/s on 2-D Euler Kelvin-Helmholtz.

Workload (one GPU): Kelvin-Helmholtz on the periodic unit square at 2048^2,
gamma 1.4, kepes_tecno4_roe flux, DSP-WENO reconstruction (the shipped
5-5-5-5-5 network), SSPRK3 at CFL 0.4, FP32 state with the network layers on
BF16 tensor cores (FP64 time, CFL max and global sums).  One step = one full
SSPRK3 step of every cell; one cell-update = one physical cell advanced by one
step.  The FP64 plain form (SP-WENO, no network) is measured beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload kh|shu_osher|batched|tgv] [--n N]
                    [--precision fp32_bf16|fp64] [--recon sp_weno_dl]

The other workloads (dspw.workloads) time the remaining problem classes:
1-D Euler Shu-Osher, the batch of the isentropic-vortex OOC list plus 4096
Burgers problems, and the 3-D Navier-Stokes Taylor-Green vortex at 256^3.

Under torchrun (N > 1) every rank advances its own 2048^2 problem (weak
scaling, no data-path collective); NCCL only carries the barrier and the
max-over-ranks of the device time.  The batched workload is one problem list
shared out over the ranks by cell count (strong scaling, dspw.partition).

`--impl reference` times the reference's own CPU solver (oracle/_ref, built
from its sources) on bounded samples of the same workload, on all host cores.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "dsp-weno_b200"))
sys.path.insert(0, str(REPO / "oracle"))

METRIC = "cell-updates/s"
NET_FILE = REPO / "tests" / "golden" / "dsp_weno.txt"
# Measurements that need another tool or a long run are recorded, one line
# each, in profiles/bench_records.txt together with the hash of the device
# sources they were taken with; the JSON line attaches a record only when that
# hash equals the current sources' (else the field says that no record of this
# build exists).
RECORDS = REPO / "profiles" / "bench_records.txt"
# the sources of libdspw.so (the network measurement library is built apart)
SOURCES = sorted(f for f in (REPO / "dsp-weno_b200" / "csrc").glob("*") if f.name != "dspw_netbench.cu") + \
    [REPO / "include" / "dspw.h"]


def strip_comments(src: str) -> str:
    """C / C++ source without its // and /* */ comments (string and character
    literals kept as they are), so that a comment edit keeps the build's hash."""
    out, i, n = [], 0, len(src)
    while i < n:
        c = src[i]
        if c in "\"'":
            j = i + 1
            while j < n and src[j] != c:
                j += 2 if src[j] == "\\" else 1
            out.append(src[i:j + 1])
            i = j + 1
        elif src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def source_hash() -> str:
    """sha256 (16 hex digits) of the device sources and the C ABI header, comments removed."""
    import hashlib
    h = hashlib.sha256()
    for f in SOURCES:
        h.update(f.name.encode())
        h.update(strip_comments(f.read_text()).encode())
    return h.hexdigest()[:16]


def read_records(kind: str) -> list[dict]:
    """Records of one kind: lines `<kind> key=value ...` (values without
    spaces, or double-quoted)."""
    import shlex
    out = []
    if not RECORDS.exists():
        return out
    for line in RECORDS.read_text().splitlines():
        if not line.startswith(kind + " "):
            continue
        rec = {}
        for tok in shlex.split(line)[1:]:
            k, _, v = tok.partition("=")
            try:
                rec[k] = float(v)
            except ValueError:
                rec[k] = v
        out.append(rec)
    return out


# ------------------------------------------------------------------ CPU legs

_REF = None


def _ref_worker_init(n, recon):
    global _REF
    import oracle as O
    cfg = dict(model="euler", x=(0, 1), y=(0, 1), Nx=n, Ny=n, Nz=2, cfl=0.4, final_time=1.0, reconstruct=recon,
               net_file=str(NET_FILE), flux="kepes_tecno4_roe", dim=2,
               ic=dict(density="1+(abs(y-0.5)<0.25)", xvelocity="-0.5+(abs(y-0.5)<0.25)",
                       yvelocity="0.01*sin(4*pi*x)", pressure="2.5"), bc="periodic")
    _REF = O.RefEuler(cfg)


def _ref_worker_step(nsteps):
    t = time.perf_counter()
    _REF.step(nsteps)
    return time.perf_counter() - t


class RefPool:
    """All host cores, one reference solver instance per process (the
    reference is single-threaded).  Started with 'spawn' before any GPU call."""

    def __init__(self, n, recon, procs):
        ctx = mp.get_context("spawn")
        self.procs = procs
        self.n = n
        self.pool = ctx.Pool(procs, initializer=_ref_worker_init, initargs=(n, recon))

    def step(self, nsteps=1):
        t0 = time.perf_counter()
        self.pool.map(_ref_worker_step, [nsteps] * self.procs)
        return time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def reference_sample(args, procs, warmup):
    """The reference's CPU solver (oracle/_ref) on all host cores: one process
    per core, each a cpu_sample_n^2 KH grid, `warmup` untimed then args.steps
    timed steps.  Returns (cell-updates/s, seconds, description)."""
    pool = RefPool(args.cpu_sample_n, args.recon, procs)
    for _ in range(warmup):
        pool.step(1)
    t = 0.0
    for _ in range(args.steps):
        t += pool.step(1)
    pool.close()
    v = procs * args.cpu_sample_n ** 2 * args.steps / t
    sample = (f"{procs} processes x reference enflo solver on a {args.cpu_sample_n}^2 (x2 in z, the reference's "
              f"2-D layout) KH grid, {args.recon}, FP64, {args.steps} steps each, physical cells counted")
    return v, t, sample


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ clocks


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ GPU legs


def algorithmic_bytes(name, stage, probs, w):
    """(algorithmic, moved) HBM bytes of one launch of kernel ``name`` in stage
    ``stage`` over problems ``probs`` = [(cells, nv, dim, ns, kernel class)],
    nv the stored components, w the word size.  A sweep launch of a mixed batch
    is named ``sweep_<d>.c<class>`` and covers the problems of that class only.

    Algorithmic bytes follow the fully fused stage: it reads U^k (and U^n from
    the second SSPRK3 stage on) and writes U^(k+1) once, 2 or 3 nv w per cell,
    8 nv w per cell-update over the three stages.  They are counted on the
    stage's last sweep (or the viscous update, for Navier-Stokes), which is
    where the fused form's reads and write happen.  `moved` adds what this
    implementation moves beyond that: the x (and for 3-D, y) sweeps read U^k
    and write the residual R, the last sweep reads R, and the Navier-Stokes
    kernels go through the entropy-variable and node-flux buffers."""
    base, _, cls = name.partition(".c")
    name = base
    alg = moved = 0
    for cells, nv, dim, ns, kcls in probs:
        if cls and int(cls) != kcls:
            continue
        fused = 3 if stage > 0 else 2   # read U^k (+ U^n), write U^(k+1)
        a = m = 0
        if ns:
            m = {"entvars": 2, "visc_nodes": 4, "sweep_x": 2, "sweep_y": 3, "sweep_z": 3,
                 "visc_update": 3 + fused}.get(name, 0)
            a = fused if name == "visc_update" else 0
        elif name.startswith("sweep_"):
            axis = "xyz".index(name[-1])
            if axis < dim:
                if axis == dim - 1:
                    a = fused
                    m = fused + (1 if dim > 1 else 0)   # + the residual of the earlier sweeps
                else:
                    m = 2 if axis == 0 else 3
        alg += cells * nv * w * a
        moved += cells * nv * w * m
    return alg, moved


def build_workload(args, precision, recon, rank, world):
    """(descs, prims, cells of this rank, cells of all ranks, scaling)."""
    from dspw import load_network_file, workloads as W
    from dspw.partition import partition

    net = load_network_file(NET_FILE)
    if args.workload == "kh":
        d, p, c = W.kh(args.n or 2048, precision, recon, net, seed=12345 + rank)
        return d, p, c, c * world, "weak"
    if args.workload == "shu_osher":
        d, p, c = W.shu_osher(args.n or 25600, precision, recon, net)
        return d, p, c, c * world, "weak"
    if args.workload == "tgv":
        d, p, c = W.tgv(args.n or 256, precision, recon, net)
        return d, p, c, c * world, "weak"
    # batched: one fixed problem list shared out by cell count (strong scaling)
    specs = W.batched_specs()
    cells = [W.spec_cells(s) for s in specs]
    mine = partition(cells, world)[rank]
    d, p, c = W.batched(precision, recon, net, select=mine)
    return d, p, c, sum(cells), "strong"


def measure_slabs(args, torch, dist, rank, world, config):
    """One KH domain cut into `world` slabs along y, one per rank, connected
    over NCCL: each rank's step graph exchanges its halo layers before every
    stage and all-reduces the CFL speed (strong scaling of one problem).
    Returns the JSON line (rank 0) or None."""
    from dspw import load_network_file, workloads as W
    from dspw.slabs import DistSlabs

    n = args.n or 2048
    (d,), (p0,), _ = W.kh(n, args.precision, args.recon, load_network_file(NET_FILE), seed=12345)
    sl = DistSlabs(d, rank, world, device_exchange=True)
    sl.upload_prim(p0)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.ExternalStream(sl.sol.stream_ptr(), device=dev)
    sl.step(args.warmup)
    sl.sol.sync()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sl.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    st = sl.sol.status()
    if rank != 0:
        return None
    return {"metric": METRIC, "value": n * n * args.steps / (ms * 1e-3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if args.precision == "fp32_bf16" else "f64",
            "data": "synthetic", "config": config, "slab_layers": [sl.lo, sl.hi],
            "health": {"code": st.code, "nonfinite": st.nonfinite_cells, "sign_violations": st.sign_violations}}


def kernel_class(d, dim):
    """Sweep kernel class of a problem (the library's spec_of): Euler / NS with a
    kepes_tecno4 flux run the kernels specialised for their dimension and
    reconstruction family (10 * dim + 1 SP-WENO, + 2 DSP-WENO), 1-D scalar
    problems the scalar kernel (100 + 1 or 2), others class 0."""
    from dspw import FLUX, RECON
    if d.model in (0, 1):
        if dim == 1 and d.recon < RECON["first"]:
            return 100 + (2 if d.recon == RECON["sp_weno_dl"] else 1)
        return 0
    if d.flux not in (FLUX["kepes_tecno4_roe"], FLUX["kepes_tecno4_rusanov"]):
        return 0
    return 10 * dim + (2 if d.recon == RECON["sp_weno_dl"] else 1)


def prob_info(descs):
    out = []
    for d in descs:
        dim = 1 + (d.ny > 1) + (d.nz > 1)
        nv = 1 if d.model in (0, 1) else dim + 2
        out.append((d.nx * d.ny * d.nz, nv, dim, d.model in (3, 4), kernel_class(d, dim)))
    return out


def measure_gpu(args, torch, dist, rank, world):
    import dspw
    from dspw import Solver

    dev = torch.device("cuda", torch.cuda.current_device())
    descs, prims, ncell, ncell_all, scaling = build_workload(args, args.precision, args.recon, rank, world)
    probs = prob_info(descs)

    def solver(d, pr):
        s = Solver(d)
        for p, a in enumerate(pr):
            s.upload_prim(a, p)
        tuned["ms"] = s.tune(reps=3)   # launch grids picked by timing (dspw_tune), before any timed step
        return s

    tuned = {}

    def timed(s, steps, warmup):
        stream = torch.cuda.ExternalStream(s.stream_ptr(), device=dev)
        s.step(warmup)
        s.sync()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    s = solver(descs, prims)
    if args.profile_only:
        # the profiler starts after upload and tuning (ncu --profile-from-start off)
        torch.cuda.profiler.start()
        s.step(args.warmup)
        s.step(args.steps)
        s.sync()
        return None
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms = timed(s, args.steps, args.warmup)
    clk = clocks.stop()
    st = s.status()
    # per-kernel durations of one (un-graphed) step for the roofline
    prof = s.profile_step()
    w = 4 if args.precision == "fp32_bf16" else 8
    first = "entvars" if any(p[3] for p in probs) else "sweep_x"   # the first launch of a stage
    stage, rows, prev = -1, [], None
    for name, kms in prof:
        base = name.partition(".c")[0]
        if base == first and prev != first:   # one x launch per kernel class
            stage += 1
        prev = base
        rows.append((name, stage, kms))
    dom = max(rows, key=lambda r: r[2])
    dom_bytes, dom_moved = algorithmic_bytes(dom[0], dom[1], probs, w)
    peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text()) if (REPO / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs")
    peak_src = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if not peak:
        peak, peak_src = 6650.0, "fallback 6650 GB/s, an earlier measurement on this pool (of fallback)"
    # a launch that carries none of the fused stage's bytes (the inviscid
    # sweeps of a Navier-Stokes stage, whose update happens in the viscous
    # kernel) is measured against the bytes it moves itself
    basis = "fused" if dom_bytes else "moved"
    achieved = (dom_bytes or dom_moved) / (dom[2] * 1e-3) / 1e9
    # the whole step: 8 nv w per cell-update of the fused form
    step_bytes = sum(c * nv * w * 8 for c, nv, dim, ns, kc in probs)
    # e2e through the C ABI with host buffers: upload every problem (pinned
    # H2D), one step, download every problem (D2H) per step
    pinned, outs = [], []
    for a in prims:
        hp = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape)
        hp[...] = a
        pinned.append(hp)
        outs.append(torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape))
    e2e_steps = max(2, min(args.steps, 10 if len(prims) < 16 else 2))
    lib = dspw.lib()
    for p, a in enumerate(pinned):
        s.upload_prim(a, p)
    s.step(1)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for p, a in enumerate(pinned):
            dspw.check(lib.dspw_upload_prim(s.h, p, a), "upload")
        dspw.check(lib.dspw_step(s.h, 1, 0.0), "step")
        for p, a in enumerate(outs):
            dspw.check(lib.dspw_download_cons(s.h, p, a), "download")
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    del s
    # FP64 plain form (SP-WENO, no network) on the same workload for the
    # ratio, and the FP64 form of the network (the reference's arithmetic)
    fp64_ms = fp64_dl_ms = None
    if args.precision == "fp32_bf16" and not args.no_fp64:
        k64 = max(1, args.steps // 4)
        d64, p64, _, _, _ = build_workload(args, "fp64", "sp_weno", rank, world)
        s64 = solver(d64, p64)
        fp64_ms = timed(s64, k64, max(1, args.warmup // 2)) / k64
        del s64
        if args.recon == "sp_weno_dl":
            d64, p64, _, _, _ = build_workload(args, "fp64", "sp_weno_dl", rank, world)
            s64 = solver(d64, p64)
            fp64_dl_ms = timed(s64, k64, max(1, args.warmup // 2)) / k64
            del s64
    nbytes = sum(a.nbytes for a in prims)
    tune_ms = tuned.get("ms")
    return dict(tune_ms=tune_ms, ms=ms, clk=clk, status=st, prof=rows, dom=dom, dom_bytes=dom_bytes,
                dom_moved=dom_moved, basis=basis, achieved=achieved, peak=peak, peak_src=peak_src, step_bytes=step_bytes,
                e2e_s=e2e_s, e2e_steps=e2e_steps, ncell=ncell, ncell_all=ncell_all, scaling=scaling,
                launches=len(prof), fp64_ms=fp64_ms, fp64_dl_ms=fp64_dl_ms, h2d=nbytes, d2h=nbytes,
                nprob=len(descs))


def matched_error(torch):
    """Time to a given L1 density error: FP64 plain SP-WENO against FP32 + BF16
    DSP-WENO, on a shock problem (Shu-Osher, error against a 51200-cell FP64
    solution averaged to each grid) and a smooth one (isentropic vortex to
    t = 2, error against the exact advected vortex).  Each form runs a grid
    sequence to the final time; device time per run is measured with CUDA
    events around dspw_run.  The FP64 cost of reaching each FP32 error is
    interpolated in log-log along the FP64 sequence."""
    from dspw import Solver, load_network_file, workloads as W

    net = load_network_file(NET_FILE)

    def run(descs, prims):
        s = Solver(descs)
        for p, a in enumerate(prims):
            s.upload_prim(a, p)
        st = torch.cuda.ExternalStream(s.stream_ptr())
        s.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        steps = s.run(chunk=256)
        e1.record(st)
        e1.synchronize()
        return s, e0.elapsed_time(e1), steps

    def interp_cost(err64, ms64, e):
        le, lt = np.log(err64), np.log(ms64)
        order = np.argsort(le)
        return float(np.exp(np.interp(np.log(e), le[order], lt[order])))

    out = {}
    d, p, _ = W.shu_osher(51200, "fp64", "sp_weno", net)
    s, _, _ = run(d, p)
    ref = s.prim()[0, 0, 0]
    del s
    rows = {}
    for prec, rec, ns in (("fp64", "sp_weno", (400, 800, 1600, 3200, 6400)),
                          ("fp32_bf16", "sp_weno_dl", (400, 800, 1600))):
        for n in ns:
            d, p, _ = W.shu_osher(n, prec, rec, net)
            s, ms, steps = run(d, p)
            e = float(np.mean(np.abs(s.prim()[0, 0, 0] - ref.reshape(n, -1).mean(axis=1))))
            rows.setdefault(prec, []).append((n, e, ms, steps))
    out["shu_osher"] = rows
    rows = {}
    t_end = 2.0
    for prec, rec, ns in (("fp64", "sp_weno", (64, 128, 256, 512, 1024)),
                          ("fp32_bf16", "sp_weno_dl", (64, 128, 256, 512))):
        for n in ns:
            d, p, _ = W.batched(prec, rec, net, levels=(n,), nburgers=0, vortex_time=t_end)
            s, ms, steps = run(d, p)
            e = float(s.errors(W.vortex_exact_density(n, s.globals().time), comp=0)[0])
            rows.setdefault(prec, []).append((n, e, ms, steps))
    out["vortex_t2"] = rows
    summary = {}
    for case, rows in out.items():
        e64 = np.array([r[1] for r in rows["fp64"]])
        t64 = np.array([r[2] for r in rows["fp64"]])
        summary[case] = [{"n": n, "fp32_dl_err": e, "fp32_dl_ms": ms, "fp64_plain_ms_at_same_err": interp_cost(e64, t64, e),
                          "speedup": interp_cost(e64, t64, e) / ms,
                          "inside_fp64_range": bool(e64.min() <= e <= e64.max())}
                         for n, e, ms, _ in rows["fp32_bf16"]]
    return {"metric": "time to matched L1 density error, FP64 plain SP-WENO / FP32+BF16 DSP-WENO",
            "unit": "ratio", "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
            "runs": {c: {k: [list(r) for r in v] for k, v in rows.items()} for c, rows in out.items()},
            "columns": ["n", "l1_err", "device_ms_per_run", "steps"], "summary": summary}


def kh_accuracy(torch, grids=(1024, 2048), n_ref=4096, t_end=1.0):
    """Accuracy of the forms on the headline problem: Kelvin-Helmholtz to
    t = 1 on 1024^2 and 2048^2 in FP32 + BF16 DSP-WENO, FP64 DSP-WENO and the
    FP64 plain form (SP-WENO), against the FP64 plain form on 4096^2
    (box-averaged to each grid).  All grids start from one noise field
    (workloads.kh_prim_nested).  L1 is the reference's volume-weighted error
    (compute_errors.cc:9-33), i.e. the mean over the unit square; L-inf the
    largest cell error; both of the density.  Device time of every run (CUDA
    events around dspw_run) and its sign-property violations are reported."""
    from dspw import Solver, load_network_file, make_desc
    from dspw.workloads import kh_prim_nested

    net = load_network_file(NET_FILE)

    def run(n, prec, recon):
        d = make_desc(model="euler", flux="kepes_tecno4_roe", recon=recon, nx=n, ny=n, nz=1, x=(0, 1), y=(0, 1),
                      bc="periodic", cfl=0.4, final_time=t_end, network=net, precision=prec)
        s = Solver(d)
        s.upload_prim(kh_prim_nested(n, n_ref))
        st = torch.cuda.ExternalStream(s.stream_ptr())
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        steps = s.run(chunk=512)
        e1.record(st)
        e1.synchronize()
        rho = s.prim()[0, 0]
        stat = s.status()
        g = s.globals()
        out = {"n": n, "precision": prec, "recon": recon, "steps": steps, "t": g.time,
               "device_ms": e0.elapsed_time(e1), "sign_violations": stat.sign_violations,
               "faces_checked": stat.faces_checked, "code": stat.code}
        del s
        return rho, out

    rho_ref, ref_info = run(n_ref, "fp64", "sp_weno")
    runs, pairs, summary = [ref_info], [], []
    for n in grids:
        r = n_ref // n
        ref = rho_ref.reshape(n, r, n, r).mean(axis=(1, 3))
        got = {}
        for prec, recon in (("fp64", "sp_weno"), ("fp64", "sp_weno_dl"), ("fp32_bf16", "sp_weno_dl")):
            rho, info = run(n, prec, recon)
            e = np.abs(rho - ref)
            info.update({"l1_vs_ref": float(e.mean()), "linf_vs_ref": float(e.max())})
            runs.append(info)
            got[(prec, recon)] = rho
        for a, b in ((("fp32_bf16", "sp_weno_dl"), ("fp64", "sp_weno_dl")),
                     (("fp64", "sp_weno_dl"), ("fp64", "sp_weno")),
                     (("fp32_bf16", "sp_weno_dl"), ("fp64", "sp_weno"))):
            e = np.abs(got[a] - got[b])
            pairs.append({"n": n, "a": "/".join(a), "b": "/".join(b), "l1": float(e.mean()), "linf": float(e.max())})
        by = {(x["precision"], x["recon"]): x for x in runs if x["n"] == n}
        l1_32 = by[("fp32_bf16", "sp_weno_dl")]["l1_vs_ref"]
        l1_64 = by[("fp64", "sp_weno")]["l1_vs_ref"]
        summary.append({"n": n, "l1_fp32_dl": l1_32, "l1_fp64_plain": l1_64, "l1_ratio": l1_32 / l1_64,
                        "linf_fp32_dl": by[("fp32_bf16", "sp_weno_dl")]["linf_vs_ref"],
                        "linf_fp64_plain": by[("fp64", "sp_weno")]["linf_vs_ref"],
                        "sign_violations_fp32_dl": by[("fp32_bf16", "sp_weno_dl")]["sign_violations"],
                        "time_ratio_fp64_plain_over_fp32_dl": by[("fp64", "sp_weno")]["device_ms"] /
                        by[("fp32_bf16", "sp_weno_dl")]["device_ms"]})
    return {"metric": "L1 / L-inf density error at t = 1 vs FP64 SP-WENO on 4096^2, KH", "unit": "density",
            "n_gpus": 1, "data": "synthetic", "source_hash": source_hash(), "reference_grid": n_ref,
            "runs": runs, "pairs": pairs, "summary": summary,
            "records": [f"accuracy n={s['n']} t=1.0 l1_fp32_dl={s['l1_fp32_dl']:.6e} "
                        f"l1_fp64_plain={s['l1_fp64_plain']:.6e} l1_ratio={s['l1_ratio']:.4f} "
                        f"linf_fp32_dl={s['linf_fp32_dl']:.6e} linf_fp64_plain={s['linf_fp64_plain']:.6e} "
                        f"sign_violations_fp32_dl={int(s['sign_violations_fp32_dl'])} "
                        f"time_ratio={s['time_ratio_fp64_plain_over_fp32_dl']:.4f} ref_grid={n_ref} "
                        f"src={source_hash()}" for s in summary]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="kh",
                    choices=["kh", "shu_osher", "batched", "tgv", "matched_error", "kh_slabs", "kh_accuracy"],
                    help="kh: 2-D Euler KH (the headline); shu_osher: 1-D Euler; batched: vortex OOC list plus "
                         "4096 Burgers problems in one batch (shared out over ranks); tgv: 3-D Navier-Stokes "
                         "Taylor-Green vortex; matched_error: time to equal L1 error of the two forms on "
                         "Shu-Osher and the isentropic vortex (its own JSON line); kh_slabs: one KH domain "
                         "cut into one slab per rank, halo layers over NCCL inside the step graphs; "
                         "kh_accuracy: L1 / L-inf density error of the forms on KH 1024^2 and 2048^2 at t = 1 "
                         "against FP64 SP-WENO on 4096^2 (its own JSON line; long)")
    ap.add_argument("--n", type=int, default=None, help="grid size (kh 2048, shu_osher 25600, tgv 256)")
    ap.add_argument("--precision", default="fp32_bf16", choices=["fp32_bf16", "fp64"])
    ap.add_argument("--recon", default="sp_weno_dl")
    ap.add_argument("--cpu-sample-n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-matched-error", action="store_true",
                    help="leave the matched-error summary out of the KH line")
    ap.add_argument("--profile-only", action="store_true",
                    help="warm-up and timed steps only (no e2e, CPU or FP64 legs), the profiler started "
                         "after upload and tuning; for ncu captures with --profile-from-start off")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload in ("matched_error", "kh_accuracy"):
        if args.impl == "reference" or rank != 0:
            return
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(matched_error(torch) if args.workload == "matched_error" else kh_accuracy(torch)))
        return
    if args.workload == "kh":
        n = args.n or 2048
        config = {"workload": f"kh{n}_{args.precision}_{args.recon}_kepes_tecno4_roe", "grid": [n, n],
                  "model": "euler2d", "flux": "kepes_tecno4_roe", "recon": args.recon, "precision": args.precision,
                  "cfl": 0.4}
    elif args.workload == "shu_osher":
        n = args.n or 25600
        config = {"workload": f"shu_osher{n}_{args.precision}_{args.recon}_kepes_tecno4_roe", "grid": [n],
                  "model": "euler1d", "flux": "kepes_tecno4_roe", "recon": args.recon, "precision": args.precision,
                  "cfl": 0.4}
    elif args.workload == "kh_slabs":
        n = args.n or 2048
        config = {"workload": f"kh{n}_slabs{world}_{args.precision}_{args.recon}_kepes_tecno4_roe", "grid": [n, n],
                  "model": "euler2d", "flux": "kepes_tecno4_roe", "recon": args.recon, "precision": args.precision,
                  "cfl": 0.4, "decomposition": f"{world} slabs of y rows, one per rank, 2 halo rows per side"}
    elif args.workload == "batched":
        config = {"workload": f"batched_vortex_ooc_burgers4096_{args.precision}_{args.recon}",
                  "problems": "isentropic vortex at 64..2048^2 (6 levels, kepes_tecno4_roe) + 4096 Burgers "
                              "Nx~U{100..5000} (bur_tecno4), one batch per rank, shared out by cell count",
                  "recon": args.recon, "precision": args.precision, "cfl": 0.5}
    else:
        n = args.n or 256
        config = {"workload": f"tgv{n}_ns_es_{args.precision}_{args.recon}_kepes_tecno4_roe", "grid": [n, n, n],
                  "model": "ns_es", "flux": "kepes_tecno4_roe", "recon": args.recon, "precision": args.precision,
                  "cfl": 0.4, "Re": 1600, "Mach": 0.1}
    config["l2"] = "no flush: per-step working set (U^n, two stage buffers, residual) exceeds the 126 MB L2"

    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload != "kh":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm samples the KH workload only"}))
            return
        procs = cpu_cores()
        v, t, sample = reference_sample(args, procs, args.warmup)
        # the sample's own configuration: the GPU arm's workload, on the grid
        # the CPU samples (physical cells counted, as the GPU arm counts them)
        ref_config = dict(config)
        ref_config.update({"workload": f"kh{args.cpu_sample_n}_fp64_{args.recon}_kepes_tecno4_roe_reference_cpu",
                           "grid": [args.cpu_sample_n, args.cpu_sample_n], "precision": "fp64",
                           "sample_of": config["workload"],
                           "layout": "the reference's 2-D layout: Nz = 2 cells, periodic"})
        print(json.dumps({"metric": METRIC, "value": v, "unit": "cell-updates/s", "impl": "reference",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": ref_config,
                          "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                                           "sample": sample},
                          "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    # CPU baseline first (spawned processes, before any GPU call)
    cpu = None
    if args.workload != "kh":
        cpu = {"value": None, "unit": "cell-updates/s", "cores": 0, "kind": "reference",
               "sample": "not sampled: the CPU baseline covers the KH workload"}
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            procs = cpu_cores()
            v, _, sample = reference_sample(args, procs, 1)
            cpu = {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "reference", "sample": sample}
        except Exception as e:  # the checker may be unbuilt on a bare box
            cpu = {"value": None, "unit": "cell-updates/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    import torch
    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist
    else:
        torch.cuda.set_device(0)
    if args.workload == "kh_slabs":
        line = measure_slabs(args, torch, dist, rank, world, config)
        if dist is not None:
            dist.barrier()
        if line is not None:
            print(json.dumps(line))
        import gc
        gc.collect()   # the slab's handle (and its NCCL communicator) before the process group
        if dist is not None:
            dist.destroy_process_group()
        return
    r = measure_gpu(args, torch, dist, rank, world)
    if r is None:
        return
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    steps = args.steps
    value = r["ncell_all"] * steps / (r["ms"] * 1e-3)
    e2e_v = r["ncell_all"] * r["e2e_steps"] / r["e2e_s"]
    dom = r["dom"]
    src = source_hash()
    # DRAM traffic and issue activity of the dominant launch from an ncu
    # capture of this very build (records with the current source hash)
    traffic = issue = None
    traffic_note = "no ncu record of this build for this launch"
    for rec in read_records("traffic"):
        if rec.get("workload") == config.get("workload") and rec.get("kernel") == dom[0] and \
                int(rec.get("stage", -9)) == dom[1] and rec.get("src") == src:
            traffic = (rec["dram_read"] + rec["dram_write"]) / rec["cells"] * r["ncell"]
            issue = rec.get("issue_active_pct")
            traffic_note = f"ncu capture: {rec.get('capture', '')}"
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / steps, "higher_is_better": True, "scaling": r["scaling"],
        "vs_baseline": None, "dtype": "f32" if args.precision == "fp32_bf16" else "f64", "data": "synthetic",
        "config": config,
        "roofline": {"bound": "hbm", "kernel": dom[0], "stage": dom[1], "achieved": r["achieved"],
                     "peak": r["peak"], "unit": "GB/s", "frac": r["achieved"] / r["peak"],
                     "traffic": traffic, "traffic_source": traffic_note,
                     "algorithmic_bytes": r["dom_bytes"] or r["dom_moved"],
                     "extra_bytes": r["dom_moved"] - (r["dom_bytes"] or r["dom_moved"]),
                     "bytes_basis": "fused stage" if r["basis"] == "fused" else
                     "the launch's own reads and writes (no fused-stage bytes fall on it)",
                     "launch_ms": dom[2], "peak_source": r["peak_src"],
                     "issue_frac": issue / 100.0 if issue is not None else None,
                     "step_achieved": r["step_bytes"] * steps / (r["ms"] * 1e-3) / 1e9,
                     "step_frac": r["step_bytes"] * steps / (r["ms"] * 1e-3) / 1e9 / r["peak"],
                     "bytes_rule": "fused stage: read U^k (+U^n), write U^(k+1); 8 nv w per cell-update"},
        "source_hash": src,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_v, "unit": "cell-updates/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "api": "dspw_upload_prim + dspw_step(1) + dspw_download_cons"},
        "gpu_launches": r["launches"] * steps,
        "tuner": {"sweeps_ms_default_grid": r["tune_ms"][0], "sweeps_ms_tuned": r["tune_ms"][1]}
        if r.get("tune_ms") else None,
        "clocks": r["clk"],
        "kernels_ms_one_step": [[a, b, round(c, 4)] for a, b, c in r["prof"]],
        "health": {"code": r["status"].code, "sign_violations": r["status"].sign_violations,
                   "faces_checked": r["status"].faces_checked, "limiter_acts": r["status"].limiter_acts,
                   "nonfinite": r["status"].nonfinite_cells, "nonpositive": r["status"].nonpositive_cells},
    }
    if r["fp64_ms"]:
        line["fp64_plain"] = {"value": r["ncell_all"] / (r["fp64_ms"] * 1e-3), "ms_per_step": r["fp64_ms"],
                              "recon": "sp_weno", "speedup_fp32_bf16_dl_over_fp64_plain": r["fp64_ms"] / (r["ms"] / steps)}
    if r["fp64_dl_ms"]:
        line["fp64_dl"] = {"value": r["ncell_all"] / (r["fp64_dl_ms"] * 1e-3), "ms_per_step": r["fp64_dl_ms"],
                           "recon": "sp_weno_dl", "note": "the FP64 form of the network, the reference's arithmetic"}
    if args.workload == "kh" and args.precision == "fp32_bf16":
        # the accuracy half of the metric at this workload's grid, from the
        # long runs of `bench.py --workload kh_accuracy`
        acc = [a for a in read_records("accuracy") if int(a.get("n", 0)) == (args.n or 2048)]
        if acc:
            a = acc[-1]
            line["accuracy"] = {k: a[k] for k in a}
            line["accuracy"]["same_build"] = a.get("src") == src
    if args.workload == "kh" and world == 1 and args.precision == "fp32_bf16" and not args.no_matched_error:
        # the metric's other half: time to the same L1 density error, FP64 plain
        # over FP32 + BF16 DSP-WENO (bench.py --workload matched_error for the runs)
        me = matched_error(torch)["summary"]
        line["matched_error"] = {
            case: [{"n": x["n"], "l1_err": x["fp32_dl_err"], "speedup": x["speedup"],
                    "inside_fp64_range": x["inside_fp64_range"]} for x in rows] for case, rows in me.items()}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
