"""Build libdspw.so (the C ABI of include/dspw.h) for sm_100a with nvcc.

Each precision is its own translation unit: the FP64 plain form is compiled
with --fmad=false (no FMA contraction, matching the reference's x86-64 build),
the FP32 form with contraction.  Objects and the library are written in-tree
(dsp-weno_b200/_build, dsp-weno_b200/libdspw.so).

    python dsp-weno_b200/build.py [--verbose-ptxas]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
BUILD = Path(os.environ.get("DSPW_BUILD_DIR", PKG / "_build"))
LIB = Path(os.environ.get("DSPW_OUT", PKG / "libdspw.so"))
EXTRA = os.environ.get("DSPW_EXTRA_FLAGS", "").split()
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          f"-I{REPO / 'include'}", "--expt-relaxed-constexpr"]

UNITS = {
    "dspw_fp64.cu": ["--fmad=false"],
    # FP32 form: approximate division and square root, denormals flushed
    # (KH 2048^2: DSP-WENO 3.15 -> 3.02 ms, SP-WENO 2.29 -> 1.91 ms per step);
    # the FP64 units keep IEEE arithmetic without contraction, for parity
    "dspw_fp32.cu": ["--fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "dspw_capi.cu": ["--fmad=false"],
    "dspw_train.cu": ["--fmad=true"],
    "dspw_noalloc.cu": ["--fmad=false"],
}


def compile_unit(name: str, flags: list[str], verbose: bool) -> Path:
    src = CSRC / name
    obj = BUILD / (name + ".o")
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc")) + [
        REPO / "include" / "dspw.h"]
    cmd = [NVCC, *ARCH, *COMMON, *EXTRA, *flags, "-c", str(src), "-o", str(obj)]
    # the object is current when it is newer than its sources and was built
    # with the same command line
    stamp = obj.with_suffix(".cmd")
    same = stamp.exists() and stamp.read_text() == " ".join(cmd)
    if same and obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps) and not verbose:
        return obj
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{r.stderr}")
    stamp.write_text(" ".join(cmd))
    if verbose and r.stderr:
        print(r.stderr)
    return obj


HOST = PKG / "host"
CLI = Path(os.environ.get("DSPW_CLI_OUT", PKG / "enflo_b200"))


def build_cli(lib: Path) -> Path:
    """The command-line driver (host/*.cc), linked against libdspw.so."""
    srcs = sorted(HOST.glob("*.cc"))
    deps = srcs + sorted(HOST.glob("*.h")) + [REPO / "include" / "dspw.h", lib]
    if CLI.exists() and all(CLI.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return CLI
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", f"-I{REPO / 'include'}", *map(str, srcs),
           "-o", str(CLI), f"-L{lib.parent}", f"-l:{lib.name}", "-Wl,-rpath,$ORIGIN", "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host driver build failed:\n{r.stderr}")
    return CLI


NETBENCH = PKG / "libdspw_netbench.so"


def build_netbench(verbose: bool) -> Path:
    """The network measurement kernels (csrc/dspw_netbench.cu: the sweep
    kernels' mma.sync form and a tcgen05 form), a library of their own."""
    obj = compile_unit("dspw_netbench.cu", ["--fmad=true", "-ftz=true"], verbose)
    if not NETBENCH.exists() or NETBENCH.stat().st_mtime < obj.stat().st_mtime:
        cmd = [NVCC, *ARCH, "-shared", "-o", str(NETBENCH), str(obj), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return NETBENCH


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        futs = [ex.submit(compile_unit, n, f, verbose) for n, f in UNITS.items()]
        objs = [f.result() for f in futs]
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    if LIB == PKG / "libdspw.so":
        build_cli(LIB)
        build_netbench(verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose-ptxas" in sys.argv))
