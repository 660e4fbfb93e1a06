"""libdspw.so loads without a GPU and exports every entry point that
include/dspw.h declares; the ctypes descriptor matches the C layout."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from dspw import capi

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (REPO / "include" / "dspw.h").read_text()
    return sorted(set(re.findall(r"DSPW_API\s+[\w\s\*]+?\b(dspw_\w+)\s*\(", text)))


def test_header_declares_api():
    names = declared_functions()
    assert "dspw_create" in names and "dspw_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    if not capi.LIB_PATH.exists():
        pytest.fail("libdspw.so is not built; run __graft_entry__.build()")
    lib = ctypes.CDLL(str(capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.dspw_version() == capi.ABI_VERSION


def test_error_strings():
    lib = capi.lib()
    for code in range(9):
        s = lib.dspw_error_string(code).decode()
        assert s.startswith(capi.STATUS[code])


def _c_offsets(struct, fields, tmp_path):
    """offsetof() of each field and sizeof() of a struct of include/dspw.h, as
    the host C compiler lays it out."""
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dspw.h"', "int main(void) {"]
    for f in fields:
        lines.append(f'  printf("%zu\\n", offsetof({struct}, {f}));')
    lines.append(f'  printf("%zu\\n", sizeof({struct}));')
    lines.append("  return 0; }")
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return [int(v) for v in out]


@pytest.mark.parametrize("struct,cls", [("dspw_desc", "Desc"), ("dspw_globals_out", "Globals"),
                                        ("dspw_status_out", "StatusOut"), ("dspw_halo_out", "HaloOut"),
                                        ("dspw_train_cfg", "TrainCfg")])
def test_struct_layouts_match_the_header(struct, cls, tmp_path):
    """Every field of the ctypes mirror sits at the C compiler's offset."""
    if shutil.which("gcc") is None:
        pytest.skip("no host C compiler")
    c = getattr(capi, cls)
    names = [f[0] for f in c._fields_]
    offs = _c_offsets(struct, names, tmp_path)
    assert offs[:-1] == [getattr(c, n).offset for n in names]
    assert offs[-1] == ctypes.sizeof(c)


def test_bad_descriptor_rejected_without_gpu():
    """Descriptor validation runs on the host before any CUDA call."""
    lib = capi.lib()
    d = capi.make_desc(nx=0)
    h = ctypes.c_void_p()
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = capi.make_desc(model="ns_es", nx=8, ny=8, nz=8, mu_ref=0.0)
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = capi.make_desc(bc=["periodic", "wall", "periodic", "periodic", "periodic", "periodic"])
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = capi.make_desc()
    d.abi_version = 99
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = capi.make_desc()
    d.abi_version = 1   # the layout before the named box / kernel / cell-size fields
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    # unused slots must stay zero; named fields are range-checked
    for field, idx, val in (("reserved_i", 0, 1), ("reserved_d", 4, 1.0), ("cell_size", 1, -1.0),
                            ("cell_size", 2, float("inf"))):
        d = capi.make_desc()
        getattr(d, field)[idx] = val
        assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1, field
    d = capi.make_desc()
    d.generic_kernels = 2
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = capi.make_desc()
    d.tile_staging = 4   # 0 automatic, 1 cp.async, 2 TMA, 3 narrow tiles
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d = capi.set_training_box(capi.make_desc(), [0, 0, 0, 0, 0], [1, 1, 1, 1, 1])
    d.nn_feat_lo[3] = 2.0   # lo above hi
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.nn_feat_lo[3] = float("nan")
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1
    # eno 3 on a wall axis of two cells: the third ghost's mirror leaves the line
    d = capi.make_desc(recon="eno3", nx=16, ny=2, bc=["periodic", "periodic", "wall", "wall", "periodic", "periodic"])
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 6
    # halo faces: only on the last swept direction, not for Navier-Stokes, and
    # with at least one ghost width of layers
    d = capi.make_desc(nx=16, ny=8, bc=["halo", "halo", "periodic", "periodic", "periodic", "periodic"])
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 6
    d = capi.make_desc(model="ns_es", nx=8, ny=8, nz=8, mu_ref=0.01,
                       bc=["periodic", "periodic", "periodic", "periodic", "halo", "halo"])
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 6
    d = capi.make_desc(nx=16, ny=2, bc=["periodic", "periodic", "halo", "halo", "periodic", "periodic"],
                       recon="eno3")
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 6
    d = capi.make_desc(nx=16, ny=8, bc=["periodic", "periodic", "halo", "periodic", "periodic", "periodic"])
    assert lib.dspw_create(ctypes.byref(d), ctypes.byref(h)) == 1   # periodic pairs with periodic only
    # slab entry points: bad handles and views are refused on the host
    assert lib.dspw_slab_connect(None, b"\0" * 128, 0, 1) == 1
    assert lib.dspw_halo_view(None, 0, 0, ctypes.byref(capi.HaloOut())) == 1
    assert lib.dspw_nccl_id(None) == 1
    # the four-cell reconstruction entry point has no six-cell stencils
    l, r, acts = np.zeros(1), np.zeros(1), ctypes.c_longlong()
    u = np.arange(4, dtype=np.float64)
    assert lib.dspw_reconstruct_batch(ctypes.byref(capi.make_desc(recon="eno3")), u, 1, l, r, ctypes.byref(acts)) == 6


def test_network_file_roundtrip(tmp_path):
    W, b = capi.load_network_file(REPO / "tests" / "golden" / "dsp_weno.txt")
    assert W.shape == (4, 5, 5) and b.shape == (4, 5)
    capi.save_network_file(tmp_path / "n.txt", W, b)
    W2, b2 = capi.load_network_file(tmp_path / "n.txt")
    assert (W2 == W).all() and (b2 == b).all()
