"""TEST INFRASTRUCTURE: Python access to the two CPU checkers.

* ``Oracle`` -- the plain-C FP64 restatement (liboracle.so, dspw_oracle.c).
* ``RefEuler`` / ``RefScalar`` -- the reference solvers compiled from their own
  sources (oracle/_ref/*.so, built by oracle/Makefile from the reference tree),
  driven through the harness in oracle/ref_harness.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs use this module.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REPO = ORACLE_DIR.parent
sys.path.insert(0, str(REPO / "dsp-weno_b200"))
from dspw.capi import DIAG_COLS, RECON, Desc, nvar  # noqa: E402
from dspw.paramfile import write_param  # noqa: E402

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _load(path):
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built (make -C oracle)")
    return C.CDLL(str(path))


_OR = None


def oracle_lib():
    global _OR
    if _OR is None:
        L = _load(ORACLE_DIR / "liboracle.so")
        P, I, D = C.c_void_p, C.c_int, C.c_double
        sig = {
            "or_create": (P, [C.POINTER(Desc)]),
            "or_destroy": (None, [P]),
            "or_set_prim": (None, [P, _dp]),
            "or_get_prim": (None, [P, _dp]),
            "or_get_cons": (None, [P, _dp]),
            "or_compute_dt": (D, [P]),
            "or_residual": (None, [P, I, _dp]),
            "or_step": (I, [P, I, D]),
            "or_step_diag": (I, [P, I, D, _dp]),
            "or_time": (None, [P, C.POINTER(D), C.POINTER(I), C.POINTER(D)]),
            "or_globals": (None, [P, C.POINTER(D), _dp, C.POINTER(D)]),
            "or_logavg": (D, [D, D]),
            "or_sp_weno": (None, [_dp, I, C.POINTER(D), C.POINTER(D)]),
            "or_nn_forward": (None, [C.POINTER(Desc), _dp, C.POINTER(D), C.POINTER(D)]),
            "or_nn_features": (None, [_dp, _dp, _dp, _dp]),
            "or_euler_face_flux": (None, [C.POINTER(Desc), _dp, I, D, D, D, _dp, _dp]),
            "or_scalar_face_flux": (D, [C.POINTER(Desc), _dp, I, D, D, D]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        _OR = L
    return _OR


class Oracle:
    """FP64 CPU restatement of the stage path for one problem."""

    def __init__(self, desc: Desc):
        self.desc = desc
        self.L = oracle_lib()
        self.h = self.L.or_create(C.byref(desc))

    def __del__(self):
        try:
            self.L.or_destroy(self.h)
        except Exception:
            pass

    def shape(self):
        d = self.desc
        return (nvar(d), d.nz, d.ny, d.nx)

    def set_prim(self, prim):
        self.L.or_set_prim(self.h, np.ascontiguousarray(prim, dtype=np.float64).reshape(self.shape()))

    def prim(self):
        a = np.empty(self.shape())
        self.L.or_get_prim(self.h, a)
        return a

    def cons(self):
        a = np.empty(self.shape())
        self.L.or_get_cons(self.h, a)
        return a

    def residual(self, rk=0):
        a = np.empty(self.shape())
        self.L.or_residual(self.h, rk, a)
        return a

    def compute_dt(self):
        return self.L.or_compute_dt(self.h)

    def step(self, n=1, fixed_dt=0.0):
        return self.L.or_step(self.h, int(n), float(fixed_dt))

    def step_diag(self, n=1, fixed_dt=0.0):
        """Steps with the per-step diagnostics rows (DIAG_COLS columns each)."""
        rows = np.zeros((int(n), DIAG_COLS))
        k = self.L.or_step_diag(self.h, int(n), float(fixed_dt), rows)
        return rows[:k]

    def time(self):
        t, i, dt = C.c_double(), C.c_int(), C.c_double()
        self.L.or_time(self.h, C.byref(t), C.byref(i), C.byref(dt))
        return t.value, i.value, dt.value

    def globals(self):
        e, k = C.c_double(), C.c_double()
        c5 = np.zeros(5)
        self.L.or_globals(self.h, C.byref(e), c5, C.byref(k))
        return e.value, c5, k.value


def sp_weno(u4, corr=0):
    l, r = C.c_double(), C.c_double()
    oracle_lib().or_sp_weno(np.ascontiguousarray(u4, dtype=np.float64), corr, C.byref(l), C.byref(r))
    return l.value, r.value


def nn_forward(desc, u4):
    l, r = C.c_double(), C.c_double()
    oracle_lib().or_nn_forward(C.byref(desc), np.ascontiguousarray(u4, dtype=np.float64), C.byref(l), C.byref(r))
    return l.value, r.value


def nn_features(u4):
    f, vx, vy = np.zeros(5), np.zeros(5), np.zeros(5)
    oracle_lib().or_nn_features(np.ascontiguousarray(u4, dtype=np.float64), f, vx, vy)
    return f, vx, vy


def stencil_cells(desc) -> int:
    """Cells of a face stencil: 2 ghost widths, 6 for eno 3 and 4 otherwise."""
    return 6 if desc.recon == RECON["eno3"] else 4


def euler_face_flux(desc, P4, direction, dx, dy, dz):
    ns = stencil_cells(desc)
    V, F = np.zeros(5 * ns), np.zeros(5)
    oracle_lib().or_euler_face_flux(C.byref(desc), np.ascontiguousarray(P4, dtype=np.float64).reshape(5 * ns),
                                    direction, dx, dy, dz, V, F)
    return F, V.reshape(ns, 5)


def scalar_face_flux(desc, u4, direction, dx, dy, dz):
    return oracle_lib().or_scalar_face_flux(C.byref(desc), np.ascontiguousarray(u4, dtype=np.float64),
                                            direction, dx, dy, dz)


def logavg(a, b):
    return oracle_lib().or_logavg(a, b)


# --------------------------------------------------------------------------
# the reference itself (built from its sources by oracle/Makefile)

REF_DIR = ORACLE_DIR / "_ref"


def ref_available() -> bool:
    return (REF_DIR / "libenflo_ref.so").exists() and (REF_DIR / "libenfloS_ref.so").exists()


_REF = {}


def _ref_lib(kind):
    if kind in _REF:
        return _REF[kind]
    P, I, D = C.c_void_p, C.c_int, C.c_double
    if kind == "E":
        L = _load(REF_DIR / "libenflo_ref.so")
        sig = {
            "refE_create": (P, [C.c_char_p, I]), "refE_destroy": (None, [P]),
            "refE_dims": (None, [P, C.POINTER(I), C.POINTER(D)]),
            "refE_get_prim": (None, [P, _dp]), "refE_get_cons": (None, [P, _dp]),
            "refE_set_prim": (None, [P, _dp]), "refE_residual": (None, [P, I, _dp]),
            "refE_compute_dt": (D, [P]), "refE_step": (I, [P, I, D]),
            "refE_step_diag": (I, [P, I, D, _dp]),
            "refE_output": (None, [P, I]),
            "refE_face_flux": (None, [P, _dp, I, _dp, _dp]),
            "refE_reconstruct": (None, [P, _dp, _dp, _dp]),
            "refE_nn_forward": (None, [P, _dp, C.POINTER(D), C.POINTER(D)]),
            "refE_logavg": (D, [D, D]),
        }
    else:
        L = _load(REF_DIR / "libenfloS_ref.so")
        sig = {
            "refS_create": (P, [C.c_char_p, I]), "refS_destroy": (None, [P]),
            "refS_dims": (None, [P, C.POINTER(I), C.POINTER(D)]),
            "refS_get": (None, [P, _dp]), "refS_set": (None, [P, _dp]),
            "refS_residual": (None, [P, I, _dp]), "refS_compute_dt": (D, [P]),
            "refS_step": (I, [P, I, D]), "refS_run_errors": (None, [P, _dp]),
            "refS_step_diag": (I, [P, I, D, _dp]),
            "refS_output": (None, [P, I]),
            "refS_face_flux": (D, [P, _dp, I]),
            "refS_reconstruct": (None, [P, _dp, C.POINTER(D), C.POINTER(D)]),
            "refS_sp_weno": (None, [_dp, I, C.POINTER(D), C.POINTER(D)]),
        }
    for n, (r, a) in sig.items():
        f = getattr(L, n)
        f.restype = r
        f.argtypes = a
    _REF[kind] = L
    return L


class _RefBase:
    def __init__(self, cfg: dict, level: int = 0):
        self.tmp = tempfile.mkdtemp(prefix="dspw_ref_")
        cfg = dict(cfg)
        cfg["output_path"] = self.tmp
        self.param_path = os.path.join(self.tmp, "param.in")
        with open(self.param_path, "w") as f:
            f.write(write_param(cfg))
        self.h = self._create(self.param_path.encode(), level)
        if not self.h:
            raise RuntimeError("reference rejected the configuration")
        n = (C.c_int * 5)()
        d = (C.c_double * 5)()
        self._dims(self.h, n, d)
        self.nx, self.ny, self.nz, self.ng = n[0], n[1], n[2], n[3]
        self.dx, self.dy, self.dz = d[0], d[1], d[2]

    def run_outputs(self):
        """Run to the end with the reference's solution writer on (t = 0 and
        every time stamp); returns {file name: text} of its SOLN_FILES folder."""
        getattr(self.L, self._prefix + "_output")(self.h, 1)
        getattr(self.L, self._prefix + "_step")(self.h, 1 << 30, 0.0)
        out = {}
        for d in os.listdir(self.tmp):
            if d.startswith("SOLN_FILES_"):
                for fn in sorted(os.listdir(os.path.join(self.tmp, d))):
                    if fn.startswith(("sol", "omg", "1Dsol")):
                        with open(os.path.join(self.tmp, d, fn)) as f:
                            out[fn] = f.read()
        return out

    def info(self):
        n = (C.c_int * 5)()
        d = (C.c_double * 5)()
        self._dims(self.h, n, d)
        return {"time": d[3], "dt": d[4], "iter": n[4]}


class RefEuler(_RefBase):
    def __init__(self, cfg, level=0):
        self.L = _ref_lib("E")
        self._prefix = "refE"
        self._create, self._dims = self.L.refE_create, self.L.refE_dims
        super().__init__(cfg, level)

    def __del__(self):
        try:
            self.L.refE_destroy(self.h)
        except Exception:
            pass

    def shape(self):
        return (5, self.nz, self.ny, self.nx)

    def prim(self):
        a = np.empty(self.shape()); self.L.refE_get_prim(self.h, a); return a

    def cons(self):
        a = np.empty(self.shape()); self.L.refE_get_cons(self.h, a); return a

    def set_prim(self, p):
        self.L.refE_set_prim(self.h, np.ascontiguousarray(p, dtype=np.float64))

    def residual(self, rk=0):
        a = np.empty(self.shape()); self.L.refE_residual(self.h, rk, a); return a

    def compute_dt(self):
        return self.L.refE_compute_dt(self.h)

    def step(self, n=1, fixed_dt=0.0):
        return self.L.refE_step(self.h, int(n), float(fixed_dt))

    def step_diag(self, n=1, fixed_dt=0.0):
        rows = np.zeros((int(n), DIAG_COLS))
        k = self.L.refE_step_diag(self.h, int(n), float(fixed_dt), rows)
        return rows[:k]

    def face_flux(self, P4, direction):
        P4 = np.ascontiguousarray(P4, dtype=np.float64)
        ns = P4.size // 5
        V, F = np.zeros(5 * ns), np.zeros(5)
        self.L.refE_face_flux(self.h, P4.reshape(5 * ns), direction, V, F)
        return F, V.reshape(ns, 5)

    def reconstruct(self, Z45):
        l, r = np.zeros(5), np.zeros(5)
        self.L.refE_reconstruct(self.h, np.ascontiguousarray(Z45, dtype=np.float64).reshape(20), l, r)
        return l, r

    def nn_forward(self, u4):
        l, r = C.c_double(), C.c_double()
        self.L.refE_nn_forward(self.h, np.ascontiguousarray(u4, dtype=np.float64), C.byref(l), C.byref(r))
        return l.value, r.value


class RefScalar(_RefBase):
    def __init__(self, cfg, level=0):
        self.L = _ref_lib("S")
        self._prefix = "refS"
        self._create, self._dims = self.L.refS_create, self.L.refS_dims
        super().__init__(cfg, level)

    def __del__(self):
        try:
            self.L.refS_destroy(self.h)
        except Exception:
            pass

    def shape(self):
        return (1, self.nz, self.ny, self.nx)

    def get(self):
        a = np.empty(self.shape()); self.L.refS_get(self.h, a); return a

    prim = get

    def set(self, u):
        self.L.refS_set(self.h, np.ascontiguousarray(u, dtype=np.float64))

    def residual(self, rk=0):
        a = np.empty(self.shape()); self.L.refS_residual(self.h, rk, a); return a

    def compute_dt(self):
        return self.L.refS_compute_dt(self.h)

    def step(self, n=1, fixed_dt=0.0):
        return self.L.refS_step(self.h, int(n), float(fixed_dt))

    def step_diag(self, n=1, fixed_dt=0.0):
        rows = np.zeros((int(n), DIAG_COLS))
        k = self.L.refS_step_diag(self.h, int(n), float(fixed_dt), rows)
        return rows[:k]

    def run_errors(self):
        e = np.zeros(3); self.L.refS_run_errors(self.h, e); return e

    def face_flux(self, u4, direction):
        return self.L.refS_face_flux(self.h, np.ascontiguousarray(u4, dtype=np.float64), direction)

    def reconstruct(self, u4):
        l, r = C.c_double(), C.c_double()
        self.L.refS_reconstruct(self.h, np.ascontiguousarray(u4, dtype=np.float64), C.byref(l), C.byref(r))
        return l.value, r.value


def ref_sp_weno(u4, corr=0):
    l, r = C.c_double(), C.c_double()
    _ref_lib("S").refS_sp_weno(np.ascontiguousarray(u4, dtype=np.float64), corr, C.byref(l), C.byref(r))
    return l.value, r.value
