"""ctypes mirror of include/dspw.h and loader for libdspw.so.

The C ABI is the product boundary; this module only describes it to Python
(tests, benchmark, trainer driver).  Enum values and the descriptor layout must
match include/dspw.h exactly.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent          # dsp-weno_b200/
LIB_PATH = PKG_DIR / "libdspw.so"

ABI_VERSION = 2

MODEL = {"linadv": 0, "burgers": 1, "euler": 2, "ns_es": 3, "ns_kep": 4}
FLUX = {
    "lin_ec": 0, "lin_ec4": 1, "lin_tecno": 2, "lin_tecno4": 3,
    "bur_ec": 4, "bur_ec4": 5, "bur_tecno": 6, "bur_tecno4": 7,
    "roe": 10, "kep": 11, "kep4": 12, "kepec": 13, "kepec4": 14,
    "roe_ec": 15, "roe_ec4": 16, "keps": 17, "keps4": 18,
    "kep_tecno_roe": 19, "kepes_tecno_roe": 20, "kepes_tecno_rusanov": 21,
    "roe_tecno_roe": 22, "kepes_tecno4_roe": 23, "kepes_tecno4_rusanov": 24,
    "roe_tecno4_roe": 25,
}
RECON = {"sp_weno": 0, "sp_wenoc": 1, "sp_weno_corr2": 2, "sp_weno_dl": 3,
         "first": 4, "second": 5, "minmod": 6, "minabs": 7, "eno2": 8,
         "eno3": 9}
BC = {"periodic": 0, "dirichlet": 1, "neumann": 2, "wall": 3, "halo": 4}
TIME = {"rk1": 0, "ssprk3": 1, "jameson_rk4": 2, "rk4": 3}
MU = {"constant": 0, "sutherland": 1, "power": 2}
PRECISION = {"fp64": 0, "fp32_bf16": 1}
# columns of a per-step diagnostics row (enum dspw_diag_col)
DIAG_NAMES = ("iter", "time", "total_entropy", "ke", "ke_diss_pr", "ke_diss_stress", "enstrophy",
              "res_mass", "res_mom_x", "res_mom_y", "res_mom_z", "res_energy")
DIAG_COLS = len(DIAG_NAMES)

STATUS = {0: "DSPW_OK", 1: "DSPW_ERR_ARG", 2: "DSPW_ERR_CUDA", 3: "DSPW_ERR_NONFINITE",
          4: "DSPW_ERR_NONPOSITIVE", 5: "DSPW_ERR_TIMEOUT", 6: "DSPW_ERR_UNSUPPORTED",
          7: "DSPW_ERR_NOMEM", 8: "DSPW_ERR_FINISHED"}


class Desc(C.Structure):
    """struct dspw_desc."""
    _fields_ = [
        ("abi_version", C.c_int), ("model", C.c_int), ("flux", C.c_int), ("recon", C.c_int),
        ("time_scheme", C.c_int), ("precision", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("bc", C.c_int * 6), ("ec1_fix", C.c_int), ("mu_model", C.c_int),
        ("max_iter", C.c_int), ("t_stamps", C.c_int), ("nn_use_box", C.c_int), ("generic_kernels", C.c_int),
        ("tile_staging", C.c_int), ("reserved_i", C.c_int * 5),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("gamma", C.c_double), ("gas_const", C.c_double), ("prandtl", C.c_double),
        ("mu_ref", C.c_double), ("T_ref", C.c_double), ("T_0", C.c_double), ("omega", C.c_double),
        ("lin_vel", C.c_double * 3), ("cfl", C.c_double), ("final_time", C.c_double),
        ("bc_state", (C.c_double * 5) * 6),
        ("nn_w", ((C.c_double * 5) * 5) * 4),
        ("nn_b", (C.c_double * 5) * 4),
        ("nn_feat_lo", C.c_double * 5), ("nn_feat_hi", C.c_double * 5),
        ("cell_size", C.c_double * 3),
        ("reserved_d", C.c_double * 5),
    ]


class Globals(C.Structure):
    _fields_ = [("time", C.c_double), ("dt", C.c_double), ("iter", C.c_int), ("finished", C.c_int),
                ("total_entropy", C.c_double), ("conserved", C.c_double * 5),
                ("kinetic_energy", C.c_double)]


class StatusOut(C.Structure):
    _fields_ = [("code", C.c_int), ("nonfinite_cells", C.c_longlong), ("nonpositive_cells", C.c_longlong),
                ("sign_violations", C.c_longlong), ("faces_checked", C.c_longlong),
                ("limiter_acts", C.c_longlong)]


class HaloOut(C.Structure):
    """dspw_halo_out: device addresses of a slab's halo and boundary layers."""
    _fields_ = [("recv_lo", C.c_void_p), ("recv_hi", C.c_void_p), ("send_lo", C.c_void_p),
                ("send_hi", C.c_void_p), ("count", C.c_longlong), ("comp_stride", C.c_longlong),
                ("ncomp", C.c_int), ("elem_bytes", C.c_int), ("ng", C.c_int), ("layer_cells", C.c_int)]


class TrainCfg(C.Structure):
    _fields_ = [("lr", C.c_double), ("beta1", C.c_double), ("beta2", C.c_double),
                ("weight_decay", C.c_double), ("eps", C.c_double), ("batch", C.c_int), ("seed", C.c_int),
                ("compute_bf16", C.c_int), ("collect_stride", C.c_int), ("reserved_i", C.c_int * 6)]


def load_network_file(path) -> tuple[np.ndarray, np.ndarray]:
    """Read a dsp_weno.txt network file (format of Neural_Network::load_network,
    enflo/src/neural_network.cc:82-130): 'Weights' then 'Biases', each a list of
    'Layer k' / BEGIN / rows / END blocks.  Returns W (4,5,5) and b (4,5)."""
    weights, biases = [], []
    mode = "w"
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    i = 0
    while i < len(lines):
        t = lines[i]
        if t == "Biases":
            mode = "b"
        elif t == "BEGIN":
            rows = []
            i += 1
            while lines[i] != "END":
                vals = [float(v) for v in lines[i].split()]
                if vals:
                    rows.append(vals)
                i += 1
            if mode == "w":
                weights.append(np.array(rows, dtype=np.float64))
            else:
                biases.append(np.array([r[0] for r in rows], dtype=np.float64))
        i += 1
    W = np.stack(weights)
    b = np.stack(biases)
    if W.shape != (4, 5, 5) or b.shape != (4, 5):
        raise ValueError(f"network file {path}: expected 4 layers of 5x5, got {W.shape} {b.shape}")
    return W, b


def save_network_file(path, W, b) -> None:
    """Write W (4,5,5) and b (4,5) in the dsp_weno.txt format (the trainer's
    save_net_weights, DSP-WENO_trainer/DSP-WENO_network_trainer.py:197-213)."""
    with open(path, "w") as f:
        f.write("Weights\n")
        for k in range(4):
            f.write(f"Layer {k + 1}\nBEGIN\n")
            for row in W[k]:
                f.write(" ".join("%.18e" % v for v in row) + "\n")
            f.write("END\n")
        f.write("Biases\n")
        for k in range(4):
            f.write(f"Layer {k + 1}\nBEGIN\n")
            for v in b[k]:
                f.write("%.18e\n" % v)
            f.write("END\n")


def xavier_network(seed: int = 6008) -> tuple[np.ndarray, np.ndarray]:
    """Xavier-uniform weights for the 5-5-5-5-5 network and PyTorch-default
    uniform(-1/sqrt(5), 1/sqrt(5)) biases (DSP-WENO_network_trainer.py:59-60)."""
    rng = np.random.default_rng(seed)
    a = np.sqrt(6.0 / (5 + 5))
    W = rng.uniform(-a, a, size=(4, 5, 5))
    b = rng.uniform(-1 / np.sqrt(5), 1 / np.sqrt(5), size=(4, 5))
    return W, b


def make_desc(model="euler", flux="kepes_tecno4_roe", recon="sp_weno", nx=64, ny=1, nz=1,
              x=(0.0, 1.0), y=(0.0, 1.0), z=(0.0, 1.0), bc="periodic", gamma=1.4, gas_const=1.0,
              prandtl=1.0, mu_ref=0.0, mu_model="constant", T_ref=1.0, T_0=1.0, omega=1.0,
              lin_vel=(1.0, 0.0, 0.0), cfl=0.4, final_time=1.0, max_iter=1 << 30, t_stamps=1,
              ec1_fix=False, precision="fp64", time_scheme="ssprk3", network=None,
              bc_state=None) -> Desc:
    """Build a dspw_desc from keyword arguments (names follow param.in)."""
    d = Desc()
    d.abi_version = ABI_VERSION
    d.model = MODEL[model]
    d.flux = FLUX[flux]
    d.recon = RECON[recon]
    d.time_scheme = TIME[time_scheme]
    d.precision = PRECISION[precision]
    d.nx, d.ny, d.nz = int(nx), int(ny), int(nz)
    if isinstance(bc, str):
        bc = [bc] * 6
    for i, k in enumerate(bc):
        d.bc[i] = BC[k]
    d.ec1_fix = int(bool(ec1_fix))
    d.mu_model = MU[mu_model]
    d.max_iter = int(max_iter)
    d.t_stamps = int(t_stamps)
    d.xmin, d.xmax = map(float, x)
    d.ymin, d.ymax = map(float, y)
    d.zmin, d.zmax = map(float, z)
    d.gamma, d.gas_const, d.prandtl = float(gamma), float(gas_const), float(prandtl)
    d.mu_ref, d.T_ref, d.T_0, d.omega = float(mu_ref), float(T_ref), float(T_0), float(omega)
    for i in range(3):
        d.lin_vel[i] = float(lin_vel[i])
    d.cfl, d.final_time = float(cfl), float(final_time)
    if bc_state is not None:
        for f in range(6):
            for c in range(5):
                d.bc_state[f][c] = float(bc_state[f][c])
    if network is not None:
        W, b = network
        for l in range(4):
            for j in range(5):
                d.nn_b[l][j] = float(b[l][j])
                for k in range(5):
                    d.nn_w[l][j][k] = float(W[l][j][k])
    return d


def set_training_box(d: Desc, lo, hi) -> Desc:
    """Give the descriptor's network a training box (nn_use_box): stencils
    whose five network inputs fall outside [lo, hi] are reconstructed by plain
    SP-WENO in the FP32 form.  lo / hi usually come from Trainer.box()."""
    d.nn_use_box = 1
    for k in range(5):
        d.nn_feat_lo[k] = float(lo[k])
        d.nn_feat_hi[k] = float(hi[k])
    return d


def nvar(d: Desc) -> int:
    return 1 if d.model in (0, 1) else 5


_LIB = None


def lib():
    """Load libdspw.so (built in-tree).  Raises if it is missing: there is no
    fallback path."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.environ.get("DSPW_LIB", str(LIB_PATH))
    if not os.path.exists(path):
        raise RuntimeError(f"libdspw.so not found at {path}; run __graft_entry__.build()")
    L = C.CDLL(path)
    P, I, D, LL = C.c_void_p, C.c_int, C.c_double, C.c_longlong
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    sig = {
        "dspw_error_string": (C.c_char_p, [I]),
        "dspw_version": (I, []),
        "dspw_create": (I, [C.POINTER(Desc), C.POINTER(P)]),
        "dspw_create_batch": (I, [C.POINTER(Desc), I, C.POINTER(P)]),
        "dspw_destroy": (I, [P]),
        "dspw_upload_prim": (I, [P, I, dp]),
        "dspw_download_prim": (I, [P, I, dp]),
        "dspw_download_cons": (I, [P, I, dp]),
        "dspw_compute_dt": (I, [P, I, C.POINTER(D)]),
        "dspw_residual": (I, [P, I, dp]),
        "dspw_stage": (I, [P, I, D]),
        "dspw_step": (I, [P, I, D]),
        "dspw_run": (I, [P, I, C.POINTER(I)]),
        "dspw_globals": (I, [P, I, C.POINTER(Globals)]),
        "dspw_last_status": (I, [P, C.POINTER(StatusOut)]),
        "dspw_errors": (I, [P, I, I, dp, dp]),
        "dspw_sync": (I, [P]),
        "dspw_reconstruct_batch": (I, [C.POINTER(Desc), dp, LL, dp, dp, C.POINTER(LL)]),
        "dspw_globals_noalloc": (I, [C.POINTER(Desc), P, LL, I, P, P]),
        "dspw_profile_step": (I, [P, dp, C.c_char_p, I, C.POINTER(I)]),
        "dspw_tune": (I, [P, I, C.POINTER(D), C.POINTER(D)]),
        "dspw_entropy_check": (I, [P, I, C.POINTER(D), C.POINTER(LL)]),
        "dspw_diag_enable": (I, [P, I]),
        "dspw_diag_pending": (I, [P, I, C.POINTER(I), C.POINTER(LL)]),
        "dspw_diag_read": (I, [P, I, dp, I, C.POINTER(I)]),
        "dspw_snap_enable": (I, [P, I]),
        "dspw_snap_pending": (I, [P, I, C.POINTER(I), C.POINTER(LL)]),
        "dspw_snap_read": (I, [P, I, dp, C.POINTER(D), C.POINTER(I)]),
        "dspw_stream": (P, [P]),
        "dspw_device_state": (I, [P, I, C.POINTER(P), C.POINTER(LL), C.POINTER(I)]),
        "dspw_halo_view": (I, [P, I, I, C.POINTER(HaloOut)]),
        "dspw_nccl_id": (I, [C.c_char_p]),
        "dspw_slab_connect": (I, [P, C.c_char_p, I, I]),
        "dspw_trainer_create": (I, [C.POINTER(TrainCfg), dp, dp, C.POINTER(P)]),
        "dspw_trainer_destroy": (I, [P]),
        "dspw_trainer_set_data": (I, [P, dp, dp, LL]),
        "dspw_trainer_collect": (I, [P, P, LL, C.POINTER(LL)]),
        "dspw_trainer_epoch": (I, [P, C.POINTER(D)]),
        "dspw_trainer_loss_grad": (I, [P, dp, dp, I, C.POINTER(D), dp, dp]),
        "dspw_trainer_get_params": (I, [P, dp, dp]),
        "dspw_trainer_info": (I, [P, C.POINTER(LL), dp]),
        "dspw_trainer_box": (I, [P, dp, dp]),
        "dspw_trainer_eval": (I, [P, C.POINTER(D)]),
        "dspw_trainer_export": (I, [P, C.c_void_p, LL, C.POINTER(LL)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def reconstruct_batch(desc: Desc, u4) -> tuple[np.ndarray, np.ndarray, int]:
    """GPU reconstruction of stencils u4 (n, 4) with desc.recon / desc.precision."""
    u = np.ascontiguousarray(u4, dtype=np.float64).reshape(-1, 4)
    n = u.shape[0]
    l = np.zeros(n)
    r = np.zeros(n)
    acts = C.c_longlong()
    check(lib().dspw_reconstruct_batch(C.byref(desc), u.reshape(-1), n, l, r, C.byref(acts)),
          "dspw_reconstruct_batch")
    return l, r, acts.value


class Trainer:
    """Owner of a dspw_trainer: GPU training of the DSP-WENO network.
    Defaults follow DSP-WENO_trainer/config.py (lr 1e-3, betas (0.5, 0.9),
    weight decay 1e-5, seed 6008) with batch 8192."""

    def __init__(self, network, lr=1e-3, betas=(0.5, 0.9), weight_decay=1e-5, eps=1e-8, batch=8192, seed=6008,
                 bf16=True, collect_stride=1):
        W, b = network
        cfg = TrainCfg(lr=lr, beta1=betas[0], beta2=betas[1], weight_decay=weight_decay, eps=eps, batch=batch,
                       seed=seed, compute_bf16=int(bool(bf16)), collect_stride=int(collect_stride))
        h = C.c_void_p()
        check(lib().dspw_trainer_create(C.byref(cfg), np.ascontiguousarray(W, dtype=np.float64).reshape(-1),
                                        np.ascontiguousarray(b, dtype=np.float64).reshape(-1), C.byref(h)),
              "dspw_trainer_create")
        self.h = h

    def close(self):
        if self.h:
            lib().dspw_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_data(self, stencils, targets):
        s = np.ascontiguousarray(stencils, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        check(lib().dspw_trainer_set_data(self.h, s, t, len(s) // 4), "dspw_trainer_set_data")

    def collect(self, solver, max_pairs):
        n = C.c_longlong()
        check(lib().dspw_trainer_collect(self.h, solver.h, int(max_pairs), C.byref(n)), "dspw_trainer_collect")
        return n.value

    def epoch(self):
        v = C.c_double()
        check(lib().dspw_trainer_epoch(self.h, C.byref(v)), "dspw_trainer_epoch")
        return v.value

    def loss_grad(self, stencils, targets):
        s = np.ascontiguousarray(stencils, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        loss = C.c_double()
        gw, gb = np.zeros(100), np.zeros(20)
        check(lib().dspw_trainer_loss_grad(self.h, s, t, len(s) // 4, C.byref(loss), gw, gb), "dspw_trainer_loss_grad")
        return loss.value, gw.reshape(4, 5, 5), gb.reshape(4, 5)

    def eval(self):
        v = C.c_double()
        check(lib().dspw_trainer_eval(self.h, C.byref(v)), "dspw_trainer_eval")
        return v.value

    def export_rows(self):
        """The valid samples as rows of the reference trainer's data file
        (dspw_trainer_export; 23 columns, see dspw.traindata)."""
        n = C.c_longlong()
        check(lib().dspw_trainer_export(self.h, None, 0, C.byref(n)), "dspw_trainer_export")
        rows = np.zeros((n.value, 23))
        got = C.c_longlong()
        check(lib().dspw_trainer_export(self.h, rows.ctypes.data_as(C.c_void_p), n.value, C.byref(got)),
              "dspw_trainer_export")
        return rows[:got.value]

    def params(self):
        w, b = np.zeros(100), np.zeros(20)
        check(lib().dspw_trainer_get_params(self.h, w, b), "dspw_trainer_get_params")
        return w.reshape(4, 5, 5), b.reshape(4, 5)

    def info(self):
        n = C.c_longlong()
        fm = np.zeros(5)
        check(lib().dspw_trainer_info(self.h, C.byref(n), fm), "dspw_trainer_info")
        return n.value, fm

    def box(self):
        """(lo, hi): the range of each network input over the training data
        (dspw_trainer_box), for set_training_box."""
        lo, hi = np.zeros(5), np.zeros(5)
        check(lib().dspw_trainer_box(self.h, lo, hi), "dspw_trainer_box")
        return lo, hi


class DspwError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)}")


def check(code, where=""):
    if code != 0:
        raise DspwError(code, where)
    return code


class Solver:
    """Thin owner of a dspw_handle (one problem or a batch)."""

    def __init__(self, descs):
        if isinstance(descs, Desc):
            descs = [descs]
        self.descs = list(descs)
        arr = (Desc * len(self.descs))(*self.descs)
        h = C.c_void_p()
        check(lib().dspw_create_batch(arr, len(self.descs), C.byref(h)), "dspw_create_batch")
        self.h = h

    def close(self):
        if self.h:
            lib().dspw_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, p=0):
        d = self.descs[p]
        return (nvar(d), d.nz, d.ny, d.nx)

    def upload_prim(self, prim, p=0):
        a = np.ascontiguousarray(prim, dtype=np.float64).reshape(self.shape(p))
        check(lib().dspw_upload_prim(self.h, p, a), "dspw_upload_prim")

    def prim(self, p=0):
        a = np.empty(self.shape(p))
        check(lib().dspw_download_prim(self.h, p, a), "dspw_download_prim")
        return a

    def cons(self, p=0):
        a = np.empty(self.shape(p))
        check(lib().dspw_download_cons(self.h, p, a), "dspw_download_cons")
        return a

    def residual(self, p=0):
        a = np.empty(self.shape(p))
        check(lib().dspw_residual(self.h, p, a), "dspw_residual")
        return a

    def compute_dt(self, p=0):
        v = C.c_double()
        check(lib().dspw_compute_dt(self.h, p, C.byref(v)), "dspw_compute_dt")
        return v.value

    def step(self, n=1, fixed_dt=0.0):
        check(lib().dspw_step(self.h, int(n), float(fixed_dt)), "dspw_step")

    def stage(self, rk, dt=0.0):
        check(lib().dspw_stage(self.h, int(rk), float(dt)), "dspw_stage")

    def halo_view(self, p=0, rk=0) -> HaloOut:
        v = HaloOut()
        check(lib().dspw_halo_view(self.h, int(p), int(rk), C.byref(v)), "dspw_halo_view")
        return v

    def run(self, chunk=64):
        s = C.c_int()
        check(lib().dspw_run(self.h, int(chunk), C.byref(s)), "dspw_run")
        return s.value

    def entropy_check(self, p=0):
        """(largest relative one-step rise of the total entropy since the
        upload, steps checked) (dspw_entropy_check)."""
        r, n = C.c_double(), C.c_longlong()
        check(lib().dspw_entropy_check(self.h, p, C.byref(r), C.byref(n)), "dspw_entropy_check")
        return r.value, n.value

    def diag_enable(self, capacity=256):
        """Record the per-step diagnostics rows (dspw_diag_enable); 0 stops."""
        check(lib().dspw_diag_enable(self.h, int(capacity)), "dspw_diag_enable")

    def diag_rows(self, p=0):
        """Pending per-step rows of problem p as an (n, DIAG_COLS) array (read
        and removed), and the count of rows dropped so far."""
        n, dropped = C.c_int(), C.c_longlong()
        check(lib().dspw_diag_pending(self.h, p, C.byref(n), C.byref(dropped)), "dspw_diag_pending")
        rows = np.zeros((n.value, DIAG_COLS))
        got = C.c_int()
        check(lib().dspw_diag_read(self.h, p, rows, n.value, C.byref(got)), "dspw_diag_read")
        return rows[:got.value], dropped.value

    def snap_enable(self, slots=4):
        """Take a snapshot whenever a step ends on an output time stamp
        (dspw_snap_enable); 0 stops."""
        check(lib().dspw_snap_enable(self.h, int(slots)), "dspw_snap_enable")

    def snapshots(self, p=0):
        """Pending snapshots of problem p as a list of (time, iter, prim) (read
        and removed), and the count of snapshots dropped so far."""
        n, dropped = C.c_int(), C.c_longlong()
        check(lib().dspw_snap_pending(self.h, p, C.byref(n), C.byref(dropped)), "dspw_snap_pending")
        out = []
        for _ in range(n.value):
            a = np.empty(self.shape(p))
            t, it = C.c_double(), C.c_int()
            check(lib().dspw_snap_read(self.h, p, a, C.byref(t), C.byref(it)), "dspw_snap_read")
            out.append((t.value, it.value, a))
        return out, dropped.value

    def globals(self, p=0):
        g = Globals()
        check(lib().dspw_globals(self.h, p, C.byref(g)), "dspw_globals")
        return g

    def status(self):
        s = StatusOut()
        lib().dspw_last_status(self.h, C.byref(s))
        return s

    def errors(self, exact, comp=0, p=0):
        e = np.zeros(3)
        a = np.ascontiguousarray(exact, dtype=np.float64)
        check(lib().dspw_errors(self.h, p, comp, a, e), "dspw_errors")
        return e

    def tune(self, reps=5):
        """Pick the launch grid of every sweep by timing (dspw_tune); returns
        the summed sweep times (ms) with the default and the chosen grids."""
        b, a = C.c_double(), C.c_double()
        check(lib().dspw_tune(self.h, int(reps), C.byref(b), C.byref(a)), "dspw_tune")
        return b.value, a.value

    def profile_step(self):
        """Durations (ms) of every kernel launch of one un-graphed step."""
        ms = np.zeros(64)
        names = C.create_string_buffer(16 * 64)
        n = C.c_int()
        check(lib().dspw_profile_step(self.h, ms, names, 64, C.byref(n)), "dspw_profile_step")
        raw = names.raw
        return [(raw[16 * i:16 * i + 16].split(b"\0")[0].decode(), float(ms[i])) for i in range(n.value)]

    def stream_ptr(self):
        return lib().dspw_stream(self.h)

    def sync(self):
        check(lib().dspw_sync(self.h), "dspw_sync")
