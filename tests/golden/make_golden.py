"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference solvers are compiled from their own sources by oracle/Makefile
(`make -C oracle ref`, needs the reference tree) and driven through the
harness in oracle/ref_harness.  Every fixture is produced by the reference's
code, never by the project's oracle or kernels:

  faces_euler.npz   Euler/NS face fluxes num_flux(P, V, n) for every TeCNO and
                    central flux x reconstruction, random 4-cell stencils, all
                    three normals (enflo/src/num_flux.cc:12-72)
  faces_scalar.npz  scalar face fluxes (enflo_scalar/src_scalar/num_flux.cc:12-57)
  recon.npz         sp_weno_rec for corr types 0/1/2 (limiter.h:193-252) and
                    Neural_Network::forward (neural_network.cc:16-77) on random
                    and structured stencils
  runs.npz          whole solver runs: initial primitive state (the reference's
                    own fparser-evaluated IC), final conserved state, time,
                    iteration count and last dt
  ooc.npz           config-1 L1/L2/Linf errors (LinAdvTest2, Nx=100..400)
  dsp_weno.txt      the shipped network weights (enflo/networks/dsp_weno.txt)

Run from the repository root (after `make -C oracle ref REF=DIR`):

    python tests/golden/make_golden.py --ref DIR
"""
from __future__ import annotations

import os
import shutil
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "dsp-weno_b200"))
import oracle as O  # noqa: E402

def _ref_tree() -> Path:
    """The reference project tree: argument --ref DIR, else the environment
    variable DSPW_REFERENCE_DIR (the same tree oracle/Makefile compiles)."""
    if "--ref" in sys.argv:
        return Path(sys.argv[sys.argv.index("--ref") + 1])
    env = os.environ.get("DSPW_REFERENCE_DIR")
    if not env:
        raise SystemExit("make_golden.py: give the reference tree with --ref DIR or DSPW_REFERENCE_DIR")
    return Path(env)


REF_TREE = _ref_tree() if __name__ == "__main__" else None
OUT = Path(__file__).resolve().parent
NET = str(OUT / "dsp_weno.txt")

EULER_FLUXES = ["kepes_tecno4_roe", "kepes_tecno_roe", "kepes_tecno4_rusanov", "kepes_tecno_rusanov",
                "kep_tecno_roe", "roe_tecno_roe", "roe_tecno4_roe", "kepec4", "kepec", "kep", "kep4",
                "roe_ec", "roe_ec4"]
RECONS = ["sp_weno", "sp_wenoc", "sp_weno_dl", "sp_weno_corr2"]

SHU_IC = dict(density="3.857143*(x<-4) + (1+0.2*sin(5*x))*(x>=-4)", xvelocity="2.629369*(x<-4)",
              pressure="10.33333*(x<-4) + 1*(x>=-4)")
KH_IC = dict(density="1+(abs(y-0.5)<0.25)", xvelocity="-0.5+(abs(y-0.5)<0.25)",
             yvelocity="0.01*sin(4*pi*x)", pressure="2.5")
VORTEX_IC = dict(  # isentropic vortex, strength 5, gamma 1.4 (enflo/examples/2D/IsentropicVortex)
    density="pow(1-(0.4)*25/(8*1.4*pi*pi)*exp(1-x*x-y*y),1/0.4)",
    xvelocity="1-5/(2*pi)*exp(0.5*(1-x*x-y*y))*y",
    yvelocity="5/(2*pi)*exp(0.5*(1-x*x-y*y))*x",
    pressure="pow(1-(0.4)*25/(8*1.4*pi*pi)*exp(1-x*x-y*y),1.4/0.4)")
TGV_IC = dict(density="1", xvelocity="sin(x)*cos(y)*cos(z)", yvelocity="-cos(x)*sin(y)*cos(z)",
              zvelocity="0", pressure="1/(1.4*M*M)+(cos(2*x)+cos(2*y))*(cos(2*z)+2)/16")
# a periodic flow without the symmetries of TGV_IC: ENO compares two jumps to
# pick its stencil, and the exact ties of a symmetric state are then decided by
# rounding, where the device's viscous sums (another order) differ from the
# reference's by ulps
SKEW_IC = dict(density="1+0.2*sin(x+0.37)*cos(2*y+0.91)+0.1*sin(z+1.3)",
               xvelocity="sin(x+0.2)*cos(y+0.7)*cos(z+0.5)", yvelocity="-cos(x+0.9)*sin(y+0.3)*cos(z+1.1)",
               zvelocity="0.3*sin(x+y+0.45)", pressure="1/(1.4*M*M)+0.3*sin(x+2*z+0.61)")


def euler_cfg(flux="kepes_tecno4_roe", recon="sp_weno", **kw):
    c = dict(model="euler", x=(0, 1), Nx=8, Ny=2, Nz=2, cfl=0.4, final_time=1.0, reconstruct=recon,
             net_file=NET, flux=flux, ic=dict(density="1", pressure="1"), bc="periodic")
    c.update(kw)
    return c


def random_prim_stencils(rng, n, ncell=4):
    P = np.zeros((n, ncell, 5))
    P[:, :, 0] = rng.uniform(0.1, 4.0, (n, ncell))
    P[:, :, 1:4] = rng.normal(0.0, 1.5, (n, ncell, 3))
    P[:, :, 4] = rng.uniform(0.1, 6.0, (n, ncell))
    # a third of the stencils are smooth (small jumps) so the log-mean series
    # branch and the smooth SP-WENO regions are exercised
    m = n // 3
    base = P[:m, 1:2, :]
    P[:m] = base * (1.0 + rng.normal(0.0, 1e-3, (m, ncell, 5)))
    # a sixth are 1-D / 2-D states (zero transverse velocity)
    P[m:m + n // 6, :, 2:4] = 0.0
    return P


def gen_faces_euler(rng):
    out = {}
    for flux in EULER_FLUXES:
        # the central fluxes do not reconstruct: one reconstruction suffices
        for recon in (RECONS if "tecno" in flux else RECONS[:1]):
            for ec1 in ((0, 1) if "roe" in flux and "tecno" in flux else (0,)):
                R = O.RefEuler(euler_cfg(flux, recon, EC1_fix="yes" if ec1 else "no",
                                         y=(0, 0.5), z=(0, 0.25)))
                n = 150
                P = random_prim_stencils(rng, n)
                dirs = np.arange(n) % 3
                F = np.zeros((n, 5)); V = np.zeros((n, 4, 5))
                for t in range(n):
                    F[t], V[t] = R.face_flux(P[t], int(dirs[t]))
                key = f"{flux}|{recon}|{ec1}"
                out[key + "|P"] = P
                out[key + "|dir"] = dirs
                out[key + "|F"] = F
                out[key + "|V"] = V
                out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    np.savez_compressed(OUT / "faces_euler.npz", **out)


def gen_faces_scalar(rng):
    out = {}
    for model, fluxes in (("linadv", ["lin_ec", "lin_ec4", "lin_tecno", "lin_tecno4"]),
                          ("burgers", ["bur_ec", "bur_ec4", "bur_tecno", "bur_tecno4"])):
        for flux in fluxes:
            for recon in RECONS:
                cfg = dict(model=model, x=("-pi", "pi"), y=(0, 0.5), z=(0, 0.25), Nx=16, Ny=2, Nz=2, cfl=0.5,
                           final_time=0.5, reconstruct=recon, net_file=NET, flux=flux, ic="sin(x)",
                           vel=(1.0, -0.5, 0.25), bc="periodic")
                R = O.RefScalar(cfg)
                n = 300
                U = rng.normal(0, 1, (n, 4))
                U[: n // 3] = np.sin(rng.uniform(0, 6.3, (n // 3, 1)) + 0.05 * np.arange(4)[None, :])
                dirs = np.arange(n) % 3
                F = np.array([R.face_flux(U[t], int(dirs[t])) for t in range(n)])
                key = f"{flux}|{recon}"
                out[key + "|U"] = U
                out[key + "|dir"] = dirs
                out[key + "|F"] = F
                out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    np.savez_compressed(OUT / "faces_scalar.npz", **out)


SIMPLE_RECONS = ["first", "second", "minmod", "minabs"]


def gen_faces_simple(rng):
    """Face fluxes with the reference's first-order, unlimited MUSCL and
    minmod / minabs limited reconstructions (reconstruct.cc:14-79, 162-186)
    inside the TeCNO fluxes, Euler and scalar."""
    out = {}
    for flux in ("kepes_tecno4_roe", "kepes_tecno_roe", "kepes_tecno4_rusanov", "roe_tecno_roe"):
        for recon in SIMPLE_RECONS:
            R = O.RefEuler(euler_cfg(flux, recon, EC1_fix="yes" if "roe" in flux else "no", y=(0, 0.5), z=(0, 0.25)))
            n = 120
            P = random_prim_stencils(rng, n)
            dirs = np.arange(n) % 3
            F = np.zeros((n, 5)); V = np.zeros((n, 4, 5))
            for t in range(n):
                F[t], V[t] = R.face_flux(P[t], int(dirs[t]))
            key = f"E|{flux}|{recon}|{int('roe' in flux)}"
            out[key + "|P"] = P
            out[key + "|dir"] = dirs
            out[key + "|F"] = F
            out[key + "|V"] = V
            out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    for model, flux in (("linadv", "lin_tecno4"), ("linadv", "lin_tecno"), ("burgers", "bur_tecno4"),
                        ("burgers", "bur_tecno")):
        for recon in SIMPLE_RECONS:
            cfg = dict(model=model, x=("-pi", "pi"), y=(0, 0.5), z=(0, 0.25), Nx=16, Ny=2, Nz=2, cfl=0.5,
                       final_time=0.5, reconstruct=recon, net_file=NET, flux=flux, ic="sin(x)",
                       vel=(1.0, -0.5, 0.25), bc="periodic")
            R = O.RefScalar(cfg)
            n = 200
            U = rng.normal(0, 1, (n, 4))
            U[: n // 3] = np.sin(rng.uniform(0, 6.3, (n // 3, 1)) + 0.05 * np.arange(4)[None, :])
            dirs = np.arange(n) % 3
            F = np.array([R.face_flux(U[t], int(dirs[t])) for t in range(n)])
            key = f"S|{flux}|{recon}"
            out[key + "|U"] = U
            out[key + "|dir"] = dirs
            out[key + "|F"] = F
            out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    # the standalone keps, keps4 and roe fluxes (keps.cc, keps4.cc, roe.cc)
    for flux in ("keps", "keps4", "roe"):
        R = O.RefEuler(euler_cfg(flux, "sp_weno", y=(0, 0.5), z=(0, 0.25)))
        n = 150
        P = random_prim_stencils(rng, n)
        dirs = np.arange(n) % 3
        F = np.zeros((n, 5)); V = np.zeros((n, 4, 5))
        for t in range(n):
            F[t], V[t] = R.face_flux(P[t], int(dirs[t]))
        key = f"E|{flux}|sp_weno|0"
        out[key + "|P"] = P
        out[key + "|dir"] = dirs
        out[key + "|F"] = F
        out[key + "|V"] = V
        out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    # point-wise ENO of level 2 (param.in "reconstruct eno 2", reconstruct.cc:84-110)
    for flux in ("kepes_tecno4_roe", "kepes_tecno_roe"):
        R = O.RefEuler(euler_cfg(flux, "eno 2", EC1_fix="yes", y=(0, 0.5), z=(0, 0.25)))
        n = 150
        P = random_prim_stencils(rng, n)
        dirs = np.arange(n) % 3
        F = np.zeros((n, 5)); V = np.zeros((n, 4, 5))
        for t in range(n):
            F[t], V[t] = R.face_flux(P[t], int(dirs[t]))
        key = f"E|{flux}|eno2|1"
        out[key + "|P"] = P
        out[key + "|dir"] = dirs
        out[key + "|F"] = F
        out[key + "|V"] = V
        out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    for model, flux in (("linadv", "lin_tecno4"), ("burgers", "bur_tecno4")):
        cfg = dict(model=model, x=("-pi", "pi"), y=(0, 0.5), z=(0, 0.25), Nx=16, Ny=2, Nz=2, cfl=0.5,
                   final_time=0.5, reconstruct="eno 2", net_file=NET, flux=flux, ic="sin(x)",
                   vel=(1.0, -0.5, 0.25), bc="periodic")
        R = O.RefScalar(cfg)
        n = 200
        U = rng.normal(0, 1, (n, 4))
        dirs = np.arange(n) % 3
        F = np.array([R.face_flux(U[t], int(dirs[t])) for t in range(n)])
        key = f"S|{flux}|eno2"
        out[key + "|U"] = U
        out[key + "|dir"] = dirs
        out[key + "|F"] = F
        out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    # point-wise ENO of level 3: the reference's stencils have 2 ng = 6 cells
    for flux in ("kepes_tecno4_roe", "kepes_tecno_roe", "kepes_tecno4_rusanov"):
        R = O.RefEuler(euler_cfg(flux, "eno 3", EC1_fix="yes" if "roe" in flux else "no", y=(0, 0.5),
                                 z=(0, 0.25)))
        n = 150
        P = random_prim_stencils(rng, n, ncell=6)
        dirs = np.arange(n) % 3
        F = np.zeros((n, 5)); V = np.zeros((n, 6, 5))
        for t in range(n):
            F[t], V[t] = R.face_flux(P[t], int(dirs[t]))
        key = f"E|{flux}|eno3|{int('roe' in flux)}"
        out[key + "|P"] = P
        out[key + "|dir"] = dirs
        out[key + "|F"] = F
        out[key + "|V"] = V
        out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    for model, flux in (("linadv", "lin_tecno4"), ("linadv", "lin_tecno"), ("burgers", "bur_tecno4")):
        cfg = dict(model=model, x=("-pi", "pi"), y=(0, 0.5), z=(0, 0.25), Nx=16, Ny=2, Nz=2, cfl=0.5,
                   final_time=0.5, reconstruct="eno 3", net_file=NET, flux=flux, ic="sin(x)",
                   vel=(1.0, -0.5, 0.25), bc="periodic")
        R = O.RefScalar(cfg)
        n = 200
        U = rng.normal(0, 1, (n, 6))
        dirs = np.arange(n) % 3
        F = np.array([R.face_flux(U[t], int(dirs[t])) for t in range(n)])
        key = f"S|{flux}|eno3"
        out[key + "|U"] = U
        out[key + "|dir"] = dirs
        out[key + "|F"] = F
        out[key + "|h"] = np.array([R.dx, R.dy, R.dz])
    np.savez_compressed(OUT / "faces_simple.npz", **out)


def structured_stencils(rng):
    """Stencils that hit the special branches: flat, linear (theta = 1), theta
    = -1 (psi = -1), extrema, jumps, tiny jumps, large magnitudes."""
    S = [
        [1, 1, 1, 1], [0, 0, 0, 0], [0, 1, 2, 3], [3, 2, 1, 0], [0, 1, 1, 0], [1, 0, 0, 1],
        [0, 0, 1, 1], [1, 1, 0, 0], [0, 1, 0, 1], [1, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0],
        [0, 1, 3, 4], [0, 1, 2, 4], [0, 2, 3, 4], [-1, 0, 1, 0], [5, 1, 2, 6], [0, 1e-14, 2e-14, 3e-14],
        [1, 1 + 1e-14, 1 + 3e-14, 1 + 6e-14], [100, 101, 103, 104], [-100, -90, -70, -60], [0.5, 0.5, 0.7, 0.7],
        [1, 2, 2, 1], [2, 1, 1, 2], [0, 1, 1, 2], [0, 2, 2, 3],
    ]
    S = np.array(S, dtype=np.float64)
    lin = np.cumsum(rng.normal(0, 1, (40, 1)) * np.ones((1, 4)), axis=1) + rng.normal(0, 1, (40, 1))
    return np.concatenate([S, lin])


def gen_recon(rng):
    n = 4000
    U = rng.normal(0, 1, (n, 4))
    U[: n // 4] = np.sin(rng.uniform(0, 6.3, (n // 4, 1)) + rng.uniform(0.01, 0.5, (n // 4, 1)) * np.arange(4)[None, :])
    U[n // 4: n // 2] = rng.uniform(-1, 1, (n // 4, 4)) * 10.0 ** rng.uniform(-3, 2, (n // 4, 1))
    U = np.concatenate([U, structured_stencils(rng)])
    out = {"U": U}
    for corr in (0, 1, 2):
        L = np.zeros(len(U)); Rr = np.zeros(len(U))
        for t in range(len(U)):
            L[t], Rr[t] = O.ref_sp_weno(U[t], corr)
        out[f"spw{corr}_l"] = L
        out[f"spw{corr}_r"] = Rr
    Rh = O.RefEuler(euler_cfg("kepes_tecno4_roe", "sp_weno_dl"))
    mask = np.abs(U[:, 2] - U[:, 1]) >= 1e-15
    out["nn_mask"] = mask
    L = np.zeros(len(U)); Rr = np.zeros(len(U))
    for t in range(len(U)):
        if mask[t]:
            L[t], Rr[t] = Rh.nn_forward(U[t])
    out["nn_l"] = L
    out["nn_r"] = Rr
    a = 10.0 ** rng.uniform(-3, 3, 2000)
    b = a * (1.0 + rng.normal(0, 0.3, 2000) * (rng.uniform(0, 1, 2000) < 0.5)) + a * rng.uniform(0, 5, 2000) * (
        rng.uniform(0, 1, 2000) >= 0.5)
    b = np.abs(b) + 1e-6
    out["la_a"] = a
    out["la_b"] = b
    out["la"] = np.array([Rh.L.refE_logavg(x, y) for x, y in zip(a, b)])
    np.savez_compressed(OUT / "recon.npz", **out)


def run_cases():
    """(name, kind, cfg, nsteps, fixed_dt)"""
    bc1d = ["neumann", "neumann", "periodic", "periodic", "periodic", "periodic"]
    cases = []
    for recon in ("sp_weno", "sp_wenoc", "sp_weno_dl"):
        cases.append((f"linadv_{recon}", "S", dict(model="linadv", x=("-pi", "pi"), Nx=100, Ny=2, Nz=2, cfl=0.5,
                      final_time=0.5, reconstruct=recon, net_file=NET, flux="lin_tecno4", ic="pow(sin(x),4)",
                      exact="pow(sin(x-t),4)", bc="periodic", time_stamps=5), 100000, 0.0))
    cases.append(("burgers_wenoc", "S", dict(model="burgers", x=("-pi", "pi"), Nx=80, Ny=2, Nz=2, cfl=0.5,
                  final_time=0.5, reconstruct="sp_wenoc", net_file=NET, flux="bur_tecno4", ic="0.5+sin(x)",
                  bc="periodic", time_stamps=5), 40, 0.0))
    cases.append(("burgers_wall_dl", "S", dict(model="burgers", x=(-1, 1), Nx=60, Ny=2, Nz=2, cfl=0.4,
                  final_time=0.3, reconstruct="sp_weno_dl", net_file=NET, flux="bur_tecno", ic="sin(pi*x)",
                  bc=["wall", "wall", "periodic", "periodic", "periodic", "periodic"], time_stamps=3), 40, 0.0))
    for recon in ("sp_weno", "sp_weno_dl"):
        cases.append((f"shuosher_{recon}", "E", euler_cfg("kepes_tecno4_roe", recon, x=(-5, 5), Nx=200, cfl=0.4,
                      final_time=1.8, ic=SHU_IC, bc=bc1d, time_stamps=5), 120, 0.0))
    cases.append(("kh_sp_weno", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", Nx=32, Ny=32, ic=KH_IC, dim=2), 20, 0.0))
    cases.append(("kh_sp_weno_dl", "E", euler_cfg("kepes_tecno4_roe", "sp_weno_dl", Nx=32, Ny=32, ic=KH_IC, dim=2),
                  10, 0.0))
    for flux in ("kepes_tecno_roe", "kepes_tecno4_rusanov", "kepes_tecno_rusanov", "kep_tecno_roe",
                 "roe_tecno_roe", "roe_tecno4_roe"):
        cases.append((f"kh_{flux}", "E", euler_cfg(flux, "sp_wenoc", Nx=16, Ny=16, ic=KH_IC, dim=2,
                      EC1_fix="yes" if flux.startswith(("kepes_tecno4_roe", "roe")) else "no"), 6, 0.0))
    wall_ic = dict(density="1+0.5*exp(-40*((x-0.4)^2+(y-0.6)^2))", xvelocity="0.3", yvelocity="-0.2",
                   pressure="1+0.5*exp(-40*((x-0.4)^2+(y-0.6)^2))")
    cases.append(("wall2d", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", Nx=24, Ny=20, ic=wall_ic, dim=2,
                  bc=["wall", "wall", "wall", "wall", "periodic", "periodic"]), 15, 0.0))
    cases.append(("neumann2d", "E", euler_cfg("kepes_tecno4_roe", "sp_weno_dl", Nx=20, Ny=24, ic=wall_ic, dim=2,
                  bc=["neumann", "neumann", "wall", "neumann", "periodic", "periodic"]), 12, 0.0))
    cases.append(("vortex", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", x=(-5, 5), y=(-5, 5), Nx=32, Ny=32,
                  ic=VORTEX_IC, dim=2, final_time=10.0), 10, 0.0))
    cases.append(("euler3d", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", x=(0, "2*pi"), y=(0, "2*pi"),
                  z=(0, "2*pi"), Nx=8, Ny=6, Nz=5, ic=TGV_IC, dim=3, constants={"M": 0.3}), 4, 0.0))
    cases.append(("tgv_ns", "E", euler_cfg("kepes_tecno4_roe", "sp_weno_dl", model="ns_es", x=(0, "2*pi"),
                  y=(0, "2*pi"), z=(0, "2*pi"), Nx=8, Ny=8, Nz=8, ic=TGV_IC, dim=3, constants={"M": 0.1},
                  mu_ref=1 / 1600, prandtl=0.71, final_time=10.0), 3, 0.0))
    cases.append(("tgv_ns_kep", "E", euler_cfg("kep4", "sp_weno", model="ns_kep", x=(0, "2*pi"), y=(0, "2*pi"),
                  z=(0, "2*pi"), Nx=8, Ny=8, Nz=8, ic=TGV_IC, dim=3, constants={"M": 0.2}, mu_ref=0.02,
                  prandtl=0.71, final_time=10.0), 4, 0.0))
    cases.append(("tgv_ns_kep_tecno", "E", euler_cfg("kepes_tecno4_roe", "sp_weno_dl", model="ns_kep", x=(0, "2*pi"),
                  y=(0, "2*pi"), z=(0, "2*pi"), Nx=8, Ny=8, Nz=8, ic=TGV_IC, dim=3, constants={"M": 0.1},
                  mu_ref=1 / 1600, prandtl=0.71, final_time=10.0), 3, 0.0))
    for ts in ("jameson_rk4", "rk4"):
        cases.append((f"shuosher_{ts}", "E", euler_cfg("kepes_tecno4_roe", "sp_wenoc", x=(-5, 5), Nx=100, cfl=0.4,
                      final_time=1.8, ic=SHU_IC, bc=bc1d, time_stamps=5, time_scheme=ts), 20, 0.0))
        cases.append((f"kh_{ts}", "E", euler_cfg("kepes_tecno4_roe", "sp_weno_dl", Nx=16, Ny=16, ic=KH_IC, dim=2,
                      time_scheme=ts), 6, 0.0))
        cases.append((f"burgers_{ts}", "S", dict(model="burgers", x=("-pi", "pi"), Nx=80, Ny=2, Nz=2, cfl=0.4,
                      final_time=0.5, reconstruct="sp_weno", net_file=NET, flux="bur_tecno4", ic="0.5+sin(x)",
                      bc="periodic", time_stamps=5, time_scheme=ts), 30, 0.0))
    cases.append(("tgv_ns_fixed", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", model="ns_es", x=(0, "2*pi"),
                  y=(0, "2*pi"), z=(0, "2*pi"), Nx=6, Ny=6, Nz=6, ic=TGV_IC, dim=3, constants={"M": 0.3},
                  mu_ref=0.05, prandtl=0.71, final_time=10.0), 3, 0.01))
    # point-wise ENO of level 3: the reference runs with three ghost cells and
    # six-cell face stencils (ng_cell = 3, parameter.cc:178-184, fv.cc:26)
    cases.append(("shuosher_eno3", "E", euler_cfg("kepes_tecno4_roe", "eno 3", x=(-5, 5), Nx=100, cfl=0.4,
                  final_time=1.8, ic=SHU_IC, bc=bc1d, time_stamps=5, EC1_fix="yes"), 25, 0.0))
    cases.append(("kh_eno3", "E", euler_cfg("kepes_tecno_roe", "eno 3", Nx=16, Ny=16, ic=KH_IC, dim=2,
                  EC1_fix="yes"), 6, 0.0))
    cases.append(("wall2d_eno3", "E", euler_cfg("kepes_tecno4_roe", "eno 3", Nx=14, Ny=11, ic=wall_ic, dim=2,
                  bc=["wall", "neumann", "wall", "wall", "periodic", "periodic"]), 8, 0.0))
    cases.append(("euler3d_eno3", "E", euler_cfg("roe_tecno4_roe", "eno 3", x=(0, "2*pi"), y=(0, "2*pi"),
                  z=(0, "2*pi"), Nx=7, Ny=5, Nz=4, ic=TGV_IC, dim=3, constants={"M": 0.3}), 3, 0.0))
    cases.append(("ns_eno3", "E", euler_cfg("kepes_tecno4_rusanov", "eno 3", model="ns_es", x=(0, "2*pi"),
                  y=(0, "2*pi"), z=(0, "2*pi"), Nx=6, Ny=7, Nz=5, ic=SKEW_IC, dim=3, constants={"M": 0.3},
                  mu_ref=0.05, prandtl=0.71, final_time=10.0), 3, 0.0))
    cases.append(("burgers_eno3", "S", dict(model="burgers", x=("-pi", "pi"), Nx=64, Ny=2, Nz=2, cfl=0.4,
                  final_time=0.5, reconstruct="eno 3", net_file=NET, flux="bur_tecno4", ic="0.5+sin(x)",
                  bc="periodic", time_stamps=5), 30, 0.0))
    cases.append(("linadv_wall_eno3", "S", dict(model="linadv", x=(-1, 1), Nx=50, Ny=2, Nz=2, cfl=0.5,
                  final_time=0.4, reconstruct="eno 3", net_file=NET, flux="lin_tecno", ic="exp(-20*x*x)",
                  bc=["wall", "neumann", "periodic", "periodic", "periodic", "periodic"], time_stamps=2), 30, 0.0))
    return cases


def gen_runs():
    out = {}
    for name, kind, cfg, nsteps, fixed_dt in run_cases():
        R = O.RefEuler(cfg) if kind == "E" else O.RefScalar(cfg)
        p0 = R.prim()
        R.step(nsteps, fixed_dt)
        fin = R.cons() if kind == "E" else R.get()
        info = R.info()
        out[f"{name}|prim0"] = p0
        out[f"{name}|final"] = fin
        out[f"{name}|tid"] = np.array([info["time"], info["iter"], info["dt"], nsteps, fixed_dt])
        out[f"{name}|h"] = np.array([R.dx, R.dy, R.dz])
        print(f"  run {name}: {R.nx}x{R.ny}x{R.nz} iter={info['iter']} t={info['time']:.6g}")
    np.savez_compressed(OUT / "runs.npz", **out)


DIAG_CASES = ("linadv_sp_weno", "burgers_wenoc", "burgers_wall_dl", "shuosher_sp_weno", "shuosher_jameson_rk4",
              "kh_sp_weno", "kh_sp_weno_dl", "kh_rk4", "wall2d", "neumann2d", "vortex", "euler3d", "tgv_ns",
              "tgv_ns_kep", "tgv_ns_kep_tecno")
DIAG_STEPS = 6


def gen_diag():
    """Per-step diagnostics rows of the reference (compute_global,
    compute_residual_norm, find_vorticity) for the first steps of some runs."""
    out = {}
    for name, kind, cfg, nsteps, fixed_dt in run_cases():
        if name not in DIAG_CASES:
            continue
        R = O.RefEuler(cfg) if kind == "E" else O.RefScalar(cfg)
        out[f"{name}|rows"] = R.step_diag(min(nsteps, DIAG_STEPS), fixed_dt)
        print(f"  diag {name}: {out[name + '|rows'].shape[0]} rows")
    np.savez_compressed(OUT / "diag.npz", **out)


def output_cases():
    """(name, kind, cfg) of short runs whose solution files (FV::output at t = 0
    and at every time stamp) are kept as golden text."""
    bc1d = ["neumann", "neumann", "periodic", "periodic", "periodic", "periodic"]
    wall_ic = dict(density="1+0.5*exp(-40*((x-0.4)^2+(y-0.6)^2))", xvelocity="0.3", yvelocity="-0.2*x",
                   pressure="1+0.5*exp(-40*((x-0.4)^2+(y-0.6)^2))")
    return [
        ("kh_out", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", Nx=16, Ny=16, ic=KH_IC, dim=2, final_time=0.02,
                                  time_stamps=2)),
        ("wall_out", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", Nx=12, Ny=10, ic=wall_ic, dim=2,
                                    bc=["wall", "wall", "wall", "neumann", "periodic", "periodic"], final_time=0.01,
                                    time_stamps=2)),
        ("shu_out", "E", euler_cfg("kepes_tecno4_roe", "sp_weno_dl", x=(-5, 5), Nx=50, cfl=0.4, final_time=0.05,
                                   ic=SHU_IC, bc=bc1d, time_stamps=2)),
        ("tgv_out", "E", euler_cfg("kepes_tecno4_roe", "sp_weno", model="ns_es", x=(0, "2*pi"), y=(0, "2*pi"),
                                   z=(0, "2*pi"), Nx=6, Ny=6, Nz=6, ic=TGV_IC, dim=3, constants={"M": 0.3},
                                   mu_ref=0.05, prandtl=0.71, final_time=0.02, time_stamps=1)),
        ("linadv_out", "S", dict(model="linadv", x=("-pi", "pi"), Nx=40, Ny=2, Nz=2, cfl=0.5, final_time=0.1,
                                 reconstruct="sp_weno", net_file=NET, flux="lin_tecno4", ic="pow(sin(x),4)",
                                 bc="periodic", time_stamps=2)),
    ]


def gen_output():
    out = {}
    for name, kind, cfg in output_cases():
        R = O.RefEuler(cfg) if kind == "E" else O.RefScalar(cfg)
        files = R.run_outputs()
        for fn, text in files.items():
            out[f"{name}|{fn}"] = np.array(text)
        print(f"  output {name}: {sorted(files)}")
    np.savez_compressed(OUT / "output.npz", **out)


def gen_ooc():
    out = {}
    for recon in ("sp_weno", "sp_wenoc", "sp_weno_dl"):
        errs = []
        for nx in (100, 200, 400):
            cfg = dict(model="linadv", x=("-pi", "pi"), Nx=nx, Ny=2, Nz=2, cfl=0.5, final_time=0.5,
                       reconstruct=recon, net_file=NET, flux="lin_tecno4", ic="pow(sin(x),4)",
                       exact="pow(sin(x-t),4)", bc="periodic", time_stamps=5)
            errs.append(O.RefScalar(cfg).run_errors())
        out[recon] = np.array(errs)
        print(f"  ooc {recon}: L1 = {out[recon][:, 0]}")
    np.savez_compressed(OUT / "ooc.npz", **out)


def main():
    if not O.ref_available():
        raise SystemExit("build the reference checker first: make -C oracle ref")
    shutil.copyfile(REF_TREE / "enflo" / "networks" / "dsp_weno.txt", OUT / "dsp_weno.txt")
    rng = np.random.default_rng(20240611)
    gen_faces_euler(rng)
    gen_faces_scalar(rng)
    gen_recon(rng)
    gen_runs()
    gen_ooc()
    gen_faces_simple(np.random.default_rng(20240612))
    gen_diag()
    gen_output()


if __name__ == "__main__":
    main()
