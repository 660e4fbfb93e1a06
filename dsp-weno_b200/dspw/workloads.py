"""Synthetic workloads of the stage path: initial states and descriptors.

Each builder returns ``(descs, prims, cells)``: the ``dspw_desc`` list of one
batch, the primitive initial state of every problem (``(nv, nz, ny, nx)``
float64, nv = 1 for scalar laws and 5 for systems) and the number of physical
cells the batch advances per step.  The states follow the reference's example
set-ups (enflo/examples, enflo_scalar/examples); seeded noise and random
Fourier data stand in for inputs that a param.in expression cannot state.

    kh        Kelvin-Helmholtz on the periodic unit square (2-D Euler); a
              grid-nested variant for convergence studies (kh_prim_nested)
    shu_osher Shu-Osher shock / entropy-wave interaction on [-5, 5] (1-D Euler)
    batched   isentropic vortex OOC mesh list plus many 1-D Burgers problems of
              uneven sizes, all in one batch
    tgv       Taylor-Green vortex, compressible Navier-Stokes on [0, 2 pi]^3
"""
from __future__ import annotations

import math

import numpy as np

from .capi import make_desc


def kh_prim(n: int, seed: int = 12345) -> np.ndarray:
    """rho 2 / 1 and u 0.5 / -0.5 inside / outside |y - 0.5| < 0.25, p 2.5,
    v = 0.01 sin(4 pi x) + U(-1e-3, 1e-3) seeded noise, on an n x n grid of [0,1]^2."""
    h = 1.0 / n
    x = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    inner = np.abs(Y - 0.5) < 0.25
    rng = np.random.default_rng(seed)
    p = np.zeros((5, 1, n, n))
    p[0, 0] = np.where(inner, 2.0, 1.0)
    p[1, 0] = np.where(inner, 0.5, -0.5)
    p[2, 0] = 0.01 * np.sin(4 * np.pi * X) + rng.uniform(-1e-3, 1e-3, (n, n))
    p[4, 0] = 2.5
    return p


def kh_prim_nested(n: int, n_fine: int, seed: int = 12345) -> np.ndarray:
    """The Kelvin-Helmholtz state of kh_prim with one noise field for every
    grid: the U(-1e-3, 1e-3) noise is drawn once per cell of the n_fine grid
    and averaged over the fine cells of each n x n cell (n divides n_fine), so
    that the grids of a convergence study start from the same function.  The
    density / velocity jumps at |y - 0.5| = 0.25 lie on cell faces when 4
    divides n; v = 0.01 sin(4 pi x) is taken as the cell-average of the fine
    grid's point values too."""
    if n_fine % n:
        raise ValueError("n must divide n_fine")
    r = n_fine // n
    rng = np.random.default_rng(seed)
    noise = rng.uniform(-1e-3, 1e-3, (n_fine, n_fine))
    hf = 1.0 / n_fine
    xf = (np.arange(n_fine) + 0.5) * hf
    vf = 0.01 * np.sin(4 * np.pi * xf)[None, :] + noise
    v = vf.reshape(n, r, n, r).mean(axis=(1, 3))
    h = 1.0 / n
    x = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    inner = np.abs(Y - 0.5) < 0.25
    p = np.zeros((5, 1, n, n))
    p[0, 0] = np.where(inner, 2.0, 1.0)
    p[1, 0] = np.where(inner, 0.5, -0.5)
    p[2, 0] = v
    p[4, 0] = 2.5
    return p


def shu_osher_prim(nx: int) -> np.ndarray:
    """(rho, u, p) = (3.857143, 2.629369, 10.33333) for x < -4, otherwise
    rho = 1 + 0.2 sin(5x), u = 0, p = 1 (enflo/examples/1D/ShuOsher)."""
    h = 10.0 / nx
    x = -5.0 + (np.arange(nx) + 0.5) * h
    left = x < -4
    p = np.zeros((5, 1, 1, nx))
    p[0, 0, 0] = np.where(left, 3.857143, 1 + 0.2 * np.sin(5 * x))
    p[1, 0, 0] = np.where(left, 2.629369, 0.0)
    p[4, 0, 0] = np.where(left, 10.33333, 1.0)
    return p


def vortex_prim(n: int, beta: float = 5.0, gamma: float = 1.4) -> np.ndarray:
    """Isentropic vortex of strength beta on the periodic [-5, 5]^2 with unit
    free stream along x (enflo/examples/2D/IsentropicVortex)."""
    h = 10.0 / n
    x = -5.0 + (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    r2 = X * X + Y * Y
    g1 = gamma - 1.0
    T = 1 - g1 * beta * beta / (8 * gamma * math.pi * math.pi) * np.exp(1 - r2)
    du = beta / (2 * math.pi) * np.exp(0.5 * (1 - r2))
    p = np.zeros((5, 1, n, n))
    p[0, 0] = T ** (1 / g1)
    p[1, 0] = 1 - du * Y
    p[2, 0] = du * X
    p[4, 0] = T ** (gamma / g1)
    return p


def vortex_exact_density(n: int, t: float, beta: float = 5.0, gamma: float = 1.4) -> np.ndarray:
    """Density of the vortex advected by (1, 0) for time t on the periodic box."""
    h = 10.0 / n
    x = -5.0 + (np.arange(n) + 0.5) * h
    xs = (x - t + 5.0) % 10.0 - 5.0
    X, Y = np.meshgrid(xs, x)
    r2 = X * X + Y * Y
    g1 = gamma - 1.0
    T = 1 - g1 * beta * beta / (8 * gamma * math.pi * math.pi) * np.exp(1 - r2)
    return (T ** (1 / g1)).reshape(1, n, n)


def tgv_prim(n: int, mach: float = 0.1, gamma: float = 1.4) -> np.ndarray:
    """Taylor-Green vortex on [0, 2 pi]^3: rho 1, u = sin x cos y cos z,
    v = -cos x sin y cos z, w = 0, p = 1/(gamma M^2) + (cos 2x + cos 2y)(cos 2z + 2)/16."""
    h = 2 * math.pi / n
    x = (np.arange(n) + 0.5) * h
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    p = np.zeros((5, n, n, n))
    p[0] = 1.0
    p[1] = np.sin(X) * np.cos(Y) * np.cos(Z)
    p[2] = -np.cos(X) * np.sin(Y) * np.cos(Z)
    p[4] = 1 / (gamma * mach * mach) + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2) / 16
    return p


def burgers_fourier(nx: int, rng: np.random.Generator, modes: int = 8) -> np.ndarray:
    """u0(x) = sum_k a_k sin(k x + phi_k), a_k ~ U(-1, 1)/k, phi_k ~ U(0, 2 pi),
    on an nx-cell grid of the periodic [-pi, pi]."""
    a = rng.uniform(-1, 1, modes) / np.arange(1, modes + 1)
    phi = rng.uniform(0, 2 * math.pi, modes)
    h = 2 * math.pi / nx
    x = -math.pi + (np.arange(nx) + 0.5) * h
    u = np.zeros(nx)
    for k in range(modes):
        u += a[k] * np.sin((k + 1) * x + phi[k])
    return u.reshape(1, 1, 1, nx)


def kh(n, precision, recon, network, seed=12345, final_time=1.0e9):
    d = make_desc(model="euler", flux="kepes_tecno4_roe", recon=recon, nx=n, ny=n, nz=1, x=(0, 1), y=(0, 1),
                  bc="periodic", cfl=0.4, final_time=final_time, network=network, precision=precision)
    return [d], [kh_prim(n, seed)], n * n


def shu_osher(nx, precision, recon, network, final_time=1.8):
    d = make_desc(model="euler", flux="kepes_tecno4_roe", recon=recon, nx=nx, ny=1, nz=1, x=(-5, 5),
                  bc=["neumann", "neumann", "periodic", "periodic", "periodic", "periodic"], cfl=0.4,
                  final_time=final_time, network=network, precision=precision)
    return [d], [shu_osher_prim(nx)], nx


def batched_specs(levels=(64, 128, 256, 512, 1024, 2048), nburgers=4096, burgers_nx=(100, 5000), seed=2024):
    """Problem list of the batched workload as (kind, nx, rng seed of its data):
    the vortex OOC levels, then ``nburgers`` Burgers problems with
    Nx ~ U{burgers_nx}.  Cheap to build; the states come from ``batched``."""
    rng = np.random.default_rng(seed)
    specs = [("vortex", n, 0) for n in levels]
    for _ in range(nburgers):
        specs.append(("burgers", int(rng.integers(burgers_nx[0], burgers_nx[1] + 1)), int(rng.integers(1 << 62))))
    return specs


def spec_cells(spec):
    kind, n, _ = spec
    return n * n if kind == "vortex" else n


def batched(precision, recon, network, levels=(64, 128, 256, 512, 1024, 2048), nburgers=4096,
            burgers_nx=(100, 5000), seed=2024, vortex_time=10.0, burgers_time=0.5, select=None):
    """Vortex OOC list (one problem per level, CFL 0.5, kepes_tecno4_roe) and
    ``nburgers`` Burgers problems (bur_tecno4, CFL 0.5, Nx ~ U{burgers_nx},
    u0 a random 8-mode Fourier series).  ``select`` (indices into the problem
    list) builds a subset, e.g. one rank's share."""
    specs = batched_specs(levels, nburgers, burgers_nx, seed)
    idx = range(len(specs)) if select is None else select
    descs, prims, cells = [], [], 0
    for i in idx:
        kind, n, s = specs[i]
        if kind == "vortex":
            descs.append(make_desc(model="euler", flux="kepes_tecno4_roe", recon=recon, nx=n, ny=n, nz=1,
                                   x=(-5, 5), y=(-5, 5), bc="periodic", cfl=0.5, final_time=vortex_time,
                                   network=network, precision=precision))
            prims.append(vortex_prim(n))
        else:
            descs.append(make_desc(model="burgers", flux="bur_tecno4", recon=recon, nx=n, ny=1, nz=1,
                                   x=(-math.pi, math.pi), bc="periodic", cfl=0.5, final_time=burgers_time,
                                   network=network, precision=precision))
            prims.append(burgers_fourier(n, np.random.default_rng(s)))
        cells += spec_cells(specs[i])
    return descs, prims, cells


def tgv(n, precision, recon, network, final_time=10.0, mach=0.1):
    d = make_desc(model="ns_es", flux="kepes_tecno4_roe", recon=recon, nx=n, ny=n, nz=n, x=(0, 2 * math.pi),
                  y=(0, 2 * math.pi), z=(0, 2 * math.pi), bc="periodic", cfl=0.4, final_time=final_time,
                  network=network, precision=precision, mu_ref=1 / 1600, prandtl=0.71)
    return [d], [tgv_prim(n, mach)], n ** 3
