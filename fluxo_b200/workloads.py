"""Synthetic workloads of the benchmark configurations (generated in code: no mesh files, no datasets).

* ``mhd_orszag_tang_state``: the resistive-MHD configuration's initial state, a 3D-extruded
  Orszag-Tang-type vortex on [0,2pi]^3: rho = gamma^2, p = gamma, v = (-sin y, sin x, 0),
  B = (-sin y, sin 2x, 0)/sqrt(4 pi), psi = 0, plus a seeded uniform z-velocity perturbation of
  amplitude 1e-3 at every node.  It is not one of the reference's ExactFunc cases (the closest are
  IniExactFunc 311/312/322 in equation/mhd/equation.f90:1248-1276), so it is fed identically to the
  oracle and the GPU.
* ``fourier_instances``: the batched / served configurations' instances, periodic boxes with smooth
  random-Fourier perturbations (|k| <= 4, amplitude 0.05) of density and velocity on rho = 1, p = 1.
"""
import numpy as np

SEED = 20261203


def mhd_prim_to_cons(prim, kappa, mu_0=1.0):
    """PrimToCons of the MHD equations (mhd/equation_vars.f90:258-278); prim (..., 9)."""
    U = np.empty_like(prim)
    rho = prim[..., 0]
    U[..., 0] = rho
    U[..., 1:4] = prim[..., 1:4] * rho[..., None]
    U[..., 4] = (prim[..., 4] / (kappa - 1.0) + 0.5 * np.sum(U[..., 1:4] * prim[..., 1:4], axis=-1) +
                 0.5 / mu_0 * np.sum(prim[..., 5:9] ** 2, axis=-1))
    U[..., 5:9] = prim[..., 5:9]
    return U


def mhd_orszag_tang_state(xGP, kappa=5.0 / 3.0, seed=SEED, perturbation=1e-3, mu_0=1.0):
    """Conservative state (nElems, n, n, n, 9) of the resistive-MHD configuration at the nodes xGP
    (nElems, n, n, n, 3)."""
    x, y = xGP[..., 0], xGP[..., 1]
    prim = np.zeros(xGP.shape[:-1] + (9,))
    prim[..., 0] = kappa ** 2
    prim[..., 1] = -np.sin(y)
    prim[..., 2] = np.sin(x)
    prim[..., 3] = perturbation * np.random.default_rng(seed).uniform(-1.0, 1.0, size=x.shape)
    prim[..., 4] = kappa
    s = 1.0 / np.sqrt(4.0 * np.pi)
    prim[..., 5] = -np.sin(y) * s
    prim[..., 6] = np.sin(2.0 * x) * s
    return mhd_prim_to_cons(prim, kappa, mu_0)


def fourier_state(xGP, xmin, xmax, rng, kmax=4, amplitude=0.05, kappa=1.4, nmodes=6):
    """Euler / Navier-Stokes state (nElems, n, n, n, 5) on rho = 1, p = 1 with smooth random-Fourier
    perturbations of density and velocity: a few modes with integer wave vectors |k| <= kmax."""
    L = np.asarray(xmax, float) - np.asarray(xmin, float)
    xi = 2.0 * np.pi * (xGP - np.asarray(xmin, float)) / L
    prim = np.zeros(xGP.shape[:-1] + (5,))
    prim[..., 0] = 1.0
    prim[..., 4] = 1.0
    for var in (0, 1, 2, 3):
        for _ in range(nmodes):
            while True:
                k = rng.integers(-kmax, kmax + 1, size=3)
                if 0 < np.linalg.norm(k) <= kmax:
                    break
            ph = rng.uniform(0.0, 2.0 * np.pi)
            a = amplitude / nmodes * rng.uniform(0.5, 1.0)
            prim[..., var] += a * np.sin(xi @ k + ph)
    U = np.empty_like(prim)
    U[..., 0] = prim[..., 0]
    U[..., 1:4] = prim[..., 1:4] * prim[..., :1]
    U[..., 4] = prim[..., 4] / (kappa - 1.0) + 0.5 * prim[..., 0] * np.sum(prim[..., 1:4] ** 2, axis=-1)
    return U
