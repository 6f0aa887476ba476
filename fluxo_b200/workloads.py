"""Synthetic workloads of the benchmark configurations (generated in code: no mesh files, no datasets).

* ``mhd_orszag_tang_state``: the resistive-MHD configuration's initial state, a 3D-extruded
  Orszag-Tang-type vortex on [0,2pi]^3: rho = gamma^2, p = gamma, v = (-sin y, sin x, 0),
  B = (-sin y, sin 2x, 0)/sqrt(4 pi), psi = 0, plus a seeded uniform z-velocity perturbation of
  amplitude 1e-3 at every node.  It is not one of the reference's ExactFunc cases (the closest are
  IniExactFunc 311/312/322 in equation/mhd/equation.f90:1248-1276), so it is fed identically to the
  oracle and the GPU.
* ``batch_instance_specs`` / ``build_instance``: the batched configuration's instances, periodic
  boxes [0,2]^3 with elements per direction from {4,6,8,12,16} and N from {3,4,5,7} drawn from one
  seeded RNG, Euler or Navier-Stokes, and ``fourier_state`` initial data: smooth random-Fourier
  perturbations (|k| <= 4, amplitude 0.05) of density and velocity on rho = 1, p = 1.
"""
import numpy as np

SEED = 20261203

BOX_MIN, BOX_MAX = (0.0, 0.0, 0.0), (2.0, 2.0, 2.0)
BATCH_ELEMS = (4, 6, 8, 12, 16)
BATCH_N = (3, 4, 5, 7)
# kernel configuration of the two equation systems in the batched / served mixes: the EC-KEP
# split form with the matrix-dissipation entropy-stable surface flux for both, CFLscale 0.5.  With
# CFLscale 0.9 the reference algorithm (the oracle) is unstable on these boxes at N = 6, 7: a 1e-14
# perturbation of the initial state ends in a negative density within ~30 steps, while at 0.5 it
# stays at 1e-14 (and with the LLF surface flux it stops some N = 6, 7 requests as well).
EULER_FIELDS = dict(eqn=0, riemann=44, volume_flux=5, kappa=1.4, cfl_scale=0.5, time_disc=0, ini_exact_func=0)
NS_FIELDS = dict(eqn=1, riemann=44, volume_flux=5, lifting=1, lifting_var=3, visc=0, mu0=1.0 / 1600.0, Pr=0.72,
                 kappa=1.4, cfl_scale=0.5, dfl_scale=0.4, time_disc=0, ini_exact_func=0)


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


def mhd_exact_func(func, t, x, kappa=5.0 / 3.0, mu_0=1.0, ref_states=((1.0, 0, 0, 0, 1.0, 1.0, 0, 0),),
                   ini_ref_state=1, center=(0.0, 0.0, 0.0), halfwidth=0.1, amplitude=0.1, frequency=1.0):
    """FillIni / ExactFunc of the MHD equations (mhd/equation.f90:540-1276) on points x (..., 3) ->
    conservative U (..., 9): 1 constant RefState(IniRefState), 3 Alfven wave, 201 soft blast between
    RefStates 1 and 2, 311 Orszag-Tang vortex, 312 its 3D perturbed form."""
    x = np.asarray(x, dtype=np.float64)
    prim = np.zeros(x.shape[:-1] + (9,))
    refs = np.asarray(ref_states, dtype=np.float64)
    if func == 1:
        prim[..., :8] = refs[ini_ref_state - 1]
    elif func == 3:  # :596-639
        omega, r, e = 2.0 * np.pi * frequency, 2.0, 0.2
        nx, ny = 1.0 / np.sqrt(r * r + 1.0), r / np.sqrt(r * r + 1.0)
        va = omega / ny
        phi = omega / ny * (nx * (x[..., 0] - 0.5 * r) + ny * (x[..., 1] - 0.5 * r)) - va * t
        U = np.zeros(x.shape[:-1] + (9,))
        U[..., 0] = 1.0
        U[..., 1] = -e * ny * np.cos(phi)
        U[..., 2] = e * nx * np.cos(phi)
        U[..., 3] = e * np.sin(phi)
        U[..., 4] = 1.0 / (kappa - 1.0) + 0.5 * np.sum(U[..., 1:4] ** 2, axis=-1)
        U[..., 5] = nx - U[..., 1]
        U[..., 6] = ny - U[..., 2]
        U[..., 7] = -U[..., 3]
        return U
    elif func == 201:  # :1239-1246
        rr = np.sqrt(np.sum((x - np.asarray(center)) ** 2, axis=-1))
        a = np.exp(5.0 * (rr - halfwidth) / amplitude)
        a = (a / (a + 1.0))[..., None]
        prim[..., :8] = (1.0 - a) * refs[0] + a * refs[1]
    elif func in (311, 312):  # :1248-1266
        sx, sy = np.sin(2 * np.pi * x[..., 0]), np.sin(2 * np.pi * x[..., 1])
        fz = 1.0 + 0.2 * np.sin(2 * np.pi * x[..., 2]) if func == 312 else 1.0
        prim[..., 0] = 1.0
        prim[..., 1] = -fz * sy
        prim[..., 2] = fz * sx
        if func == 312:
            prim[..., 3] = 0.2 * np.sin(2 * np.pi * x[..., 2])
        prim[..., 4] = 1.0 / kappa
        prim[..., 5] = -sy / kappa
        prim[..., 6] = np.sin(4 * np.pi * x[..., 0]) / kappa
    else:
        raise ValueError("MHD IniExactFunc %d not implemented" % func)
    return mhd_prim_to_cons(prim, kappa, mu_0)


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


def batch_instance_specs(n=64, seed=SEED):
    """The batched configuration: n instances drawn from one RNG (elements per direction, N,
    equation system, and the seed of each instance's initial data)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        e = int(rng.choice(BATCH_ELEMS))
        N = int(rng.choice(BATCH_N))
        eqn = int(rng.integers(0, 2))
        specs.append(dict(index=i, elems=e, N=N, eqn=eqn, seed=int(rng.integers(0, 2 ** 31 - 1))))
    return specs


def instance_fields(spec):
    """fluxo_cfg fields of an instance spec."""
    f = dict(NS_FIELDS if spec["eqn"] == 1 else EULER_FIELDS)
    f["N"] = spec["N"]
    return f


def build_instance(spec, mesh_cache=None):
    """(mesh arrays, initial state) of an instance spec; meshes of equal (N, elements) are shared."""
    from .solver import box_mesh

    key = (spec["N"], spec["elems"])
    mesh = None if mesh_cache is None else mesh_cache.get(key)
    if mesh is None:
        mesh = box_mesh(spec["N"], (spec["elems"],) * 3, BOX_MIN, BOX_MAX)
        if mesh_cache is not None:
            mesh_cache[key] = mesh
    U = fourier_state(mesh["Elem_xGP"], BOX_MIN, BOX_MAX, np.random.default_rng(spec["seed"]))
    return mesh, U


def serve_request_specs(rate, duration, seed=SEED, elems=(4, 24), N=(3, 7), t_end=(0.05, 1.0)):
    """The served configuration's request stream: Poisson arrivals at `rate` per second over
    `duration` seconds; each request an Euler or Navier-Stokes periodic box with elements per
    direction uniform in elems[0]..elems[1], N uniform in N[0]..N[1], end time log-uniform in
    t_end, and its own seed for the ``fourier_state`` initial data."""
    rng = np.random.default_rng(seed)
    specs, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        specs.append(dict(index=len(specs), arrival=t, elems=int(rng.integers(elems[0], elems[1] + 1)),
                          N=int(rng.integers(N[0], N[1] + 1)), eqn=int(rng.integers(0, 2)),
                          t_end=float(np.exp(rng.uniform(np.log(t_end[0]), np.log(t_end[1])))),
                          seed=int(rng.integers(0, 2 ** 31 - 1))))
    return specs
