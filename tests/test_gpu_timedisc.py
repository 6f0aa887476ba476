"""Every TimeDiscMethod on the GPU against the oracle (src/timedisc/timedisc_vars.f90:94-726): one time
step with the host's dt (fluxo_gpu_timestep) and three steps of the device-resident TimeDisc loop
(fluxo_gpu_time_disc, dt from CALCTIMESTEP on the device), for the Navier-Stokes right-hand side (BR1
lifting) and, for the schemes whose stage update is not fused into the volume kernel, for resistive MHD.
CFLscale 0.4: Ketcheson RK4-20 takes the CFL scaling of Niegemann RK4-14 in the reference's table and
is unstable at 0.9 on these cases (the oracle and the GPU both blow up).  Tolerance: relative L2 <= 1e-12."""
import numpy as np
import pytest

from oracle.oracle import OracleCase
from test_gpu_parity import pair

pytestmark = pytest.mark.gpu
TOL = 1e-12
NAMES = ["carpenterrk4-5", "standardrk3-3", "niegemannrk4-14", "toulorgerk4-8c", "toulorgerk3-7c", "toulorgerk4-8f",
         "ketchesonrk4-20", "ketchesonrk4-18", "ssprk4-5", "ssprk3-3"]


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


@pytest.mark.parametrize("td", range(10), ids=NAMES)
def test_navier_stokes_every_scheme(gpu_lib, td):
    c, op = pair(eqn=1, mu0=0.02, ini_exact_func=7, N=3, nElems=(2, 3, 2), NGeo=2, deform_amp=0.05,
                 xmin=(-np.pi,) * 3, xmax=(np.pi,) * 3, lifting=1, lifting_var=3, riemann=44, volume_flux=5,
                 time_disc=td, perturb=0.02, cfl_scale=0.4)
    dt_ref, _ = c.calc_timestep()
    dt, err = op.calc_timestep()
    assert err == 0 and dt == pytest.approx(dt_ref, rel=1e-13)
    c.timestep(0.0, dt_ref)
    op.timestep(0.0, dt_ref)
    assert rel_l2(op.get_state(), c.get_U()) <= TOL
    t_ref, n_ref = c.run(dt_ref, 10.0, max_iter=3)
    t, n, err = op.time_disc(dt_ref, 10.0, 3)
    assert err == 0 and n == n_ref == 3 and t == pytest.approx(t_ref, rel=1e-13)
    assert rel_l2(op.get_state(), c.get_U()) <= TOL


@pytest.mark.parametrize("td", [6, 8, 9], ids=["ketchesonrk4-20", "ssprk4-5", "ssprk3-3"])
def test_resistive_mhd_unfused_schemes(gpu_lib, td):
    from test_gpu_mhd import mhd_pair

    c, op = mhd_pair(eqn=3, N=3, volume_flux=10, riemann=10, noncons=1, nc_glm=1, eta=0.02, mu0=0.01,
                     time_disc=td, cfl_scale=0.4)
    t_ref, n_ref = c.run(0.0, 10.0, max_iter=2)
    t, n, err = op.time_disc(0.0, 10.0, 2)
    assert err == 0 and n == n_ref == 2 and t == pytest.approx(t_ref, rel=1e-13)
    assert rel_l2(op.get_state(), c.get_U()) <= TOL
