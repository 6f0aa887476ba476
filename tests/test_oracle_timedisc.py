"""The oracle's time integrators (every TimeDiscMethod of src/timedisc/timedisc_vars.f90:94-726): the
two-register LSERKW2 family, the three-register Ketcheson schemes (LSERKK3), SSPRK4-5 and SSPRK3-3 reach
their design order in time on a smooth Euler density wave (errors against a reference run with a 10x
smaller step of the Carpenter scheme), and the CFL scaling follows FillCFL_DFL (timedisc.f90:697-741)."""
import numpy as np
import pytest

from oracle.oracle import OracleCase

SCHEMES = {0: ("carpenterrk4-5", 4), 1: ("standardrk3-3", 3), 2: ("niegemannrk4-14", 4), 3: ("toulorgerk4-8c", 4),
           4: ("toulorgerk3-7c", 3), 5: ("toulorgerk4-8f", 4), 6: ("ketchesonrk4-20", 4), 7: ("ketchesonrk4-18", 4),
           8: ("ssprk4-5", 4), 9: ("ssprk3-3", 3)}
CASE = dict(N=4, nElems=(2, 2, 2), NGeo=1, deform_amp=0.0, xmin=(-1, -1, -1), xmax=(1, 1, 1), riemann=1,
            volume_flux=10, ini_exact_func=2, ini_amplitude=0.2, adv_vel=(0.3, -0.2, 0.5))
T = 0.4


def run(time_disc, nsteps):
    c = OracleCase(time_disc=time_disc, **CASE)
    dt = T / nsteps
    t = 0.0
    for _ in range(nsteps):
        c.timestep(t, dt)
        t += dt
    return c.get_U()


@pytest.fixture(scope="module")
def reference():
    return run(0, 512)


@pytest.mark.parametrize("td", sorted(SCHEMES), ids=[SCHEMES[k][0] for k in sorted(SCHEMES)])
def test_temporal_order(reference, td):
    name, order = SCHEMES[td]
    n = 6 if td == 6 else 24  # Ketcheson RK4-20 is accurate to roundoff at 24 steps already
    e1 = np.abs(run(td, n) - reference).max()
    e2 = np.abs(run(td, 2 * n) - reference).max()
    rate = np.log2(e1 / e2)
    assert rate > order - 0.4, (name, e1, e2, rate)


def test_cfl_scaling_and_stages():
    """CFLScale = CFLscale * alpha(N) / (2N+1) with the table's alpha: the oracle's dt scales with it."""
    alpha_n4 = {0: 2.4739, 1: 1.5075, 2: 7.0965, 3: 4.2616, 4: 4.2156, 5: 4.1376, 6: 7.0965, 7: None, 8: 2.4739,
                9: 1.5075}
    dts = {td: OracleCase(time_disc=td, **CASE).calc_timestep()[0] for td in SCHEMES}
    for td, a in alpha_n4.items():
        if a is not None:
            assert dts[td] / dts[0] == pytest.approx(a / 2.4739, rel=1e-12), SCHEMES[td][0]
