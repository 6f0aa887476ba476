"""The algorithmic operation counts that bench.py uses for the roofline equal the oracle's count."""
import numpy as np

import bench
from oracle.oracle import count_flops


def test_falg_constants_match_oracle_count():
    w = bench.workload(elems=2)
    total, phases = count_flops(N=w["N"], nElems=w["elems"], xmin=w["xmin"], xmax=w["xmax"], NGeo=w["NGeo"],
                                deform_amp=w["deform_amp"], eqn=1, lifting=1, lifting_var=3, mu0=w["mu0"],
                                riemann=44, volume_flux=5, ini_exact_func=7)
    for k, v in bench.FALG_PER_DOF.items():
        assert abs(phases[k] - v) < 1e-9, k
    assert abs(total - sum(bench.FALG_PER_DOF.values())) < 1e-9
    # the volume kernel's work: split form, surface integral, Jacobian, LSERK stage; the viscous volume
    # integral belongs to the lifting kernel, which computes it
    assert np.isclose(bench.VOLUME_KERNEL_FALG, 1124.5 + 7.5 + 5.0 + 20.0)
    assert np.isclose(bench.LIFTING_KERNEL_FALG, 519.75 + 384.0)
    assert np.isclose(bench.VOLUME_KERNEL_FALG + bench.LIFTING_KERNEL_FALG + bench.FALG_PER_DOF["face_flux"],
                      total + bench.FALG_RK_STAGE_PER_DOF)


def test_mhd_falg_constants_match_oracle_count():
    """The resistive-MHD configuration's counts, on its initial state (4^3 elements, N=4)."""
    from oracle.oracle import PHASES, OracleCase, _lib
    from fluxo_b200.workloads import mhd_orszag_tang_state

    w = bench.mhd_workload(elems=4)
    kw = dict(N=w["N"], nElems=w["elems"], xmin=w["xmin"], xmax=w["xmax"], NGeo=w["NGeo"], deform_amp=w["deform_amp"],
              eqn=3, kappa=w["kappa"], eta=w["eta"], mu0=0.0, lifting=1, lifting_var=3, volume_flux=10, riemann=14,
              noncons=1, nc_glm=0, nfvse=1, ini_exact_func=0, glm_scale=0.5, cfl_scale=w["cfl_scale"],
              dfl_scale=w["dfl_scale"])
    ref = OracleCase(**kw)
    ref.set_U(mhd_orszag_tang_state(ref.mesh()["Elem_xGP"], kappa=w["kappa"]))
    ref.calc_timestep()  # sets GLM_ch as in a time step
    c = OracleCase(counting=True, **kw)
    c.set_U(ref.get_U())
    c.glm_ch = ref.glm_ch
    lib = _lib(counting=True)
    lib.orc_reset_flops()
    c.dg_time_derivative(0.0)
    nd = c.nElems * c.np ** 3
    phases = {k: lib.orc_phase_flops(i) / nd for i, k in enumerate(PHASES)}
    assert phases["nfvse"] == 0.0
    for k, v in bench.MHD_FALG_PER_DOF.items():
        assert abs(phases[k] - v) < 1e-9, k


def test_batch_falg_constants_match_oracle_count():
    """The batched configuration's per-(equation, N) counts, on a 2^3 instance with the mix's data."""
    from oracle.oracle import OracleCase, _lib
    from fluxo_b200.workloads import BOX_MAX, BOX_MIN, SEED, fourier_state, instance_fields

    for (eqn, N), v in bench.BATCH_FALG_PER_DOF.items():
        c = OracleCase(counting=True, nElems=(2, 2, 2), xmin=BOX_MIN, xmax=BOX_MAX, NGeo=1, deform_amp=0.0,
                       **instance_fields(dict(N=N, eqn=eqn)))
        c.set_U(fourier_state(c.mesh()["Elem_xGP"], BOX_MIN, BOX_MAX, np.random.default_rng(SEED)))
        lib = _lib(counting=True)
        lib.orc_reset_flops()
        c.dg_time_derivative(0.0)
        assert abs(lib.orc_flops() / (c.nElems * c.np ** 3) - v) < 1e-9, (eqn, N)
