"""Kinetic energy and enstrophy of the Navier-Stokes Taylor-Green workload from t=0 to t=1 on the GPU,
against the oracle's trace (tests/golden/tgv_trace_N7_8x8x8.json, made by make_tgv_trace.py).

The GPU side runs the product path a Fortran host would drive: the mesh and initial state from the
product's host setup, fluxo_gpu_time_disc between analysis points (dt clipped to each analysis time as
in timedisc.f90:306-317), and fluxo_gpu_analyze at every 0.05.  Both traces must agree to 3 significant
digits (relative 5e-4) at every analysis point, with the same number of time steps; in practice they
agree to ~1e-10, the roundoff of 670 time steps."""
import json
import os

import numpy as np
import pytest

import bench
import fluxo_b200 as fb

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tgv_trace_N7_8x8x8.json")


def test_tgv_trace_to_t1_matches_oracle(gpu_lib):
    with open(GOLDEN) as f:
        g = json.load(f)
    w = bench.workload(elems=8)
    mesh = fb.box_mesh(w["N"], w["elems"], w["xmin"], w["xmax"], NGeo=w["NGeo"], deform_amp=w["deform_amp"])
    op = fb.DGOperator(N=w["N"], eqn=1, riemann=w["riemann"], volume_flux=w["volume_flux"], lifting=1, lifting_var=3,
                       visc=0, mu0=w["mu0"], Pr=w["Pr"], kappa=w["kappa"], cfl_scale=w["cfl_scale"],
                       dfl_scale=w["dfl_scale"], time_disc=0)
    op.set_mesh(mesh)
    op.set_state(fb.exact_func(7, 0.0, mesh["Elem_xGP"], kappa=w["kappa"]))
    t, steps, worst = 0.0, 0, 0.0
    for row in g["trace"]:
        if row["t"] > 0.0:
            t, n, err = op.time_disc(t, row["t"])
            assert err == 0
            steps += n
        assert t == pytest.approx(row["t"], abs=1e-12) and steps == row["steps"]
        a = op.analyze(t)
        for k in ("ekin", "enstrophy"):
            r = abs(a[k] - row[k]) / abs(row[k])
            worst = max(worst, r)
            assert r <= 5e-4, (t, k, a[k], row[k])
    assert worst <= 5e-4
    # the trace is physical: kinetic energy decays, enstrophy grows over t in [0, 1]
    ek = np.array([r["ekin"] for r in g["trace"]])
    en = np.array([r["enstrophy"] for r in g["trace"]])
    assert np.all(np.diff(ek) < 0) and en[-1] > en[0]
    op.close()
