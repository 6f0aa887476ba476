"""Generates tests/golden/tgv_trace_N7_8x8x8.json: the kinetic-energy and enstrophy trace of the
Navier-Stokes Taylor-Green workload (N=7, curved [-pi,pi]^3 box with NGeo 2 and deformation 0.05,
Re 1600, Ma 0.1, BR1 entropy variables, EC-KEP volume flux, Riemann 44, LSERK4-5 at CFLscale 0.5 /
DFLscale 0.5) on 8^3 elements from t=0 to t=1, analysed every 0.05, computed by the CPU oracle.

Each analysis point follows the reference's TimeDisc (src/timedisc/timedisc.f90:300-404): the time
step is clipped to the analysis time, a right-hand side is evaluated at that time, then the
Taylor-Green integrands (1/Vol integral of 1/2 rho |v|^2 and 1/2 rho |curl v|^2 with the collocation
weights wGPVol/sJ) are reduced.  Run (about 4 minutes on 8 cores): python tests/golden/make_tgv_trace.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

ELEMS = 8
T_END = 1.0
ANALYZE_DT = 0.05


def case_kwargs():
    import bench

    w = bench.workload(elems=ELEMS)
    return dict(N=w["N"], nElems=w["elems"], xmin=w["xmin"], xmax=w["xmax"], NGeo=w["NGeo"],
                deform_amp=w["deform_amp"], eqn=1, lifting=1, lifting_var=3, mu0=w["mu0"], Pr=w["Pr"],
                kappa=w["kappa"], riemann=w["riemann"], volume_flux=w["volume_flux"], ini_exact_func=7,
                cfl_scale=w["cfl_scale"], dfl_scale=w["dfl_scale"])


def main():
    from oracle.oracle import OracleCase

    c = OracleCase(**case_kwargs())
    t, steps, rows = 0.0, 0, []
    t0 = time.time()
    k = 0
    while True:
        c.dg_time_derivative(t)
        a = c.analyze(t)
        rows.append({"t": t, "steps": steps, "ekin": a["ekin"], "enstrophy": a["enstrophy"]})
        print("t=%.4f steps=%d ekin=%.12e enstrophy=%.12e (%.0f s)" % (t, steps, a["ekin"], a["enstrophy"],
                                                                      time.time() - t0), flush=True)
        if t >= T_END:
            break
        k += 1
        t_next = min(k * ANALYZE_DT, T_END)
        t, n = c.run(t, t_next)
        steps += n
        assert abs(t - t_next) <= 1e-12, (t, t_next)
    out = {"case": case_kwargs(), "analyze_dt": ANALYZE_DT, "t_end": T_END, "trace": rows,
           "generator": "tests/golden/make_tgv_trace.py (CPU oracle)"}
    with open(os.path.join(HERE, "tgv_trace_N7_8x8x8.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
