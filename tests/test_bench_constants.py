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
    assert np.isclose(bench.VOLUME_KERNEL_FALG, 1124.5 + 384.0 + 7.5 + 5.0 + 20.0)
