"""fluxo_gpu_dg_time_derivative_noalloc: the allocation-free Euler right-hand side.

It runs the same face-flux and volume kernels as fluxo_gpu_dg_time_derivative, on device arrays
the caller owns (here torch tensors) and with the face fluxes in the library's static scratch
array.  Two calls at N=3 on two different states, with a call at N=5 between them that
overwrites the operator tables in the shared scratch, must each reproduce the existing entry
point's Ut (relative L2 <= 1e-14 at N=3: the same kernels and summation order on the same inputs;
1e-13 at N=5, whose volume-kernel launch shape may differ between the two paths).
The file is named to be collected last, so it also runs after every other test in one process."""
import ctypes
import os

import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200 import _lib
from oracle.oracle import OracleCase

TOL = 1e-14
# a call at another N in between overwrites the operator tables in the shared scratch; the volume
# kernel's launch shape at that N may differ from the handle path's (first use in the process), and
# shapes agree to roundoff only
TOL_OTHER_N = 1e-13
CASE = dict(N=3, nElems=(4, 3, 2), NGeo=2, deform_amp=0.1, riemann=44, volume_flux=5, ini_exact_func=2,
            ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), xmin=(-1, -1, -1), xmax=(1, 1, 1))
CASE_N5 = dict(CASE, N=5, nElems=(2, 3, 2))


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def cfg_for(p):
    return fb.solver.make_cfg(N=p.N, eqn=0, riemann=p.riemann, volume_flux=p.volume_flux, kappa=p.kappa, R=p.R,
                              ini_exact_func=p.ini_exact_func)


def device_layout(m, N):
    """The reference's mesh arrays in the device layouts of fluxo_gpu_set_mesh (0-based ids)."""
    NP = N + 1
    nE, nS = m["ElemToSide"].shape[0], m["SideToElem"].shape[0]
    met = np.concatenate([m[k].reshape(nE, NP ** 3, 3).transpose(0, 2, 1)
                          for k in ("Metrics_fTilde", "Metrics_gTilde", "Metrics_hTilde")], axis=1)
    geo = np.concatenate([m[k].reshape(nS, NP * NP, 3).transpose(0, 2, 1) for k in ("NormVec", "TangVec1", "TangVec2")]
                         + [m["SurfElem"].reshape(nS, 1, NP * NP)], axis=1)
    s2e = m["SideToElem"].astype(np.int32).copy()
    s2e[:, :2] -= 1
    e2s = m["ElemToSide"].astype(np.int32).copy()
    e2s[:, :, 0] -= 1
    return {"metrics": np.ascontiguousarray(met), "sJ": np.ascontiguousarray(m["sJ"]),
            "facegeo": np.ascontiguousarray(geo), "s2e": s2e, "e2s": e2s}


def last_error(lib):
    buf = ctypes.create_string_buffer(512)
    lib.fluxo_gpu_last_error(None, buf, len(buf))
    return buf.value.decode()


def test_noalloc_rejects_oversized_mesh():
    """The size check comes before any device access, so it runs without a GPU."""
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fluxo_gpu.h")).read()
    assert "#define FLUXO_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)" in hdr
    assert _lib.NOALLOC_SCRATCH_BYTES == 8 * 1024 * 1024
    lib = _lib.load()
    c = OracleCase(**CASE)
    cfg = cfg_for(c.params)
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the call returns before touching memory
    too_many = (_lib.NOALLOC_SCRATCH_BYTES - 2304) // (5 * 16 * 8) + 1
    r = lib.fluxo_gpu_dg_time_derivative_noalloc(ctypes.byref(cfg), 10, too_many, *([fake] * 7), None)
    assert r == -1
    msg = last_error(lib)
    assert "maximum is %d" % _lib.NOALLOC_SCRATCH_BYTES in msg and "%d sides" % too_many in msg
    r = lib.fluxo_gpu_dg_time_derivative_noalloc(ctypes.byref(cfg), 10, too_many - 1, None, *([fake] * 6), None)
    assert r == -1 and "null array" in last_error(lib)
    # NFVSE blends the volume integral on the handle path; this entry point has no blending, so it
    # refuses the configuration instead of returning the unblended right-hand side
    cfg.nfvse = 1
    r = lib.fluxo_gpu_dg_time_derivative_noalloc(ctypes.byref(cfg), 10, 30, *([fake] * 7), None)
    assert r == -1 and "NFVSE" in last_error(lib)


@pytest.mark.gpu
def test_noalloc_matches_dg_time_derivative(gpu_lib):
    import torch

    lib = gpu_lib
    c = OracleCase(**CASE)
    p = c.params
    m = c.mesh()
    rng = np.random.default_rng(7)
    U0 = c.get_U()
    states = [U0 * (1 + 0.05 * rng.standard_normal(U0.shape)), U0 * (1 + 0.05 * rng.standard_normal(U0.shape))]

    # the existing entry point (handle, host arrays)
    op = fb.DGOperator(N=p.N, eqn=0, riemann=p.riemann, volume_flux=p.volume_flux, kappa=p.kappa, R=p.R,
                       ini_exact_func=p.ini_exact_func)
    op.set_mesh(m)
    refs = []
    for U in states:
        op.set_state(U)
        op.dg_time_derivative(0.0)
        refs.append(op.get_ut())

    # caller-owned device arrays
    dev = torch.device("cuda:0")
    lay = device_layout(m, p.N)
    t = {k: torch.from_numpy(v).to(dev) for k, v in lay.items()}
    dU = [torch.from_numpy(np.ascontiguousarray(U)).to(dev) for U in states]
    dUt = [torch.full(states[0].shape, float("nan"), dtype=torch.float64, device=dev) for _ in states]
    stream = torch.cuda.current_stream(dev)

    # a second mesh at N=5 (its own handle-path reference)
    c5 = OracleCase(**CASE_N5)
    p5, m5 = c5.params, c5.mesh()
    U5 = c5.get_U() * (1 + 0.05 * rng.standard_normal(c5.get_U().shape))
    t5 = {k: torch.from_numpy(v).to(dev) for k, v in device_layout(m5, p5.N).items()}
    dU5 = torch.from_numpy(np.ascontiguousarray(U5)).to(dev)
    dUt5 = torch.full(U5.shape, float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)

    def call(cfg, m_, t_, u, ut):
        nE, nS = m_["ElemToSide"].shape[0], m_["SideToElem"].shape[0]
        r = lib.fluxo_gpu_dg_time_derivative_noalloc(
            ctypes.byref(cfg), nE, nS, u.data_ptr(), ut.data_ptr(), t_["metrics"].data_ptr(),
            t_["sJ"].data_ptr(), t_["facegeo"].data_ptr(), t_["s2e"].data_ptr(), t_["e2s"].data_ptr(),
            ctypes.c_void_p(stream.cuda_stream))
        assert r == 0, last_error(lib)

    cfg = cfg_for(p)
    # N=3, then N=5 (tables overwritten), then N=3 again (tables restored): all share the scratch
    call(cfg, m, t, dU[0], dUt[0])
    call(cfg_for(p5), m5, t5, dU5, dUt5)
    call(cfg, m, t, dU[1], dUt[1])
    # the N=5 reference comes afterwards: in a fresh process the call above ran the volume kernel in
    # its untuned launch shape, and the handle path then tunes it
    op5 = fb.DGOperator(N=p5.N, eqn=0, riemann=p5.riemann, volume_flux=p5.volume_flux, kappa=p5.kappa, R=p5.R,
                        ini_exact_func=p5.ini_exact_func)
    op5.set_mesh(m5)
    op5.set_state(U5)
    op5.dg_time_derivative(0.0)
    ref5 = op5.get_ut()
    for k in range(2):
        out = dUt[k].cpu().numpy()
        assert np.isfinite(out).all()
        assert rel_l2(out, refs[k]) <= TOL
    out5 = dUt5.cpu().numpy()
    assert np.isfinite(out5).all() and rel_l2(out5, ref5) <= TOL_OTHER_N
    assert rel_l2(refs[0], refs[1]) > 1e-6  # the two states give different right-hand sides
    op.close()
    op5.close()
