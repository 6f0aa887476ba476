"""Python host side of the B200 DGSEM path, mirroring the reference's operator interface.

``DGOperator`` wraps one ``fluxo_handle`` of the C ABI with explicit arrays (the drop-in
path a Fortran host would take: it passes its own mesh metrics and state).  ``Fluxo`` runs the
reference's initialisation order (InitInterpolation -> InitMesh -> InitEquation -> InitDG
(FillIni) -> InitTimeDisc, src/fluxo.f90:62-178) from a ``parameter.ini`` and exposes
``DGTimeDerivative``, ``CalcTimeStep``, ``TimeStep`` and ``TimeDisc`` with the reference's names.
All compute runs on the GPU through ``libfluxo_gpu.so``; there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

from . import _lib
from .params import RK_STAGES, _flag, parse_ini, resolve, to_cfg_fields


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def make_cfg(**fields):
    cfg = _lib.FluxoCfg()
    cfg.struct_size = ctypes.sizeof(_lib.FluxoCfg)
    defaults = dict(N=3, eqn=0, riemann=1, volume_flux=0, lifting=1, lifting_var=3, visc=0, kappa=1.4, R=287.058,
                    Pr=0.72, mu0=0.0, Ts=110.4, Tref=280.0, ExpoSuth=1.5, ExpoPow=0.0, etaBR2=2.0, time_disc=0,
                    cfl_scale=0.9, dfl_scale=0.4, ini_exact_func=1, ini_frequency=1.0, ini_amplitude=0.1, device=0,
                    mu_0=1.0, eta=0.0, glm_scale=0.5, glm_scr=0.0, noncons=1, nc_glm=0,
                    nfvse=0, compute_alpha=1, shock_blend_coef=0.0, modal_threshold=1, alpha_max=0.5,
                    alpha_min=0.01, space_prop_factor=0.5, space_prop_sweeps=1, time_rel_factor=0.0,
                    indicator_quantity=3, sub_fv_method=1, recons_boundaries=1, nfvse_corr=0,
                    posit_corr_factor=0.1, posit_max_iter=10, node_type=2)
    defaults.update(fields)
    for k, v in defaults.items():
        setattr(cfg, k, v)
    return cfg


def box_mesh(N, elems, xmin, xmax, NGeo=1, deform_amp=0.0, node_type=2):
    """Reference-layout mesh arrays of a periodic box (C ABI ``fluxo_host_box_mesh``; node_type 1: Gauss
    nodes, ``fluxo_host_box_mesh_gauss``, with ``SurfMetrics[e,side,q,p,:]``).

    Numpy shapes are the C-order views of the Fortran arrays, e.g. ``Metrics_fTilde[e,k,j,i,:]``.
    """
    lib = _lib.load()
    ne = _c(elems, np.int32)
    nE, nS = ctypes.c_int(), ctypes.c_int()
    _lib.check(lib.fluxo_host_box_sizes(_ptr(ne), ctypes.byref(nE), ctypes.byref(nS)))
    n = N + 1
    nE, nS = nE.value, nS.value
    m = dict(
        SideToElem=np.zeros((nS, 5), np.int32), ElemToSide=np.zeros((nE, 6, 2), np.int32),
        Metrics_fTilde=np.zeros((nE, n, n, n, 3)), Metrics_gTilde=np.zeros((nE, n, n, n, 3)),
        Metrics_hTilde=np.zeros((nE, n, n, n, 3)), sJ=np.zeros((nE, n, n, n)),
        NormVec=np.zeros((nS, n, n, 3)), TangVec1=np.zeros((nS, n, n, 3)), TangVec2=np.zeros((nS, n, n, 3)),
        SurfElem=np.zeros((nS, n, n)), Elem_xGP=np.zeros((nE, n, n, n, 3)),
    )
    if node_type == 1:
        m["SurfMetrics"] = np.zeros((nE, 6, n, n, 3))
        r = lib.fluxo_host_box_mesh_gauss(N, _ptr(ne), _ptr(_c(xmin)), _ptr(_c(xmax)), NGeo, float(deform_amp),
                                          *[_ptr(m[k]) for k in MESH_KEYS], _ptr(m["SurfMetrics"]))
    else:
        r = lib.fluxo_host_box_mesh(N, _ptr(ne), _ptr(_c(xmin)), _ptr(_c(xmax)), NGeo, float(deform_amp),
                                    *[_ptr(m[k]) for k in MESH_KEYS])
    _lib.check(r)
    return m


MESH_KEYS = ("SideToElem", "ElemToSide", "Metrics_fTilde", "Metrics_gTilde", "Metrics_hTilde", "sJ", "NormVec",
             "TangVec1", "TangVec2", "SurfElem", "Elem_xGP")


def exact_func(func, t, x, kappa=1.4, adv_vel=(1.0, 1.0, 1.0), amplitude=0.1, wavenumber=(1.0, 1.0, 1.0),
               frequency=1.0, ref_state=(1.0, 0.0, 0.0, 0.0, 0.71428571)):
    """FillIni / ExactFunc on points x[...,3] -> conservative U[...,5] (C ABI ``fluxo_host_exact_func``)."""
    x = _c(x)
    U = np.zeros(x.shape[:-1] + (5,))
    r = _lib.load().fluxo_host_exact_func(int(func), float(t), x.size // 3, _ptr(x), float(kappa), _ptr(_c(adv_vel)),
                                          float(amplitude), _ptr(_c(wavenumber)), float(frequency),
                                          _ptr(_c(ref_state)), _ptr(U))
    _lib.check(r)
    return U


class DGOperator:
    """One GPU handle: the reference's DGTimeDerivative / TimeStep / CALCTIMESTEP on device state."""

    def __init__(self, cfg=None, **fields):
        self.lib = _lib.load()
        self.cfg = cfg if cfg is not None else make_cfg(**fields)
        h = ctypes.c_void_p()
        r = self.lib.fluxo_gpu_create(ctypes.byref(self.cfg), ctypes.byref(h))
        _lib.check(r, None)
        self.h = h
        self.N = self.cfg.N
        self.nVar = 9 if self.cfg.eqn in (2, 3) else 5
        self.nElems = self.nSides = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.fluxo_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, r):
        _lib.check(r, self.h)

    def set_mesh(self, m):
        S2E = _c(m["SideToElem"], np.int32)
        self.nSides = S2E.shape[0]
        self.nElems = _c(m["ElemToSide"], np.int32).shape[0]
        arrs = [_c(m[k]) for k in MESH_KEYS[2:10]]
        xgp = m.get("Elem_xGP")
        self._keep = (S2E, _c(m["ElemToSide"], np.int32), arrs, None if xgp is None else _c(xgp))
        r = self.lib.fluxo_gpu_set_mesh(self.h, self.nElems, self.nSides, _ptr(self._keep[0]), _ptr(self._keep[1]),
                                        *[_ptr(a) for a in arrs], _ptr(self._keep[3]))
        self._check(r)
        if m.get("SurfMetrics") is not None:  # Gauss nodes: SurfMetrics(3,0:N,0:N,6,nElems)
            self._check(self.lib.fluxo_gpu_set_surf_metrics(self.h, _ptr(_c(m["SurfMetrics"]))))

    @property
    def shape(self):
        n = self.N + 1
        return (self.nElems, n, n, n, self.nVar)

    @property
    def glm_ch(self):
        """MHD: GLM_ch of the next right-hand side (set by calc_timestep / time_disc)."""
        ch = ctypes.c_double()
        self._check(self.lib.fluxo_gpu_get_glm_ch(self.h, ctypes.byref(ch)))
        return ch.value

    @glm_ch.setter
    def glm_ch(self, ch):
        self._check(self.lib.fluxo_gpu_set_glm_ch(self.h, float(ch)))

    def alpha(self):
        """NFVSE blending coefficients of the last right-hand side (one per element)."""
        a = np.empty(self.nElems)
        self._check(self.lib.fluxo_gpu_get_alpha(self.h, _ptr(a)))
        return a

    def set_alpha(self, alpha):
        """Sets the NFVSE blending coefficients that the next right-hand side starts from
        (ComputeAlpha 20 keeps them)."""
        a = _c(alpha)
        assert a.size == self.nElems, "alpha needs one value per element"
        self._check(self.lib.fluxo_gpu_set_alpha(self.h, _ptr(a)))

    def set_state(self, U):
        U = _c(U)
        assert U.size == int(np.prod(self.shape)), "U has the wrong size"
        self._check(self.lib.fluxo_gpu_set_state(self.h, _ptr(U)))

    def get_state(self):
        U = np.empty(self.shape)
        self._check(self.lib.fluxo_gpu_get_state(self.h, _ptr(U)))
        return U

    def get_ut(self):
        Ut = np.empty(self.shape)
        self._check(self.lib.fluxo_gpu_get_ut(self.h, _ptr(Ut)))
        return Ut

    def get_gradients(self):
        g = [np.empty(self.shape) for _ in range(3)]
        self._check(self.lib.fluxo_gpu_get_gradients(self.h, *[_ptr(a) for a in g]))
        return g

    def dg_time_derivative(self, t=0.0):
        self._check(self.lib.fluxo_gpu_dg_time_derivative(self.h, float(t)))

    def analyze(self, t=0.0, exact=None):
        """Analysis at time t on the device (fluxo_gpu_analyze): a right-hand side at t, then CalcErrorNorms
        (when ``exact`` names an exact function: dict with func, adv_vel, ini_wavenumber, ini_amplitude,
        ini_frequency, ref_state_prim, ini_center), CalcEntropy, dS/dU.Ut and the Taylor-Green integrands."""
        ex = None
        if exact is not None and exact.get("func", 0):
            ex = _lib.FluxoExact()
            ex.func = int(exact["func"])
            for k, n in (("adv_vel", 3), ("ini_wavenumber", 3), ("ref_state_prim", 5), ("ini_center", 3)):
                v = exact.get(k, (0.0,) * n)
                getattr(ex, k)[:] = [float(z) for z in v]
            ex.ini_amplitude = float(exact.get("ini_amplitude", 0.0))
            ex.ini_frequency = float(exact.get("ini_frequency", 1.0))
        nv = self.nVar
        L2, Li, Lc, sc = np.zeros(nv), np.zeros(nv), np.zeros(nv), np.zeros(5)
        self._check(self.lib.fluxo_gpu_analyze(self.h, float(t), None if ex is None else ctypes.byref(ex), _ptr(L2),
                                               _ptr(Li), _ptr(Lc), _ptr(sc)))
        out = {"entropy": sc[0], "dSdU_Ut": sc[1], "ekin": sc[2], "enstrophy": sc[3], "volume": sc[4]}
        if ex is not None:
            out.update(L2=L2, Linf=Li, L2_colloc=Lc)
        return out

    def calc_timestep(self):
        dt, err = ctypes.c_double(), ctypes.c_int()
        r = self.lib.fluxo_gpu_calc_timestep(self.h, ctypes.byref(dt), ctypes.byref(err))
        if r not in (_lib.FLUXO_OK, -4):
            self._check(r)
        return dt.value, err.value

    def timestep(self, t, dt):
        self._check(self.lib.fluxo_gpu_timestep(self.h, float(t), float(dt)))

    def time_disc(self, t, t_end, max_iter=-1):
        tout, n, err = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        r = self.lib.fluxo_gpu_time_disc(self.h, float(t), float(t_end), int(max_iter), ctypes.byref(tout),
                                         ctypes.byref(n), ctypes.byref(err))
        if r not in (_lib.FLUXO_OK, -4):
            self._check(r)
        return tout.value, n.value, err.value

    def device_buffers(self):
        dU, dUt, st = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self.lib.fluxo_gpu_device_buffers(self.h, ctypes.byref(dU), ctypes.byref(dUt), ctypes.byref(st)))
        return dU.value, dUt.value, st.value

    def launch_count(self):
        n = ctypes.c_uint64()
        self._check(self.lib.fluxo_gpu_launch_count(self.h, ctypes.byref(n)))
        return n.value


class Fluxo:
    """The reference's program flow for one ``parameter.ini`` on one GPU."""

    def __init__(self, ini=None, device=0, restart_file=None, base_dir=None, **overrides):
        """``ini``: parameter.ini text or a dict of options; ``restart_file``: a State file to start
        from (the reference's second command-line argument); ``base_dir``: the directory that a
        relative ``MeshFile`` is taken from (the reference's working directory; default: cwd)."""
        opts = parse_ini(ini) if isinstance(ini, str) else dict(ini or {})
        opts.update({k.lower(): v for k, v in overrides.items()})
        self.opts = resolve(opts)
        o = self.opts
        fields = to_cfg_fields(o)
        fields["device"] = device
        node_type = fields.get("node_type", 2)
        # InitMesh + CalcMetrics: the HOPR file of MeshFile, else the periodic box of the Box* keys
        if o["meshfile"]:
            from . import hopr
            path = o["meshfile"]
            if not os.path.isabs(path):
                path = os.path.join(base_dir or os.getcwd(), path)
            self.mesh_file = o["meshfile"]
            self.mesh = hopr.load_mesh(path, o["n"], node_type=node_type, mesh_scale=o["meshscale"],
                                       use_curveds=_flag(o["usecurveds"]), boundary_types=o["boundarytypes"])
        else:
            self.mesh_file = ""
            self.mesh = box_mesh(o["n"], o["boxelems"], o["boxmin"], o["boxmax"], o["ngeo"], o["meshdeformamp"],
                                 node_type=node_type)
        self.op = DGOperator(**fields)
        self.op.set_mesh(self.mesh)
        # InitDG: FillIni(IniExactFunc, U)
        if fields["eqn"] in (2, 3):
            from .workloads import mhd_exact_func
            self.U0 = mhd_exact_func(o["iniexactfunc"], 0.0, self.mesh["Elem_xGP"], kappa=o["kappa"],
                                     mu_0=o["mu_0"], ref_states=o["refstates"], ini_ref_state=o["inirefstate"],
                                     center=o["inicenter"], halfwidth=o["inihalfwidth"],
                                     amplitude=o["iniamplitude"], frequency=o["inifrequency"])
        else:
            self.U0 = exact_func(o["iniexactfunc"], 0.0, self.mesh["Elem_xGP"], kappa=o["kappa"],
                                 adv_vel=o["advvel"], amplitude=o["iniamplitude"], wavenumber=o["iniwavenumber"],
                                 frequency=o["inifrequency"], ref_state=o["refstate"])
        self.t = 0.0
        if restart_file:  # InitRestart / Restart (restart.f90:60-217), interpolated when N or the nodes differ
            from . import hopr
            st = hopr.read_state(restart_file)
            U = hopr.restart_state(st, o["n"], node_type)
            if U.shape != self.U0.shape:
                raise ValueError("restart file %s: DG_Solution shape %s does not match %s"
                                 % (restart_file, U.shape, self.U0.shape))
            self.U0 = U
            self.t = 0.0 if _flag(o["resettime"]) else st["Time"]
        self.op.set_state(self.U0)
        self.nDOF = self.op.nElems * (o["n"] + 1) ** 3
        self.nRKStages = RK_STAGES[fields["time_disc"]]

    # reference names -----------------------------------------------------------------------
    def DGTimeDerivative(self, t):
        self.op.dg_time_derivative(t)

    def CalcTimeStep(self):
        return self.op.calc_timestep()

    def TimeStep(self, t, dt):
        self.op.timestep(t, dt)

    def TimeDisc(self, t_end=None, max_iter=None):
        t_end = self.opts["tend"] if t_end is None else t_end
        max_iter = self.opts["maxiter"] if max_iter is None else max_iter
        if t_end is None:
            raise KeyError("parameter.ini: TEnd missing")
        self.t, n, err = self.op.time_disc(self.t, t_end, max_iter)
        if err:
            raise _lib.FluxoError(-4, "CALCTIMESTEP errType=%d at t=%g" % (err, self.t))
        return n

    def WriteState(self, path=None, next_time=None):
        """WriteState (src/io_hdf5/hdf5_output.f90:74-160): the current U and t to a State file
        (default name ProjectName_State_<time>.h5 in the working directory); returns the path."""
        from . import hopr
        o = self.opts
        path = path or hopr.state_file_name(o["projectname"], self.t)
        hopr.write_state(path, self.U, self.t, self.mesh_file, o["projectname"],
                         node_type="GAUSS" if self.op.cfg.node_type == 1 else "GAUSS-LOBATTO",
                         next_time=next_time)
        return path

    @property
    def U(self):
        return self.op.get_state()

    @U.setter
    def U(self, value):
        self.op.set_state(value)

    @property
    def Ut(self):
        return self.op.get_ut()


def _state_ptr_call(op, fn, ptr):
    op._check(fn(op.h, ctypes.c_void_p(ptr)))


def set_state_ptr(op, host_ptr):
    """set_state from a raw host pointer (e.g. a pinned torch tensor)."""
    _state_ptr_call(op, op.lib.fluxo_gpu_set_state, host_ptr)


def get_state_ptr(op, host_ptr):
    _state_ptr_call(op, op.lib.fluxo_gpu_get_state, host_ptr)


def profile(op, kind):
    """(total ms, launches) of one kernel kind since profiling was enabled (resets)."""
    ms, n = ctypes.c_double(), ctypes.c_uint64()
    op._check(op.lib.fluxo_gpu_get_profile(op.h, int(kind), ctypes.byref(ms), ctypes.byref(n)))
    return ms.value, n.value


def set_profiling(op, on):
    op._check(op.lib.fluxo_gpu_set_profiling(op.h, 1 if on else 0))


def fp64_peak(device=0):
    t = ctypes.c_double()
    _lib.check(_lib.load().fluxo_gpu_fp64_peak(int(device), ctypes.byref(t)))
    return t.value


def volume_shape(N, volume_flux, visc=False):
    """(candidate count, chosen index or -1, elements per block, lines per warp) of the volume kernel."""
    c, i, e, l = (ctypes.c_int() for _ in range(4))
    _lib.check(_lib.load().fluxo_gpu_volume_shape(int(N), int(volume_flux), int(bool(visc)), ctypes.byref(c),
                                                  ctypes.byref(i), ctypes.byref(e), ctypes.byref(l)))
    return c.value, i.value, e.value, l.value


def set_volume_shape(N, volume_flux, visc, index):
    """Pins the volume kernel's launch shape of (N, volume_flux, visc); index < 0 re-enables tuning."""
    _lib.check(_lib.load().fluxo_gpu_set_volume_shape(int(N), int(volume_flux), int(bool(visc)), int(index)))
