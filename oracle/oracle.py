"""Oracle test infrastructure: ctypes loader for the CPU restatement of the
reference DGSEM right-hand side (``liboracle.so``, built by ``oracle/Makefile``).

Only the test-suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg
of ``bench.py`` import this module, and only as the checker.  Arrays follow the
reference's Fortran layouts (first index fastest); numpy arrays returned here
are C-ordered views of those buffers, e.g. ``U[e, k, j, i, v]``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int),
        ("nElems", ctypes.c_int * 3),
        ("xmin", ctypes.c_double * 3),
        ("xmax", ctypes.c_double * 3),
        ("NGeo", ctypes.c_int),
        ("deform_amp", ctypes.c_double),
        ("eqn", ctypes.c_int),
        ("lifting", ctypes.c_int),
        ("lifting_var", ctypes.c_int),
        ("visc", ctypes.c_int),
        ("riemann", ctypes.c_int),
        ("volume_flux", ctypes.c_int),
        ("kappa", ctypes.c_double),
        ("R", ctypes.c_double),
        ("Pr", ctypes.c_double),
        ("mu0", ctypes.c_double),
        ("Ts", ctypes.c_double),
        ("Tref", ctypes.c_double),
        ("ExpoSuth", ctypes.c_double),
        ("ExpoPow", ctypes.c_double),
        ("etaBR2", ctypes.c_double),
        ("ini_exact_func", ctypes.c_int),
        ("adv_vel", ctypes.c_double * 3),
        ("ini_amplitude", ctypes.c_double),
        ("ini_wavenumber", ctypes.c_double * 3),
        ("ini_frequency", ctypes.c_double),
        ("ref_state", ctypes.c_double * 5),
        ("cfl_scale", ctypes.c_double),
        ("dfl_scale", ctypes.c_double),
        ("time_disc", ctypes.c_int),
        ("mu_0", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("glm_scale", ctypes.c_double),
        ("glm_scr", ctypes.c_double),
        ("glm_ch", ctypes.c_double),
        ("noncons", ctypes.c_int),
        ("nc_glm", ctypes.c_int),
        ("mhd_ref_state", (ctypes.c_double * 8) * 2),
        ("ini_center", ctypes.c_double * 3),
        ("ini_halfwidth", ctypes.c_double),
        ("nfvse", ctypes.c_int),
        ("compute_alpha", ctypes.c_int),
        ("shock_blend_coef", ctypes.c_double),
        ("modal_threshold", ctypes.c_int),
        ("alpha_max", ctypes.c_double),
        ("alpha_min", ctypes.c_double),
        ("space_prop_factor", ctypes.c_double),
        ("space_prop_sweeps", ctypes.c_int),
        ("time_rel_factor", ctypes.c_double),
        ("indicator_quantity", ctypes.c_int),
        ("sub_fv_method", ctypes.c_int),
        ("recons_boundaries", ctypes.c_int),
        ("nfvse_corr", ctypes.c_int),
        ("posit_corr_factor", ctypes.c_double),
        ("posit_max_iter", ctypes.c_int),
        ("node_type", ctypes.c_int),
    ]


DEFAULTS = dict(
    N=3, nElems=(2, 2, 2), xmin=(0.0, 0.0, 0.0), xmax=(2.0, 2.0, 2.0), NGeo=1, deform_amp=0.0,
    eqn=0, lifting=1, lifting_var=3, visc=0, riemann=1, volume_flux=10,
    kappa=1.4, R=287.058, Pr=0.72, mu0=0.0, Ts=110.4, Tref=280.0, ExpoSuth=1.5, ExpoPow=0.0,
    etaBR2=2.0, ini_exact_func=2, adv_vel=(1.0, 1.0, 1.0), ini_amplitude=0.1,
    ini_wavenumber=(1.0, 1.0, 1.0), ini_frequency=1.0, ref_state=(1.0, 0.3, 0.0, 0.0, 0.71428571),
    cfl_scale=0.9, dfl_scale=0.4, time_disc=0,
    mu_0=1.0, eta=0.0, glm_scale=0.5, glm_scr=0.0, glm_ch=0.0, noncons=1, nc_glm=0,
    mhd_ref_state=((1.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0), (1.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0)),
    ini_center=(0.0, 0.0, 0.0), ini_halfwidth=0.1,
    nfvse=0, compute_alpha=1, shock_blend_coef=0.0, modal_threshold=1, alpha_max=0.5, alpha_min=0.01,
    space_prop_factor=0.5, space_prop_sweeps=1, time_rel_factor=0.0, indicator_quantity=3,
    sub_fv_method=1, recons_boundaries=1, nfvse_corr=0, posit_corr_factor=0.1, posit_max_iter=10,
    node_type=2,
)


def build(quiet=True):
    """Compile the oracle libraries in place (gcc; no GPU needed)."""
    out = subprocess.run(["make", "-C", _HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _lib(counting=False):
    name = "liboracle_count.so" if counting else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    d, i = ctypes.c_double, ctypes.c_int
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [P(OrcParams)]
    lib.orc_create_hopr.restype = ctypes.c_void_p
    lib.orc_create_hopr.argtypes = [P(OrcParams), i, ctypes.c_void_p, i, ctypes.c_void_p, i, ctypes.c_void_p, i, i,
                                    ctypes.c_void_p, d, i]
    lib.orc_destroy.argtypes = [ctypes.c_void_p]
    lib.orc_sizes.argtypes = [ctypes.c_void_p, P(i), P(i), P(i), P(i)]
    lib.orc_get_mesh.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 11
    lib.orc_set_metrics.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 8
    lib.orc_get_U.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_set_U.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_dg_time_derivative.argtypes = [ctypes.c_void_p, d, ctypes.c_void_p]
    lib.orc_get_gradients.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 3
    lib.orc_calc_timestep.restype = d
    lib.orc_calc_timestep.argtypes = [ctypes.c_void_p, P(i)]
    lib.orc_timestep.argtypes = [ctypes.c_void_p, d, d]
    lib.orc_run.restype = d
    lib.orc_run.argtypes = [ctypes.c_void_p, d, d, i, P(i)]
    lib.orc_analyze.argtypes = [ctypes.c_void_p, d] + [ctypes.c_void_p] * 6
    lib.orc_exact_func.argtypes = [ctypes.c_void_p, i, d, i, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_basis.argtypes = [i] + [ctypes.c_void_p] * 8
    lib.orc_flops.restype = ctypes.c_uint64
    lib.orc_phase_flops.restype = ctypes.c_uint64
    lib.orc_phase_flops.argtypes = [i]
    lib.orc_volume_flux.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
    lib.orc_riemann_point.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6
    lib.orc_ln_mean.restype = d
    lib.orc_ln_mean.argtypes = [d, d]
    lib.orc_get_alpha.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_set_alpha.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_corr_error.restype = ctypes.c_int
    lib.orc_get_surf_metrics.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_corr_error.argtypes = [ctypes.c_void_p]
    lib.orc_set_glm_ch.argtypes = [ctypes.c_void_p, d]
    lib.orc_get_glm_ch.restype = d
    lib.orc_get_glm_ch.argtypes = [ctypes.c_void_p]
    _LIBS[name] = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def make_params(**kw):
    vals = dict(DEFAULTS)
    for k, v in kw.items():
        if k not in vals:
            raise KeyError(k)
        vals[k] = v
    p = OrcParams()
    for k, v in vals.items():
        f = getattr(p, k)
        if isinstance(f, ctypes.Array):
            for n, x in enumerate(v):
                if isinstance(f[n], ctypes.Array):
                    for m, y in enumerate(x):
                        f[n][m] = y
                else:
                    f[n] = x
        else:
            setattr(p, k, v)
    return p


class OracleCase:
    """One discretised case (mesh + state) in the CPU oracle."""

    def __init__(self, counting=False, hopr=None, **kw):
        """``hopr``: the arrays of a HOPR mesh file (keys ElemInfo, SideInfo, BCType, NodeCoords,
        NGeo, optional nodes_gl, mesh_scale, use_curveds) instead of the periodic box."""
        self.lib = _lib(counting)
        self.params = make_params(**kw)
        if hopr is None:
            self.h = self.lib.orc_create(ctypes.byref(self.params))
        else:
            self._hopr = {k: np.ascontiguousarray(hopr[k], dtype=np.int32) for k in ("ElemInfo", "SideInfo", "BCType")}
            self._hopr["NodeCoords"] = np.ascontiguousarray(hopr["NodeCoords"], dtype=np.float64)
            self.h = self.lib.orc_create_hopr(
                ctypes.byref(self.params), self._hopr["ElemInfo"].shape[0], _ptr(self._hopr["ElemInfo"]),
                self._hopr["SideInfo"].shape[0], _ptr(self._hopr["SideInfo"]), self._hopr["BCType"].shape[0],
                _ptr(self._hopr["BCType"]), int(hopr["NGeo"]), int(hopr.get("nodes_gl", 0)),
                _ptr(self._hopr["NodeCoords"]), float(hopr.get("mesh_scale", 1.0)), int(hopr.get("use_curveds", 1)))
        if not self.h:
            raise RuntimeError("oracle: case creation failed")
        ne, ns, nv, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.orc_sizes(self.h, ne, ns, nv, n)
        self.nElems, self.nSides, self.nVar, self.N = ne.value, ns.value, nv.value, n.value
        self.np = self.N + 1

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    # shapes in C order (reverse of the Fortran dimensions)
    def vol_shape(self, lead):
        n = self.np
        return (self.nElems, n, n, n) + ((lead,) if lead else ())

    def face_shape(self, lead):
        n = self.np
        return (self.nSides, n, n) + ((lead,) if lead else ())

    def mesh(self):
        m = {
            "SideToElem": np.zeros((self.nSides, 5), np.int32),
            "ElemToSide": np.zeros((self.nElems, 6, 2), np.int32),
            "Metrics_fTilde": np.zeros(self.vol_shape(3)),
            "Metrics_gTilde": np.zeros(self.vol_shape(3)),
            "Metrics_hTilde": np.zeros(self.vol_shape(3)),
            "sJ": np.zeros(self.vol_shape(0)),
            "NormVec": np.zeros(self.face_shape(3)),
            "TangVec1": np.zeros(self.face_shape(3)),
            "TangVec2": np.zeros(self.face_shape(3)),
            "SurfElem": np.zeros(self.face_shape(0)),
            "Elem_xGP": np.zeros(self.vol_shape(3)),
        }
        self.lib.orc_get_mesh(self.h, *[_ptr(m[k]) for k in (
            "SideToElem", "ElemToSide", "Metrics_fTilde", "Metrics_gTilde", "Metrics_hTilde", "sJ",
            "NormVec", "TangVec1", "TangVec2", "SurfElem", "Elem_xGP")])
        if self.params.node_type == 1:
            m["SurfMetrics"] = self.surf_metrics()
        return m

    def set_metrics(self, m):
        arrs = [np.ascontiguousarray(m[k], dtype=np.float64) for k in (
            "Metrics_fTilde", "Metrics_gTilde", "Metrics_hTilde", "sJ", "NormVec", "TangVec1",
            "TangVec2", "SurfElem")]
        self.lib.orc_set_metrics(self.h, *[_ptr(a) for a in arrs])

    def get_U(self):
        U = np.zeros(self.vol_shape(self.nVar))
        self.lib.orc_get_U(self.h, _ptr(U))
        return U

    def set_U(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == self.nElems * self.np ** 3 * self.nVar
        self.lib.orc_set_U(self.h, _ptr(U))

    def dg_time_derivative(self, t=0.0):
        Ut = np.zeros(self.vol_shape(self.nVar))
        self.lib.orc_dg_time_derivative(self.h, t, _ptr(Ut))
        return Ut

    def gradients(self):
        g = [np.zeros(self.vol_shape(self.nVar)) for _ in range(3)]
        self.lib.orc_get_gradients(self.h, *[_ptr(a) for a in g])
        return g

    def calc_timestep(self):
        err = ctypes.c_int()
        dt = self.lib.orc_calc_timestep(self.h, ctypes.byref(err))
        return dt, err.value

    def timestep(self, t, dt):
        self.lib.orc_timestep(self.h, t, dt)

    def run(self, t, t_end, max_iter=-1):
        n = ctypes.c_int()
        t = self.lib.orc_run(self.h, t, t_end, max_iter, ctypes.byref(n))
        return t, n.value

    def analyze(self, t):
        L2, Linf = np.zeros(self.nVar), np.zeros(self.nVar)
        S, dS, ek, en = (ctypes.c_double() for _ in range(4))
        self.lib.orc_analyze(self.h, t, _ptr(L2), _ptr(Linf), ctypes.byref(S), ctypes.byref(dS),
                             ctypes.byref(ek), ctypes.byref(en))
        return dict(L2=L2, Linf=Linf, entropy=S.value, dSdU_Ut=dS.value, ekin=ek.value,
                    enstrophy=en.value)

    def exact(self, func, t, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        U = np.zeros((x.shape[0], self.nVar))
        self.lib.orc_exact_func(self.h, func, t, x.shape[0], _ptr(x), _ptr(U))
        return U

    def alpha(self):
        """NFVSE blending coefficient per element after the last right-hand side."""
        a = np.zeros(self.nElems)
        self.lib.orc_get_alpha(self.h, _ptr(a))
        return a

    def set_alpha(self, alpha):
        """NFVSE blending coefficients that the next right-hand side starts from."""
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        assert a.size == self.nElems
        self.lib.orc_set_alpha(self.h, _ptr(a))

    def surf_metrics(self):
        """Gauss nodes: SurfMetrics(3,0:N,0:N,6,nElems) as a C-order array [e, side, q, p, 3]."""
        n = self.N + 1
        a = np.zeros((self.nElems, 6, n, n, 3))
        self.lib.orc_get_surf_metrics(self.h, _ptr(a))
        return a

    @property
    def corr_error(self):
        """NFVSE_CORR: element + 1 whose safe state was not admissible (0: none)."""
        return self.lib.orc_corr_error(self.h)

    @property
    def glm_ch(self):
        return self.lib.orc_get_glm_ch(self.h)

    @glm_ch.setter
    def glm_ch(self, ch):
        self.lib.orc_set_glm_ch(self.h, float(ch))

    def volume_flux(self, UL, UR, mL, mR):
        F = np.zeros(self.nVar)
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (UL, UR, mL, mR)]
        self.lib.orc_volume_flux(self.h, *[_ptr(v) for v in a], _ptr(F))
        return F

    def riemann(self, UL, UR, nv, t1, t2):
        F = np.zeros(self.nVar)
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (UL, UR, nv, t1, t2)]
        self.lib.orc_riemann_point(self.h, *[_ptr(v) for v in a], _ptr(F))
        return F


def basis(N):
    lib = _lib()
    n = N + 1
    out = dict(xGP=np.zeros(n), wGP=np.zeros(n), wBary=np.zeros(n), D=np.zeros((n, n)),
               Dvolsurf=np.zeros((n, n)), Dhat=np.zeros((n, n)), Lminus=np.zeros(n), Lplus=np.zeros(n))
    lib.orc_basis(N, *[_ptr(out[k]) for k in ("xGP", "wGP", "wBary", "D", "Dvolsurf", "Dhat", "Lminus", "Lplus")])
    # matrices come back column-major (Fortran): transpose to (row, col)
    for k in ("D", "Dvolsurf", "Dhat"):
        out[k] = out[k].T.copy()
    return out


PHASES = ("volume_split_form", "lifting", "volume_viscous", "face_flux", "surface_integral", "jacobian_source",
          "nfvse")


def count_flops(**kw):
    """FP64 operation count of one DGTimeDerivative (counting build): total and per phase,
    both per DOF.  Counting rules in oracle/counted.h."""
    lib = _lib(counting=True)
    c = OracleCase(counting=True, **kw)
    lib.orc_reset_flops()
    c.dg_time_derivative(0.0)
    nd = c.nElems * c.np ** 3
    return int(lib.orc_flops()) / nd, {k: int(lib.orc_phase_flops(i)) / nd for i, k in enumerate(PHASES)}


def ln_mean(a, b):
    return _lib().orc_ln_mean(a, b)
