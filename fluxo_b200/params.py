"""``parameter.ini`` reader with the reference's syntax (src/readintools/readintools.f90:453-640):
case-insensitive ``key = value`` lines, ``!`` and ``#`` comments, Fortran array literals
``(/ a, b, c /)``, logicals ``T/F/.true./.false.``.

Only the keys of the accelerated path are interpreted (see ``KEYS``).  The mesh is the
reference's ``MeshFile`` (a HOPR HDF5 file, read by ``hopr``; ``useCurveds``, ``meshScale`` and
``BoundaryName`` / ``BoundaryType`` pairs apply as in src/mesh/mesh.f90 and mesh_readin.f90), or,
without it, a periodic box described by the ``Box*`` keys.
"""
import re

# key -> (type, default); type 'i' int, 'r' real, 'ra' real array, 'ia' int array, 's' string
KEYS = {
    # interpolation / mesh
    "n": ("i", None),
    # node set (CMake FLUXO_DISC_NODETYPE, a key here): GAUSS-LOBATTO or GAUSS
    "nodetype": ("s", "GAUSS-LOBATTO"),
    "boxelems": ("ia", (8, 8, 8)),
    "boxmin": ("ra", (-1.0, -1.0, -1.0)),
    "boxmax": ("ra", (1.0, 1.0, 1.0)),
    "ngeo": ("i", 1),
    "meshdeformamp": ("r", 0.0),
    "meshfile": ("s", None),
    "usecurveds": ("s", "T"),
    "meshscale": ("r", 1.0),
    "boundaryname": ("s", None),
    "boundarytype": ("ia", None),
    "projectname": ("s", "FLUXO"),
    "resettime": ("s", "F"),
    # equation (navierstokes/equation.f90:65-155)
    "equation": ("s", "navierstokes"),
    "parabolic": ("s", "T"),
    "riemann": ("i", 1),
    "volumeflux": ("i", 0),
    "kappa": ("r", None),  # 1.4 (Navier-Stokes), 5/3 (MHD)
    "r": ("r", 287.058),
    "pr": ("r", 0.72),
    "mu0": ("r", 0.0),
    "ts": ("r", 110.4),
    "tref": ("r", 280.0),
    "exposuth": ("r", 1.5),
    "expopow": ("r", 0.0),
    "viscosity": ("s", "constant"),
    "lifting": ("s", "br1"),
    "liftingvar": ("s", "entropy_var"),
    "etabr2": ("r", 2.0),
    "iniexactfunc": ("i", 1),
    "advvel": ("ra", (1.0, 1.0, 1.0)),
    "iniamplitude": ("r", 0.1),
    "iniwavenumber": ("ra", (1.0, 1.0, 1.0)),
    "inifrequency": ("r", 1.0),
    "refstate": ("ra", (1.0, 0.0, 0.0, 0.0, 0.71428571)),
    # MHD with GLM (mhd/equation.f90:65-135); the equation system, NONCONS and NC_GLM are build
    # options of the reference (CMake FLUXO_EQNSYSNAME, FLUXO_EQN_NONCONS_TYPE, FLUXO_EQN_NONCONS_GLM)
    # and keys here
    "inirefstate": ("i", 1),
    "inicenter": ("ra", (0.0, 0.0, 0.0)),
    "inihalfwidth": ("r", 0.1),
    "mu_0": ("r", 1.0),
    "eta": ("r", 0.0),
    "mu": ("r", 0.0),
    "glm_scale": ("r", 0.5),
    "glm_scr": ("r", 0.0),
    "noncons": ("i", 1),
    "nc_glm": ("s", "F"),
    # NFVSE shock capturing (shockcapturing.f90:55-75, nfvse.f90:63-102); "nfvse" stands for the
    # reference's build option FLUXO_SHOCKCAP_NFVSE
    "nfvse": ("s", "F"),
    "computealpha": ("i", 1),
    "shockblendcoef": ("r", 0.0),
    "modalthreshold": ("i", 1),
    "alpha_max": ("r", 0.5),
    "alpha_min": ("r", 0.01),
    "spacepropfactor": ("r", 0.5),
    "spacepropsweeps": ("i", 1),
    "timerelfactor": ("r", 0.0),
    "shockindicatorquantity": ("s", "DensityTimesPressure"),
    "subfvmethod": ("i", 1),
    "reconsboundaries": ("i", 1),
    # NFVSE_CORR (nfvse.f90:148-152); "nfvse_corr" stands for the build option FLUXO_SHOCK_NFVSE_CORR
    "nfvse_corr": ("s", "F"),
    "positcorrfactor": ("r", 0.1),
    "positmaxiter": ("i", 10),
    # time discretisation (timedisc.f90:53-70)
    "timediscmethod": ("s", "carpenterrk4-5"),
    "tend": ("r", None),
    "cflscale": ("r", None),
    "dflscale": ("r", 0.4),
    "maxiter": ("i", -1),
    "analyze_dt": ("r", 0.0),
}

# TimeDiscMethod names (timedisc_vars.f90:94-726) -> fluxo_cfg.time_disc, and their stage counts
_TIMEDISC = {"carpenterrk4-5": 0, "standardrk3-3": 1, "niegemannrk4-14": 2, "toulorgerk4-8c": 3, "toulorgerk3-7c": 4,
             "toulorgerk4-8f": 5, "ketchesonrk4-20": 6, "ketchesonrk4-18": 7, "ssprk4-5": 8, "ssprk3-3": 9}
RK_STAGES = {0: 5, 1: 3, 2: 14, 3: 8, 4: 7, 5: 8, 6: 20, 7: 18, 8: 5, 9: 3}
_INDICATOR = {"density": 1, "pressure": 2, "densitytimespressure": 3, "kinplusmagenergy": 4}
_LIFTVAR = {"cons_var": 1, "prim_var": 2, "entropy_var": 3}
_VISC = {"constant": 0, "sutherland": 1, "powerlaw": 2}


def _strip(line):
    for c in ("!", "#"):
        k = line.find(c)
        if k >= 0:
            line = line[:k]
    return line.strip()


def _parse_value(t, raw):
    raw = raw.strip()
    if t in ("ra", "ia"):
        m = re.match(r"^\(/(.*)/\)$", raw.replace(" ", ""))
        items = (m.group(1) if m else raw).split(",")
        conv = float if t == "ra" else int
        return tuple(conv(x.replace("d", "e").replace("D", "e")) for x in items if x.strip())
    if t == "i":
        return int(raw)
    if t == "r":
        return float(raw.replace("d", "e").replace("D", "e"))
    return raw


def parse_ini(text):
    """Parses parameter.ini text into a dict keyed by lower-case option name."""
    out = {}
    for line in text.splitlines():
        line = _strip(line)
        if not line or "=" not in line:
            continue
        k, v = line.split("=", 1)
        k = k.strip().lower()
        if k in KEYS:
            out[k] = _parse_value(KEYS[k][0], v)
        else:
            out[k] = v.strip()
        if k == "refstate":  # a repeated option: IniRefState selects one (equation.f90 RefStatePrim)
            out.setdefault("refstates", []).append(out[k])
        if k == "boundaryname":  # repeated pairs BoundaryName / BoundaryType (mesh_readin.f90:80-90)
            out.setdefault("boundarynames", []).append(out[k])
        if k == "boundarytype":
            out.setdefault("boundarytypes", []).append(out[k])
    return out


def resolve(opts):
    """Fills defaults and checks mandatory keys; returns a dict of resolved values."""
    res = {}
    for k, (t, dflt) in KEYS.items():
        if k in opts:
            v = opts[k]
            if isinstance(v, str) and t != "s":
                v = _parse_value(t, v)
            res[k] = v
        elif dflt is None and k in ("n", "cflscale"):
            raise KeyError("parameter.ini: mandatory option '%s' missing" % k)
        else:
            res[k] = dflt
    mhd = str(res["equation"]).strip().lower() == "mhd"
    if res["kappa"] is None:
        res["kappa"] = 5.0 / 3.0 if mhd else 1.4
    res["refstates"] = opts.get("refstates", [res["refstate"]])
    names, types = opts.get("boundarynames", []), opts.get("boundarytypes", [])
    if len(names) != len(types):
        raise ValueError("parameter.ini: every BoundaryName needs a BoundaryType")
    res["boundarytypes"] = dict(zip(names, types))
    return res


def _flag(v):
    return str(v).strip().lower() in ("t", ".true.", "true", "1")


def to_cfg_fields(res):
    """Maps resolved options onto the fields of ``fluxo_cfg``."""
    parabolic = _flag(res["parabolic"])
    eqsys = str(res["equation"]).strip().lower()
    if eqsys not in ("navierstokes", "mhd"):
        raise ValueError("equation system %r not implemented (navierstokes, mhd)" % res["equation"])
    lifting = str(res["lifting"]).strip().lower()
    if lifting not in ("br1", "br2"):
        raise ValueError("lifting must be br1 or br2")
    tdm = str(res["timediscmethod"]).replace(" ", "").lower()
    if tdm not in _TIMEDISC:
        raise ValueError("TimeDiscMethod %r not implemented" % res["timediscmethod"])
    f = dict(
        N=res["n"], eqn=1 if parabolic else 0, riemann=res["riemann"], volume_flux=res["volumeflux"],
        lifting=1 if lifting == "br1" else 2, lifting_var=_LIFTVAR[str(res["liftingvar"]).lower()],
        visc=_VISC[str(res["viscosity"]).lower()], kappa=res["kappa"], R=res["r"], Pr=res["pr"], mu0=res["mu0"],
        Ts=res["ts"], Tref=res["tref"], ExpoSuth=res["exposuth"], ExpoPow=res["expopow"], etaBR2=res["etabr2"],
        time_disc=_TIMEDISC[tdm], cfl_scale=res["cflscale"], dfl_scale=res["dflscale"],
        ini_exact_func=res["iniexactfunc"], ini_frequency=res["inifrequency"], ini_amplitude=res["iniamplitude"],
    )
    nodes = str(res["nodetype"]).strip().upper()
    if nodes not in ("GAUSS", "GAUSS-LOBATTO"):
        raise ValueError("NodeType %r not implemented (GAUSS, GAUSS-LOBATTO)" % res["nodetype"])
    f["node_type"] = 1 if nodes == "GAUSS" else 2
    ind = str(res["shockindicatorquantity"]).strip().lower()
    if ind not in _INDICATOR:
        raise ValueError("ShockIndicatorQuantity %r not implemented" % res["shockindicatorquantity"])
    f.update(nfvse=1 if _flag(res["nfvse"]) else 0,
             compute_alpha=res["computealpha"], shock_blend_coef=res["shockblendcoef"],
             modal_threshold=res["modalthreshold"], alpha_max=res["alpha_max"], alpha_min=res["alpha_min"],
             space_prop_factor=res["spacepropfactor"], space_prop_sweeps=res["spacepropsweeps"],
             time_rel_factor=res["timerelfactor"], indicator_quantity=_INDICATOR[ind],
             sub_fv_method=res["subfvmethod"], recons_boundaries=res["reconsboundaries"],
             nfvse_corr=1 if _flag(res["nfvse_corr"]) else 0, posit_corr_factor=res["positcorrfactor"],
             posit_max_iter=res["positmaxiter"])
    if eqsys == "mhd":
        f.update(eqn=3 if parabolic else 2, mu0=res["mu"], mu_0=res["mu_0"], eta=res["eta"],
                 glm_scale=res["glm_scale"], glm_scr=res["glm_scr"], noncons=res["noncons"],
                 nc_glm=1 if _flag(res["nc_glm"]) else 0)
    return f
