"""``parameter.ini`` reader with the reference's syntax (src/readintools/readintools.f90:453-640):
case-insensitive ``key = value`` lines, ``!`` and ``#`` comments, Fortran array literals
``(/ a, b, c /)``, logicals ``T/F/.true./.false.``.

Only the keys of the accelerated path are interpreted (see ``KEYS``); the mesh of the
reference (``MeshFile``, a HOPR HDF5 file) is replaced by a periodic box described by
the ``Box*`` keys.
"""
import re

# key -> (type, default); type 'i' int, 'r' real, 'ra' real array, 'ia' int array, 's' string
KEYS = {
    # interpolation / mesh
    "n": ("i", None),
    "boxelems": ("ia", (8, 8, 8)),
    "boxmin": ("ra", (-1.0, -1.0, -1.0)),
    "boxmax": ("ra", (1.0, 1.0, 1.0)),
    "ngeo": ("i", 1),
    "meshdeformamp": ("r", 0.0),
    # equation (navierstokes/equation.f90:65-155)
    "equation": ("s", "navierstokes"),
    "parabolic": ("s", "T"),
    "riemann": ("i", 1),
    "volumeflux": ("i", 0),
    "kappa": ("r", 1.4),
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
    # time discretisation (timedisc.f90:53-70)
    "timediscmethod": ("s", "carpenterrk4-5"),
    "tend": ("r", None),
    "cflscale": ("r", None),
    "dflscale": ("r", 0.4),
    "maxiter": ("i", -1),
    "analyze_dt": ("r", 0.0),
}

_TIMEDISC = {"carpenterrk4-5": 0, "standardrk3-3": 1}
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
    return res


def to_cfg_fields(res):
    """Maps resolved options onto the fields of ``fluxo_cfg``."""
    parabolic = str(res["parabolic"]).strip().lower() in ("t", ".true.", "true", "1")
    if str(res["equation"]).strip().lower() != "navierstokes":
        raise ValueError("only the navierstokes equation system is implemented")
    lifting = str(res["lifting"]).strip().lower()
    if lifting not in ("br1", "br2"):
        raise ValueError("lifting must be br1 or br2")
    tdm = str(res["timediscmethod"]).replace(" ", "").lower()
    if tdm not in _TIMEDISC:
        raise ValueError("TimeDiscMethod %r not implemented" % res["timediscmethod"])
    return dict(
        N=res["n"], eqn=1 if parabolic else 0, riemann=res["riemann"], volume_flux=res["volumeflux"],
        lifting=1 if lifting == "br1" else 2, lifting_var=_LIFTVAR[str(res["liftingvar"]).lower()],
        visc=_VISC[str(res["viscosity"]).lower()], kappa=res["kappa"], R=res["r"], Pr=res["pr"], mu0=res["mu0"],
        Ts=res["ts"], Tref=res["tref"], ExpoSuth=res["exposuth"], ExpoPow=res["expopow"], etaBR2=res["etabr2"],
        time_disc=_TIMEDISC[tdm], cfl_scale=res["cflscale"], dfl_scale=res["dflscale"],
        ini_exact_func=res["iniexactfunc"], ini_frequency=res["inifrequency"], ini_amplitude=res["iniamplitude"],
    )
