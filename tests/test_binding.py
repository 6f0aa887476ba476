"""The Fortran binding documented in INTEGRATION.md matches the C ABI of include/fluxo_gpu.h.

A maintainer pastes that ISO_C_BINDING module into the reference (there is no Fortran compiler in this
image, so it is checked here by parsing): the TYPE, BIND(C) blocks must list the C structs' fields in
the same order with interoperable kinds and give the same size under C layout rules (and the same as
the ctypes binding of fluxo_b200/_lib.py), and every fluxo_gpu_* / fluxo_batch_* entry point of the
header must have an INTERFACE with the same name, argument count, and for each argument an
interoperable kind passed by value or by reference as the C prototype takes it."""
import ctypes
import os
import re

import pytest

from fluxo_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = open(os.path.join(ROOT, "include", "fluxo_gpu.h")).read()
DOC = open(os.path.join(ROOT, "INTEGRATION.md")).read()

C_SCALAR = {"int": ("C_INT", 4), "double": ("C_DOUBLE", 8), "size_t": ("C_SIZE_T", 8)}


def strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def c_structs():
    """{name: [(field, c_type, count)]} of the typedef'd structs of the header."""
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", strip_c_comments(HEADER), flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ty, rest = decl.split(None, 1)
            for name in rest.split(","):
                name = name.strip()
                a = re.match(r"(\w+)\[(\d+)\]", name)
                fields.append((a.group(1), ty, int(a.group(2))) if a else (name, ty, 1))
        out[m.group(1)] = fields
    return out


def c_functions():
    """{name: [normalised parameter types]} of the header's prototypes."""
    out = {}
    for m in re.finditer(r"\bint (fluxo_\w+)\((.*?)\);", strip_c_comments(HEADER), flags=re.S):
        params = []
        for p in m.group(2).split(","):
            p = " ".join(p.replace("const ", "").split())
            ty = re.match(r"([\w ]+?)\s*(\**)\s*\w+$", p)
            params.append(ty.group(1).strip() + ty.group(2))
        out[m.group(1)] = params
    return out


def fortran_statements():
    """Statements of the documented Fortran code (continuations joined, ';' split, comments dropped)."""
    code = "\n".join(re.findall(r"```fortran\n(.*?)```", DOC, flags=re.S))
    code = re.sub(r"!.*", "", code)
    code = re.sub(r"&\s*\n\s*", " ", code)
    stmts = []
    for line in code.splitlines():
        stmts += [s.strip() for s in line.split(";") if s.strip()]
    return stmts


def parse_decl(stmt):
    """'REAL(C_DOUBLE), VALUE :: a, b(3)' -> (kind, value, [(name, count)])."""
    spec, names = stmt.split("::")
    kind = re.match(r"(?:INTEGER|REAL|CHARACTER|TYPE)\((?:KIND=)?(\w+)\)", spec.strip()).group(1)
    value = "VALUE" in spec.upper()
    out = []
    for n in re.findall(r"(\w+)(\([^)]*\))?", names):
        dims = n[1]
        cnt = int(dims[1:-1]) if dims and dims[1:-1].isdigit() else (None if dims else 1)
        out.append((n[0], cnt))
    return kind, value, out


def fortran_types():
    out, cur = {}, None
    for s in fortran_statements():
        m = re.match(r"TYPE, BIND\(C\) :: (\w+)", s)
        if m:
            cur = out.setdefault(m.group(1), [])
            continue
        if s.startswith("END TYPE"):
            cur = None
            continue
        if cur is not None:
            kind, _, names = parse_decl(s)
            cur += [(n, kind, c) for n, c in names]
    return out


def fortran_functions():
    out, cur = {}, None
    for s in fortran_statements():
        m = re.match(r"INTEGER\(C_INT\) FUNCTION (\w+)\(([^)]*)\)\s*BIND\(C, NAME='(\w+)'\)", s)
        if m:
            assert m.group(1) == m.group(3), s
            cur = {"args": [a.strip() for a in m.group(2).split(",") if a.strip()], "decl": {}}
            out[m.group(1)] = cur
            continue
        if s.startswith("END FUNCTION"):
            cur = None
            continue
        if cur is not None and "::" in s:
            kind, value, names = parse_decl(s)
            for n, _ in names:
                cur["decl"][n] = (kind, value)
    return out


def c_layout_size(fields):
    off, align = 0, 1
    for _, ty, cnt in fields:
        sz = C_SCALAR[ty][1]
        off = (off + sz - 1) // sz * sz + sz * cnt
        align = max(align, sz)
    return (off + align - 1) // align * align


@pytest.mark.parametrize("name,ctype", [("fluxo_cfg", _lib.FluxoCfg), ("fluxo_exact", _lib.FluxoExact)])
def test_structs_match(name, ctype):
    c = c_structs()[name]
    f = fortran_types()[name]
    assert [x[0] for x in f] == [x[0] for x in c], name
    for (fn, fk, fc), (cn, ct, cc) in zip(f, c):
        assert fk == C_SCALAR[ct][0] and fc == cc, (name, fn, fk, ct)
    py = [(n, t) for n, t in ctype._fields_]
    assert [n for n, _ in py] == [x[0] for x in c]
    for (n, t), (_, ct, cc) in zip(py, c):
        base = {"int": ctypes.c_int, "double": ctypes.c_double}[ct]
        assert t == (base if cc == 1 else base * cc), n
    assert c_layout_size(c) == ctypes.sizeof(ctype)


def compatible(ctype, kind, value):
    if ctype in ("int", "double", "size_t"):
        return value and kind == C_SCALAR[ctype][0]
    if ctype == "fluxo_exchange_fn":  # a C function pointer passed by value
        return value and kind == "C_FUNPTR"
    if ctype.endswith("**"):
        return kind == "C_PTR" and not value
    base = ctype[:-1]
    if value:  # a pointer passed as an address
        return kind == "C_PTR" and base in ("void", "fluxo_handle", "fluxo_batch", "fluxo_batch_prepared", "double", "int")
    return {"int": "C_INT", "double": "C_DOUBLE", "size_t": "C_SIZE_T", "uint64_t": "C_INT64_T", "char": "C_CHAR",
            "fluxo_cfg": "fluxo_cfg", "fluxo_exact": "fluxo_exact"}.get(base) == kind


def test_every_entry_point_bound():
    cf, ff = c_functions(), fortran_functions()
    need = [n for n in cf if n.startswith(("fluxo_gpu_", "fluxo_batch_"))]
    assert len(need) >= 35
    missing = [n for n in need if n not in ff]
    assert not missing, missing
    for name in need:
        f = ff[name]
        assert len(f["args"]) == len(cf[name]), name
        for a, ct in zip(f["args"], cf[name]):
            kind, value = f["decl"][a]
            assert compatible(ct, kind, value), (name, a, ct, kind, value)
