"""The Fortran ISO_C_BINDING interfaces (nemoh_b200/fortran/*.f90) against the
C prototypes of include/nemoh_b200.h, position by position: a Fortran host that
compiles these modules passes each argument the way the C entry point reads
it. No Fortran compiler is needed; the check is on the source text."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nemoh_b200.h")
FORTRAN = sorted(glob.glob(os.path.join(ROOT, "nemoh_b200", "fortran", "*.f90")))


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"(?:^|\n)\s*([A-Za-z_][\w\s\*]*?)\b(nemoh_b200_\w+)\s*\(([^;{]*?)\)\s*;", text):
        params = [p.strip() for p in m.group(3).split(",") if p.strip() and p.strip() != "void"]
        kinds = []
        for p in params:
            p = re.sub(r"\s+", " ", p)
            ptr = p.count("*")
            base = re.sub(r"\bconst\b", "", p.replace("*", " ")).split()[0]
            kinds.append((base, ptr))
        out[m.group(2)] = kinds
    return out


def fortran_interfaces(path):
    lines, buf = [], ""
    for raw in open(path):
        line = raw.split("!", 1)[0].rstrip()
        if buf:
            line = buf + " " + line.strip()
            buf = ""
        if line.endswith("&"):
            buf = line[:-1]
            continue
        lines.append(line)
    out = {}
    it = iter(lines)
    for line in it:
        m = re.search(r"FUNCTION\s+(\w+)\s*\(([^)]*)\)\s*BIND\s*\(\s*C\s*,\s*NAME\s*=\s*'(\w+)'", line, re.I)
        if not m:
            continue
        args = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
        decl = {}
        for body in it:
            if re.match(r"\s*END\s+FUNCTION", body, re.I):
                break
            d = re.match(r"\s*(INTEGER\(C_INT\)|REAL\(C_DOUBLE\)|COMPLEX\(C_DOUBLE_COMPLEX\)|TYPE\(C_PTR\))"
                         r"((?:\s*,\s*[\w(),*:]+?)*)\s*::\s*(.+)$", body, re.I)
            if not d:
                continue
            ftype = d.group(1).upper()
            attrs = d.group(2).upper()
            for name in d.group(3).split(","):
                decl[name.strip().lower()] = (ftype, "VALUE" in attrs)
        out[m.group(3)] = [decl[a] for a in args]
    return out


def compatible(c, f):
    (base, ptr), (ftype, value) = c, f
    if base == "nemoh_ctx":
        # the context handle: by value (C_PTR, VALUE) or its address (C_PTR)
        return ftype == "TYPE(C_PTR)" and value == (ptr == 1)
    if ptr == 0:
        return value and ftype == {"int": "INTEGER(C_INT)", "double": "REAL(C_DOUBLE)"}.get(base)
    if ptr == 1 and not value:
        # complex arrays cross as interleaved doubles
        return ftype in {"int": ("INTEGER(C_INT)",), "double": ("REAL(C_DOUBLE)", "COMPLEX(C_DOUBLE_COMPLEX)")}.get(
            base, ())
    return False


@pytest.mark.parametrize("path", FORTRAN, ids=[os.path.basename(p) for p in FORTRAN])
def test_fortran_interfaces_match_c_prototypes(path):
    protos = c_prototypes()
    ifaces = fortran_interfaces(path)
    assert ifaces, path
    for name, fargs in ifaces.items():
        assert name in protos, name
        cargs = protos[name]
        assert len(fargs) == len(cargs), (name, len(fargs), len(cargs))
        for i, (c, f) in enumerate(zip(cargs, fargs)):
            assert compatible(c, f), (name, i, c, f)


def test_header_parser_sees_every_entry_point():
    protos = c_prototypes()
    for name in ("nemoh_b200_create", "nemoh_b200_set_mesh", "nemoh_b200_solve_problem",
                 "nemoh_b200_solve_frequencies", "nemoh_b200_kochin", "nemoh_b200_free_surface", "nemoh_b200_irf"):
        assert name in protos
    assert protos["nemoh_b200_create"] == [("nemoh_ctx", 2), ("int", 0), ("int", 0)]
