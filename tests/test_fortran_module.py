"""The Fortran interface module (include/cfd_b200_mod.f90) against the C header: every
function of cfd_b200.h has a bind(c) interface of the same name, the same argument count,
C scalars passed with `value` and C pointers passed by reference or as type(c_ptr), value;
the bind(c) derived types list the C struct fields in the same order (CPU; no Fortran
compiler is needed to check this)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "cfd_b200.h")
MOD = os.path.join(ROOT, "include", "cfd_b200_mod.f90")


def _strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def header_functions():
    s = _strip_c_comments(open(HDR).read())
    out = {}
    for m in re.finditer(r"(?:^|\n)\s*(?:int|const char \*)\s*(cfd_\w+)\s*\(([^)]*)\)\s*;", s):
        params = [p.strip() for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        out[m.group(1)] = [("*" in p) for p in params]
    return out


def header_structs():
    s = _strip_c_comments(open(HDR).read())
    out = {}
    for m in re.finditer(r"typedef struct (cfd_\w+) \{(.*?)\}", s, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            names = decl.split(None, 1)[1] if not decl.startswith("const") else decl.split("*", 1)[1]
            for n in names.replace("*", " ").split(","):
                n = re.sub(r"\[.*?\]", "", n).strip().split()[-1]
                fields.append(n)
        out[m.group(1)] = fields
    return out


def module_text():
    lines = []
    for ln in open(MOD):
        ln = ln.split("!")[0].rstrip()
        if lines and lines[-1].endswith("&"):
            lines[-1] = lines[-1][:-1] + " " + ln.strip()
        else:
            lines.append(ln)
    return "\n".join(lines)


def module_functions():
    t = module_text()
    out = {}
    for m in re.finditer(r"function (cfd_\w+)\(([^)]*)\)\s*bind\(c, name='(\w+)'\)(.*?)end function", t, flags=re.S):
        name, args, cname, body = m.group(1), m.group(2), m.group(3), m.group(4)
        assert name == cname, (name, cname)
        dummies = [a.strip() for a in args.split(",") if a.strip()]
        kinds = []
        for a in dummies:
            part = None
            for line in body.split("\n"):
                for seg in line.split(";"):
                    if "::" in seg and re.search(r"\b%s\b" % a, seg.split("::")[1]):
                        part = seg
            assert part is not None, (name, a)
            attrs = part.split("::")[0]
            kinds.append(("value" in attrs, "type(c_ptr)" in attrs))
        out[name] = kinds
    return out


def module_types():
    t = module_text()
    out = {}
    for m in re.finditer(r"type, bind\(c\) :: (cfd_\w+)(.*?)end type", t, flags=re.S):
        fields = []
        for line in m.group(2).split("\n"):
            if "::" in line:
                for n in line.split("::")[1].split(","):
                    fields.append(re.sub(r"\(.*?\)", "", n).strip())
        out[m.group(1)] = fields
    return out


def test_every_header_function_has_an_interface():
    h, f = header_functions(), module_functions()
    assert len(h) > 40
    assert sorted(h) == sorted(f), (set(h) ^ set(f))


@pytest.mark.parametrize("name", sorted(header_functions()))
def test_argument_passing(name):
    cptr = header_functions()[name]
    fk = module_functions()[name]
    assert len(cptr) == len(fk), name
    for i, (is_ptr, (value, is_cptr)) in enumerate(zip(cptr, fk)):
        if is_ptr:   # by reference, or a c_ptr passed by value
            assert (not value) or is_cptr, (name, i)
        else:        # a C scalar: by value, not a pointer type
            assert value and not is_cptr, (name, i)


def test_struct_layouts():
    h, f = header_structs(), module_types()
    for s in ("cfd_config", "cfd_ib_list", "cfd_tuning", "cfd_stats_config"):
        assert h[s] == f[s], (s, h[s], f[s])
