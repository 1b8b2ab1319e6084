"""The Fortran iso_c_binding module (ibfs-if2d_b200/fortran/ibfs_gpu.f90)
against include/ibfs_capi.h: every BIND(C) name is a declared entry point with
the same number of arguments, and the BIND(C) derived types list the C
structs' fields in the same order with matching kinds. (No Fortran compiler is
installed here, so the module is checked as text.)"""
import os
import re

from conftest import PKG, ROOT

F90 = open(os.path.join(PKG, "fortran", "ibfs_gpu.f90")).read()
MAIN = open(os.path.join(PKG, "fortran", "main_gpu.f90")).read()
HDR = open(os.path.join(ROOT, "include", "ibfs_capi.h")).read()


def c_functions():
    out = {}
    for m in re.finditer(r"\b(?:int|const char\*)\s+(ibfs_[a-z0-9_]+)\s*\(([^;]*?)\);", HDR, re.S):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def f_functions():
    out = {}
    for m in re.finditer(r"FUNCTION\s+(\w+)\s*\(([^)]*)\)\s*&?\s*BIND\(C,\s*name=\"(\w+)\"\)", F90):
        out[m.group(3)] = len([a for a in m.group(2).split(",") if a.strip()])
    return out


def c_struct(name):
    body = {m.group(2): m.group(1) for m in re.finditer(r"typedef struct \{(.*?)\}\s*(\w+);", HDR, re.S)}[name]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, names = decl.split(None, 1)
        fields += [(typ, n.strip()) for n in names.split(",")]
    return fields


def f_type(name):
    body = re.search(r"TYPE, BIND\(C\) :: " + name + r"\n(.*?)END TYPE", F90, re.S).group(1)
    fields = []
    for line in body.splitlines():
        m = re.match(r"\s*(INTEGER\(C_INT\)|REAL\(C_DOUBLE\))\s*::\s*(.*)", line)
        if m:
            typ = "int" if m.group(1).startswith("INTEGER") else "double"
            fields += [(typ, n.strip()) for n in m.group(2).split(",")]
    return fields


def test_bind_c_names_and_arity():
    c, f = c_functions(), f_functions()
    assert len(f) >= 10
    for name, n in f.items():
        assert name in c, name
        assert c[name] == n, (name, c[name], n)


def test_bind_c_types_match_structs():
    for name in ("ibfs_params_c", "ibfs_options_c"):
        assert f_type(name) == c_struct(name), name


def test_driver_program_uses_the_module():
    assert "USE ibfs_gpu" in MAIN and "CALL input" in MAIN and "CALL setup_variables" in MAIN
    for fn in re.findall(r"\b(ibfs_[a-z_]+)\(", MAIN):
        assert fn in f_functions() or fn in ("ibfs_stop_on", "ibfs_params_c", "ibfs_options_c"), fn
