"""The Fortran host's ISO_C_BINDING module against the C header it binds.

No Fortran compiler is needed: the module is read as text.  Its derived type
mhd3d_params must list the C struct's fields in the same order with matching
kinds, every bind(C) function must name an exported symbol with the C
prototype's argument count, and the named constants must equal the header's.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "rast-3dmhd_b200", "fortran", "mhd3d_gpu.f90")
HDR = os.path.join(ROOT, "include", "mhd3d.h")


def _f90():
    src = open(F90).read()
    src = re.sub(r"!.*", "", src)                 # comments
    return re.sub(r"&\s*\n\s*&?", " ", src)       # continuation lines


def _hdr():
    return re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)


def _c_struct_fields():
    body = re.search(r"typedef struct mhd3d_params \{(.*?)\} mhd3d_params;", _hdr(), re.S).group(1)
    out = []
    for decl in body.split(";"):
        m = re.match(r"\s*(int32_t|double)\s+(.*)", decl.strip())
        if m:
            kind = "int" if m.group(1) == "int32_t" else "double"
            out += [(n.strip(), kind) for n in m.group(2).split(",")]
    return out


def _f_type_fields():
    body = re.search(r"type, bind\(C\) :: mhd3d_params(.*?)end type", _f90(), re.S | re.I).group(1)
    out = []
    for line in body.strip().splitlines():
        m = re.match(r"\s*(integer\(c_int32_t\)|real\(c_double\))\s*::\s*(.*)", line, re.I)
        if m:
            kind = "int" if m.group(1).lower().startswith("integer") else "double"
            out += [(n.strip(), kind) for n in m.group(2).split(",")]
    return out


def test_params_type_matches_struct():
    c, f = _c_struct_fields(), _f_type_fields()
    assert len(c) > 40
    assert f == c


def _c_argc(name):
    m = re.search(r"\b%s\s*\(([^)]*)\)" % name, _hdr(), re.S)
    assert m, name
    args = m.group(1).strip()
    return 0 if args in ("", "void") else len(args.split(","))


def test_bound_functions_match_prototypes(mhd3d):
    lib = mhd3d.gpu_lib()
    funcs = re.findall(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", _f90(), re.I)
    assert len(funcs) >= 8
    for fname, args, cname in funcs:
        assert fname == cname
        assert hasattr(lib, cname), cname
        nargs = len([a for a in args.split(",") if a.strip()])
        assert nargs == _c_argc(cname), (cname, nargs, _c_argc(cname))


def test_constants_match_header():
    hdr = dict(re.findall(r"#define\s+(MHD3D_\w+)\s+(-?\d+)", _hdr()))
    consts = re.findall(r"(MHD3D_\w+)\s*=\s*(-?\d+)", _f90())
    assert len(consts) >= 10
    for name, val in consts:
        assert name in hdr, name
        assert int(hdr[name]) == int(val), name
