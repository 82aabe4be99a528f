"""include/half_api.f90, the Fortran twin of the C ABI, against the C headers
and the built library (CPU only: text parsing plus symbol lookup).

Every bind(C) interface must name a symbol that include/half.h or
include/half_b200.h declares and libhalf.so exports, with the same argument
count; every C entry point must have a Fortran interface; the named constants
must carry the C enum values.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def _strip_c_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def c_prototypes():
    protos = {}
    for name in ("half.h", "half_b200.h"):
        text = _strip_c_comments(open(os.path.join(INC, name)).read())
        for m in re.finditer(r"\b(?:int|const char\s*\*|half_handle)\s*(half_\w+)\s*\(([^;{]*?)\)\s*;", text):
            args = m.group(2).strip()
            n = 0 if args in ("", "void") else len(args.split(","))
            protos[m.group(1)] = n
    return protos


def c_enum_values():
    vals = {}
    for name in ("half.h", "half_b200.h"):
        text = _strip_c_comments(open(os.path.join(INC, name)).read())
        for m in re.finditer(r"\b(HALF_[A-Z0-9_]+)\s*=\s*([0-9]+)(?:\s*<<\s*([0-9]+))?", text):
            v = int(m.group(2)) << (int(m.group(3)) if m.group(3) else 0)
            vals[m.group(1)] = v
    return vals


def fortran_interfaces():
    text = open(os.path.join(INC, "half_api.f90")).read()
    text = re.sub(r"![^\n]*", "", text)          # comments
    text = re.sub(r"&\s*\n\s*", " ", text)       # continuation lines
    out = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", text):
        fname, args, cname = m.group(1), m.group(2).strip(), m.group(3)
        assert fname == cname, (fname, cname)
        out[cname] = 0 if not args else len(args.split(","))
    return out, text


def test_every_fortran_interface_matches_a_c_prototype():
    protos = c_prototypes()
    ifaces, _ = fortran_interfaces()
    assert set(ifaces) == set(protos), (sorted(set(protos) ^ set(ifaces)))
    for name, n in ifaces.items():
        assert n == protos[name], (name, n, protos[name])


def test_fortran_constants_match_the_c_enums():
    vals = c_enum_values()
    _, text = fortran_interfaces()
    params = {m.group(1): int(m.group(2))
              for m in re.finditer(r"parameter\s*::\s*(HALF_[A-Z0-9_]+)\s*=\s*([0-9]+)", text)}
    assert params, "no named constants found"
    for name, v in params.items():
        assert name in vals, name
        assert vals[name] == v, (name, v, vals[name])
    # every status, selector and capability of half.h is available to Fortran
    for name in vals:
        if name.startswith(("HALF_ERROR", "HALF_SUCCESS", "HALF_SOLVER", "HALF_BACKEND", "HALF_XC", "HALF_CAP",
                            "HALF_PRECISION", "HALF_DENSITY")):
            assert name in params, name


def test_every_fortran_interface_is_exported():
    import halfb200
    try:
        lib = halfb200.load_library()
    except OSError:
        pytest.skip("libhalf.so is not built")
    ifaces, _ = fortran_interfaces()
    for name in ifaces:
        assert hasattr(lib, name), name
