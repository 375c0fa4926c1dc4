"""The Julia binding (etherparallelparticles.jl_b200/julia/EPPBackend.jl) against include/epp.h.

Julia is not installed here, so the binding is checked as text: every C struct it mirrors has the
header's fields in the header's order with matching types (and so the same size and offsets
under C layout rules), every `ccall` names an exported entry point with the header's parameter
count and types, and the named action / criterion ids and the ABI version are the header's."""
import ctypes as C
import os
import re

import pytest

from epp import abi
from epp import lib as epplib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "etherparallelparticles.jl_b200", "julia", "EPPBackend.jl")
HEADER = os.path.join(ROOT, "include", "epp.h")

SCALARS = {C.c_int32: "Int32", C.c_float: "Float32", C.c_double: "Float64", C.c_int64: "Int64"}
STRUCTS = {"EppDomain": abi.epp_domain, "EppPhysics": abi.epp_physics, "EppConfig": abi.epp_config,
           "EppColumnMap": abi.epp_column_map, "EppIntegrals": abi.epp_integrals}


def jl_text():
    with open(JL) as f:
        return f.read()


def jl_structs():
    out = {}
    for name, body in re.findall(r"^struct (Epp\w+)\n(.*?)^end", jl_text(), re.M | re.S):
        out[name] = [tuple(x.strip() for x in line.split("::")) for line in body.strip().splitlines()]
    return out


def jl_type_of(ctype):
    if ctype in SCALARS:
        return SCALARS[ctype]
    if issubclass(ctype, C.Array):
        return "NTuple{%d, %s}" % (ctype._length_, jl_type_of(ctype._type_))
    for jn, ct in STRUCTS.items():
        if ct is ctype:
            return jn
    raise KeyError(ctype)


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_struct_fields_match_the_header(name):
    """Field names, order and types of each Julia struct equal the ctypes mirror, which
    tests/test_abi.py checks against the compiled header (sizes and offsets)."""
    fields = jl_structs()[name]
    want = [(f, jl_type_of(t)) for f, t in STRUCTS[name]._fields_]
    assert fields == want


def jl_sizeof(t, structs):
    """(size, alignment) of a Julia isbits type under C layout rules."""
    base = {"Int32": 4, "Float32": 4, "Float64": 8, "Int64": 8}
    if t in base:
        return base[t], base[t]
    m = re.fullmatch(r"NTuple\{(\d+), (\w+)\}", t)
    if m:
        s, a = jl_sizeof(m.group(2), structs)
        return int(m.group(1)) * s, a
    off, al = 0, 1
    for _, ft in structs[t]:
        s, a = jl_sizeof(ft, structs)
        off = (off + a - 1) // a * a + s
        al = max(al, a)
    return (off + al - 1) // al * al, al


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_struct_sizes_match_the_header(name):
    assert jl_sizeof(name, jl_structs())[0] == C.sizeof(STRUCTS[name])


def header_prototypes():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for ret, name, args in re.findall(r"^\s*(int32_t|const char\*|void)\s+(epp_\w+)\s*\(([^)]*)\)\s*;", text, re.M):
        params = [a.strip() for a in args.replace("\n", " ").split(",") if a.strip() and a.strip() != "void"]
        out[name] = (ret, [re.sub(r"\s+\w+$", "", p).strip() for p in params])
    return out


def c_to_jl(ctype):
    """The Julia argument types a C parameter type may be passed as."""
    ct = ctype.replace("const ", "").replace(" ", "")
    table = {"int32_t": {"Int32"}, "int64_t": {"Int64"}, "float": {"Float32"}, "double": {"Float64"},
             "epp_ctx*": {"Ptr{Cvoid}"}, "void*": {"Ptr{Cvoid}"}, "epp_ctx**": {"Ref{Ptr{Cvoid}}"},
             "int32_t*": {"Ptr{Int32}", "Ref{Int32}"}, "uint32_t*": {"Ptr{UInt32}", "Ref{UInt32}"},
             "int64_t*": {"Ptr{Int64}", "Ref{Int64}"}, "float*": {"Ptr{Float32}", "Ref{Float32}"},
             "double*": {"Ptr{Float64}", "Ref{Float64}"}}
    if ct in table:
        return table[ct]
    m = re.fullmatch(r"epp_(\w+)\*", ct)
    if m:
        jn = "Epp" + "".join(w.capitalize() for w in m.group(1).split("_"))
        return {"Ref{%s}" % jn, "Ptr{%s}" % jn}
    raise KeyError(ctype)


def jl_ccalls():
    out = {}
    for name, ret, types in re.findall(r"ccall\(\(:(epp_\w+), libepp\),\s*(\w+),\s*\(([^)]*(?:\)[^)]*)*?)\)\s*,?",
                                       jl_text()):
        parts = [t.strip() for t in re.split(r",(?![^{]*\})", types) if t.strip()]
        out[name] = (ret, parts)
    return out


def test_ccalls_match_the_header_prototypes():
    protos = header_prototypes()
    calls = jl_ccalls()
    assert len(calls) >= 12
    exported = set(epplib.EXPORTS)
    for name, (ret, types) in calls.items():
        assert name in protos and name in exported, name
        cret, cparams = protos[name]
        assert ret == ("Cstring" if cret == "const char*" else "Int32"), name
        assert len(types) == len(cparams), (name, types, cparams)
        for jt, ct in zip(types, cparams):
            assert jt in c_to_jl(ct), (name, jt, ct)


def test_named_ids_and_abi_version_match_the_header():
    text = jl_text()
    consts = dict((k, int(v)) for k, v in re.findall(r"^const (\w+) = Int32\((-?\d+)\)", text, re.M))
    pairs = {"ABI_VERSION": "EPP_ABI_VERSION", "CriterionDefault": "EPP_CRITERION_DEFAULT",
             "CriterionSymmetry": "EPP_CRITERION_SYMMETRY", "ActionNone": "EPP_ACTION_NONE",
             "DamBreakContinuity": "EPP_ACTION_DAMBREAK_CONTINUITY",
             "DamBreakDensity": "EPP_ACTION_DAMBREAK_DENSITY", "DamBreakMomentum": "EPP_ACTION_DAMBREAK_MOMENTUM",
             "DamBreakIntegrate": "EPP_ACTION_DAMBREAK_INTEGRATE", "ZeroDVelocity": "EPP_ACTION_ZERO_DVELOCITY",
             "CountNeighbours": "EPP_ACTION_COUNT_NEIGHBOURS", "KernelFilter": "EPP_ACTION_KERNEL_FILTER",
             "KernelFilterSelf": "EPP_ACTION_KERNEL_FILTER_SELF",
             "ExtrapolatePressure": "EPP_ACTION_EXTRAPOLATE_PRESSURE",
             "ExtrapolatePressureSelf": "EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF",
             "SearchEmitList": "EPP_SEARCH_EMIT_LIST"}
    header = dict(re.findall(r"^#define (EPP_\w+)\s+(-?\d+)", open(HEADER).read(), re.M))
    for jn, cn in pairs.items():
        assert consts[jn] == int(header[cn]), (jn, cn)


def test_reference_api_methods_are_defined():
    """The binding adds methods of the reference's own functions for the B200 backend, so a driver
    keeps calling Algorithm.search!/interaction!/selfaction! and Class.asyncto!/syncto!."""
    text = jl_text()
    for f in ("Algorithm.search!", "Algorithm.static_search!", "Algorithm.dynamic_search!",
              "Algorithm.interaction!", "Algorithm.selfaction!", "Class.syncto!", "Class.asyncto!",
              "Class.host_initializeNeighbourSystem!"):
        assert re.search(r"^(function )?%s\(" % re.escape(f), text, re.M), f
