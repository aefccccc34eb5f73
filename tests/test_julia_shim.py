"""Static check of the Julia extension's ccalls against include/momed.h (no Julia here).

Every `ccall((:momed_*, libmomed), Ret, (T1, ..., Tn), a1, ..., an)` in
momentumed.jl_b200/julia/MomentumEDB200Ext.jl must name a function the header declares, pass
as many arguments as it declares types, declare as many types as the C prototype has
parameters, and use a Julia type that matches each C parameter type (the binding a maintainer
adds to MomentumED.jl's GPU hooks, gpu_interface.jl:13-21).
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "momed.h")
SHIM = os.path.join(ROOT, "momentumed.jl_b200", "julia", "MomentumEDB200Ext.jl")

# C parameter type -> Julia types that pass it correctly
C_TO_JULIA = {
    "momed_handle*": {"Ptr{Cvoid}"},
    "const momed_handle*": {"Ptr{Cvoid}"},
    "momed_handle**": {"Ref{Ptr{Cvoid}}", "Ptr{Ptr{Cvoid}}"},
    "momed_server*": {"Ptr{Cvoid}"},
    "momed_server**": {"Ref{Ptr{Cvoid}}", "Ptr{Ptr{Cvoid}}"},
    "void*": {"Ptr{Cvoid}", "Ptr{ComplexF64}", "Ptr{ComplexF32}"},
    "const void*": {"Ptr{Cvoid}", "Ptr{ComplexF64}", "Ptr{ComplexF32}"},
    "const momed_para*": {"Ref{MomedPara}", "Ptr{MomedPara}"},
    "const momed_solve_opts*": {"Ref{MomedSolveOpts}", "Ptr{MomedSolveOpts}"},
    "momed_info*": {"Ref{MomedInfo}", "Ptr{MomedInfo}"},
    "const int64_t*": {"Ptr{Int64}", "Ref{Int64}"},
    "int64_t*": {"Ptr{Int64}", "Ref{Int64}"},
    "const uint64_t*": {"Ptr{UInt64}"},
    "uint64_t*": {"Ptr{UInt64}"},
    "const int32_t*": {"Ptr{Int32}"},
    "int32_t*": {"Ptr{Int32}", "Ref{Int32}"},
    "const double*": {"Ptr{Float64}", "Ptr{ComplexF64}", "Ptr{Cvoid}"},
    "double*": {"Ptr{Float64}", "Ptr{ComplexF64}", "Ref{Float64}", "Ptr{Cvoid}"},
    "int": {"Cint", "Int32"},
    "int32_t": {"Int32", "Cint"},
    "int64_t": {"Int64"},
    "double": {"Float64", "Cdouble"},
}
RET_TO_JULIA = {"int": {"Cint", "Int32"}, "const char*": {"Cstring", "Ptr{UInt8}"}, "int64_t": {"Int64"}}


def _norm(t: str) -> str:
    t = re.sub(r"\s+", " ", t.strip())
    t = re.sub(r"\s*\*", "*", t)
    return t


def header_prototypes():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    protos = {}
    for m in re.finditer(r"MOMED_API\s+([\w\s\*]+?)\s*\b(momed_\w+)\s*\(([^)]*)\)\s*;", src):
        ret, name, params = m.group(1), m.group(2), m.group(3)
        plist = []
        if params.strip() != "void":
            for p in params.split(","):
                p = _norm(p)
                # drop the parameter name (last identifier)
                p = re.sub(r"\b\w+$", "", p).strip()
                plist.append(_norm(p))
        protos[name] = (_norm(ret), plist)
    return protos


def _split_top(s: str):
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        out.append("".join(cur).strip())
    return out


def shim_ccalls():
    return ccalls_in(open(SHIM).read())


def ccalls_in(src: str):
    """(name, Julia return type, [Julia argument types], [arguments]) of every ccall in src."""
    src = "\n".join(l.split("#", 1)[0] if not l.lstrip().startswith("#") else "" for l in src.splitlines())
    calls = []
    for m in re.finditer(r"ccall\(", src):
        i, depth = m.end(), 1
        while depth:
            depth += {"(": 1, ")": -1}.get(src[i], 0)
            i += 1
        parts = _split_top(src[m.end():i - 1])
        name = re.match(r"\(:(\w+),", parts[0]).group(1)
        types = _split_top(parts[2].strip()[1:-1])
        calls.append((name, parts[1].strip(), [re.sub(r"\s+", "", t) for t in types], parts[3:]))
    return calls


def test_every_ccall_matches_the_header():
    protos = header_prototypes()
    calls = shim_ccalls()
    assert len(calls) >= 15
    seen = set()
    for name, ret, types, args in calls:
        assert name in protos, f"{name} is not declared in momed.h"
        cret, cparams = protos[name]
        assert ret in RET_TO_JULIA[cret], f"{name}: return {ret} vs C {cret}"
        assert len(types) == len(cparams), f"{name}: {len(types)} Julia types vs {len(cparams)} C parameters"
        assert len(args) == len(types), f"{name}: {len(args)} arguments vs {len(types)} types"
        for k, (jt, ct) in enumerate(zip(types, cparams)):
            assert ct in C_TO_JULIA, f"{name}: unmapped C type {ct}"
            assert jt in C_TO_JULIA[ct], f"{name} argument {k + 1}: Julia {jt} for C {ct}"
        seen.add(name)
    # the hooks the extension implements reach these entry points
    for need in ("momed_create", "momed_destroy", "momed_set_basis", "momed_set_scatter", "momed_matvec",
                 "momed_eigsolve", "momed_set_sparse_csr", "momed_enumerate_basis", "momed_enumeration_copy"):
        assert need in seen, need


def test_no_unrooted_temporary_pointers():
    """pointer(f(x)) of a temporary array is not rooted across a ccall; the shim must not do it."""
    src = open(SHIM).read()
    assert not re.search(r"pointer\(\s*[\w.]+\.\(", src), "pointer() of a broadcast temporary"
    assert not re.search(r"pointer\(\s*(ComplexF64|Vector|Int64|UInt64)\s*[\.(\[]", src)


def test_header_parser_sees_every_exported_symbol():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "momentumed.jl_b200"))
    from momed import _lib
    assert set(header_prototypes()) == set(_lib.SIGNATURES)


def header_structs():
    """{struct name: [(field, C type)]} of the header's typedef'd structs, in declaration order."""
    src = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"typedef\s+struct\s*\{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
        fields = []
        for decl in m.group(1).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            tm = re.match(r"((?:const\s+)?\w+\s*\**)\s*(.*)", decl)
            ctype = _norm(tm.group(1))
            for nm in tm.group(2).split(","):
                nm = nm.strip()
                star = "*" * nm.count("*")
                fields.append((nm.strip("* "), _norm(ctype + star)))
        out[m.group(2)] = fields
    return out


def test_shim_structs_match_the_header():
    """The shim's MomedPara / MomedSolveOpts / MomedInfo: same fields, order and widths as C."""
    c_to_jl = {"int32_t": "Int32", "int64_t": "Int64", "uint64_t": "UInt64", "double": "Float64",
               "const int64_t*": "Ptr{Int64}"}
    src = open(SHIM).read()
    hs = header_structs()
    for cname, jname in (("momed_para", "MomedPara"), ("momed_solve_opts", "MomedSolveOpts"),
                         ("momed_info", "MomedInfo")):
        m = re.search(r"(?:mutable\s+)?struct\s+" + jname + r"\s*\n(.*?)\nend", src, flags=re.S)
        assert m, jname
        jf = [tuple(x.strip() for x in l.split("::")) for l in m.group(1).splitlines() if "::" in l]
        assert [f for f, _ in jf] == [f for f, _ in hs[cname]], jname
        for (f, jt), (_, ct) in zip(jf, hs[cname]):
            assert c_to_jl[ct] == jt, f"{jname}.{f}: {jt} vs C {ct}"
