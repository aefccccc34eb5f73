"""The Python mirror's ctypes table (momed._lib.SIGNATURES) against include/momed.h: every
prototype has an entry with its arity, its return type and, per parameter, a ctypes type that
passes the C type (scalars by width, pointers as c_void_p or a pointer to the matching type)."""
import ctypes as C
import os
import sys

from test_julia_shim import ROOT, header_prototypes

sys.path.insert(0, os.path.join(ROOT, "momentumed.jl_b200"))
from momed import _lib  # noqa: E402

SCALAR = {"int": {C.c_int, C.c_int32}, "int32_t": {C.c_int32, C.c_int}, "int64_t": {C.c_int64},
          "double": {C.c_double}}
POINTEE = {"int64_t*": C.c_int64, "const int64_t*": C.c_int64, "int32_t*": C.c_int32,
           "const int32_t*": C.c_int32, "double*": C.c_double, "const double*": C.c_double,
           "uint64_t*": C.c_uint64, "const uint64_t*": C.c_uint64, "momed_handle**": C.c_void_p,
           "momed_server**": C.c_void_p, "const momed_para*": _lib.Para,
           "const momed_solve_opts*": _lib.SolveOpts, "momed_info*": _lib.Info}
RET = {"int": C.c_int, "const char*": C.c_char_p, "int64_t": C.c_int64}


def passes(ctype, cparam: str) -> bool:
    if cparam in SCALAR:
        return ctype in SCALAR[cparam]
    assert cparam.endswith("*"), cparam
    if ctype is C.c_void_p:
        return True
    want = POINTEE.get(cparam)
    return want is not None and ctype is C.POINTER(want)


def test_every_prototype_has_a_matching_ctypes_entry():
    protos = header_prototypes()
    assert set(protos) == set(_lib.SIGNATURES)
    for name, (cret, cparams) in protos.items():
        res, args = _lib.SIGNATURES[name]
        assert res is RET[cret], f"{name}: return {res} vs C {cret}"
        assert len(args) == len(cparams), f"{name}: {len(args)} ctypes vs {len(cparams)} C parameters"
        for k, (ct, cp) in enumerate(zip(args, cparams)):
            assert passes(ct, cp), f"{name} argument {k + 1}: {ct} for C {cp}"


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof and every field offset of momed_para / momed_solve_opts / momed_info as gcc lays
    them out from the header, against the ctypes structures the mirror passes."""
    import shutil
    import subprocess
    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    structs = {"momed_para": _lib.Para, "momed_solve_opts": _lib.SolveOpts, "momed_info": _lib.Info}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "momed.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, f"{cname}.{f}"
