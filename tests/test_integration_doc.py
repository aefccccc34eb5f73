"""The typed ccall of every entry point listed in INTEGRATION.md's appendix against
include/momed.h (no Julia here): each header prototype appears exactly once, with as many
Julia types as C parameters, as many arguments as types, and a Julia type that passes each C
parameter type (the same table as the extension's own check)."""
import os
import re

from test_julia_shim import C_TO_JULIA, RET_TO_JULIA, ROOT, ccalls_in, header_prototypes

DOC = os.path.join(ROOT, "INTEGRATION.md")


def appendix_block() -> str:
    text = open(DOC).read()
    i = text.index("## Appendix: every entry point")
    m = re.search(r"```julia\n(.*?)```", text[i:], flags=re.S)
    assert m, "no julia block in the appendix"
    return m.group(1)


def test_appendix_binds_every_prototype_once():
    protos = header_prototypes()
    calls = ccalls_in(appendix_block())
    names = [c[0] for c in calls]
    assert sorted(names) == sorted(protos), (set(protos) - set(names), set(names) - set(protos))
    assert len(names) == len(set(names))
    for name, ret, types, args in calls:
        cret, cparams = protos[name]
        assert ret in RET_TO_JULIA[cret], f"{name}: return {ret} vs C {cret}"
        assert len(types) == len(cparams), f"{name}: {len(types)} Julia types vs {len(cparams)} C parameters"
        assert len(args) == len(types), f"{name}: {len(args)} arguments vs {len(types)} types"
        for k, (jt, ct) in enumerate(zip(types, cparams)):
            assert ct in C_TO_JULIA, f"{name}: unmapped C type {ct}"
            assert jt in C_TO_JULIA[ct], f"{name} argument {k + 1}: Julia {jt} for C {ct}"


def test_appendix_follows_header_order():
    order = list(header_prototypes())
    names = [c[0] for c in ccalls_in(appendix_block())]
    assert names == order
