"""The Fortran drop-in (fortran/advection_b200.f90) against the C header.

No Fortran compiler exists on the build machine, so the module is checked
as text: every bind(C) name must be a function the header declares and the
library exports, with the same number of arguments, and the two bind(C)
structs must list the C structs' members in the same order.  The module
must also keep the reference's public interface (advect, adv_init,
adv_var_request; src/physics/advection_driver.f90:21).
"""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
F90 = ROOT / "fortran" / "advection_b200.f90"
HEADER = ROOT / "include" / "icar_adv.h"


def _header():
    txt = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    funcs = {}
    for m in re.finditer(r"\b(?:int|const char \*)\s*(icar_adv_\w+)\s*\(([^)]*)\)\s*;", txt):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        funcs[m.group(1)] = len(args)
    structs = {}
    for m in re.finditer(r"typedef struct \{(.*?)\}\s*(\w+);", txt, flags=re.S):
        body = re.sub(r"//.*", "", m.group(2 - 1))
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            decl = re.sub(r"\[[^\]]*\]", "", decl)
            parts = decl.replace("*", " ").split()
            # "int32_t nx, ny, nz" -> nx ny nz
            for name in " ".join(parts[1:]).split(","):
                names.append(name.strip().split()[-1])
        structs[m.group(2)] = names
    return funcs, structs


def _fortran():
    src = F90.read_text()
    src_nc = re.sub(r"!.*", "", src)
    binds = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*&?\s*bind\(C,\s*name=\"(\w+)\"\)", src_nc,
                         flags=re.S | re.I):
        args = [a for a in m.group(2).split(",") if a.strip()]
        binds[m.group(3)] = len(args)
    types = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", src_nc, flags=re.S | re.I):
        names = []
        for line in m.group(2).splitlines():
            if "::" in line:
                decl = re.sub(r"\([^)]*\)", "", line.split("::", 1)[1])
                names += [n.strip() for n in decl.split(",") if n.strip()]
        types[m.group(1)] = names
    return src_nc, binds, types


def test_every_bound_name_is_declared_and_exported(cuda_lib):
    funcs, _ = _header()
    _, binds, _ = _fortran()
    lib = cuda_lib.load()
    assert len(binds) >= 10
    for name, nargs in binds.items():
        if name == "strlen":
            continue
        assert name in funcs, f"{name} is not declared in include/icar_adv.h"
        assert funcs[name] == nargs, f"{name}: {nargs} arguments bound, {funcs[name]} declared"
        assert hasattr(lib, name), f"{name} is not exported by libicar_adv.so"


def test_bind_c_structs_match_the_header():
    _, structs = _header()
    _, _, types = _fortran()
    for t in ("icar_adv_desc", "icar_adv_opts"):
        assert types[t] == structs[t], (t, types[t], structs[t])


def test_module_keeps_the_reference_interface():
    src, _, _ = _fortran()
    m = re.search(r"module advection\b(.*?)end module advection", src, flags=re.S | re.I)
    assert m, "module advection is missing"
    body = m.group(1)
    assert re.search(r"public\s*::\s*advect\s*,\s*adv_init\s*,\s*adv_var_request", body, flags=re.I)
    for sub, args in (("adv_init", "domain, options"), ("adv_var_request", "options"),
                      ("advect", "domain, options, dt")):
        assert re.search(rf"subroutine\s+{sub}\s*\(\s*{args}\s*\)", body, flags=re.I), sub
    # every library call goes through the status check
    calls = re.findall(r"icar_adv_(?:create|set_field|get_field|advect|var_request|restart_vars|destroy|default_opts)\(", body)
    checked = re.findall(r"call check\(icar_adv_", body)
    assert len(calls) == len(checked)
