"""The C ABI library builds, loads without a GPU and exports every declared symbol."""

import ctypes as C
import os
import re

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "edzt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(edzt_[a-z_0-9]+)\s*\(", src)))


def test_header_matches_python_mirror(pkg):
    assert sorted(pkg.EXPORTS) == _declared()


def test_library_exports_every_symbol(pkg):
    pkg.build()
    lib = C.CDLL(pkg.LIB_PATH)
    for name in _declared():
        assert hasattr(lib, name), name


def test_version_and_null_context(pkg):
    pkg.build()
    L = pkg.load_library()
    assert L.edzt_version().startswith(b"edzt-b200")
    assert L.edzt_last_error(None) == b"null context"
    assert L.edzt_hx(None, 1, 1, None, None, 0) == pkg.EDZT_ERR_ARG
    assert L.edzt_launch_count(None) == 0


def test_context_creation_fails_cleanly_without_gpu(pkg):
    import torch
    if torch.cuda.is_available():
        return
    pkg.build()
    L = pkg.load_library()
    h = C.c_void_p()
    assert L.edzt_ctx_create(0, C.byref(h)) == pkg.EDZT_ERR_CUDA
    assert not h.value


def test_model_defaults(pkg):
    import numpy as np
    m = pkg.Model(2, 2, np.zeros((2, 2)), np.zeros((2, 2)), np.zeros((2, 2, 2)), U=2.0, Jex=0.5, mu=1.0)
    assert m.Up == 1.0 and m.Jp == 0.5          # src/dmft_params.f90:90-96
    w = pkg.matsubara(3, np.pi)
    assert np.allclose(w, [1.0, 3.0, 5.0])


def test_struct_layouts_match_python_mirror(pkg, tmp_path):
    """The ctypes mirrors of edzt_instance and edzt_dmft_params have the C
    layout: sizes and every field offset, from a C program built against
    include/edzt.h with the host compiler."""
    import subprocess
    structs = {"edzt_instance": pkg.Instance, "edzt_dmft_params": pkg.DMFTParams}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "edzt.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def _c_prototypes():
    """{name: [parameter declarations]} of every function in include/edzt.h."""
    src = open(os.path.join(ROOT, "include", "edzt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(edzt_[a-z_0-9]+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        params = [p.strip() for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        protos[m.group(1)] = params
    return protos


def _fortran_bindings():
    """{C name: (dummy arguments, names passed by value)} from fortran/edzt_iface.f90."""
    src = open(os.path.join(ROOT, "fortran", "edzt_iface.f90")).read()
    src = re.sub(r"!.*", "", src)
    src = re.sub(r"&\s*\n\s*", " ", src)                       # join continuation lines
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+\w+\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)(.*?)end\s+(?:function|subroutine)",
                         src, flags=re.S | re.I):
        args = [a.strip().lower() for a in m.group(1).split(",") if a.strip()]
        byval, cptr = set(), set()
        for decl in re.findall(r"^\s*[^\n]*::[^\n]*$", m.group(3), flags=re.M):
            attrs, names = decl.split("::", 1)
            names = {n.strip().split("(")[0].lower() for n in names.split(",")}
            if "value" in attrs.lower():
                byval |= names
            if "c_ptr" in attrs.lower():
                cptr |= names
        out[m.group(2)] = (args, byval, cptr)
    return out


def test_fortran_interface_matches_header(pkg):
    """Every bind(C) interface of fortran/edzt_iface.f90 names an exported
    entry point and has the C prototype's parameter count; a parameter the C
    prototype takes by value (no pointer) is a Fortran value argument, and a
    pointer parameter is passed by reference or as a type(c_ptr) value."""
    protos = _c_prototypes()
    binds = _fortran_bindings()
    assert len(binds) >= 18
    for name, (args, byval, cptr) in binds.items():
        if name == "strlen":
            continue
        assert name in pkg.EXPORTS, name
        params = protos[name]
        assert len(args) == len(params), (name, args, params)
        for a, p in zip(args, params):
            if "*" in p:
                assert a not in byval or a in cptr, (name, a, p)
            else:
                assert a in byval and a not in cptr, (name, a, p)
