"""The Fortran side of the boundary (fortran/solar_gpu_bind.f90, fortran/timestep_gpu.f90)
against the C header, without a Fortran compiler (none exists in this image).

* The bind(C) derived type solar_desc lists the C struct's fields in the same order with
  interoperable kinds; the offsets those kinds give under the C layout rules equal the
  offsetof values of a C translation unit compiled against include/solar_gpu.h, and so
  does the ctypes mirror in solar_b200/_lib.py.
* Every bind(C, name=...) interface names a function the header declares, with as many
  dummy arguments as the C prototype has parameters.
* The drop-in RK4 keeps the reference's call surface (no arguments) and its time update
  (timestep.f90:41, 82).
Where gfortran exists, the two files are also compiled.
"""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from solar_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIND = os.path.join(ROOT, "fortran", "solar_gpu_bind.f90")
STEP = os.path.join(ROOT, "fortran", "timestep_gpu.f90")
HEADER = os.path.join(ROOT, "include", "solar_gpu.h")

KIND_SIZE = {"integer(c_int)": 4, "real(c_double)": 8, "type(c_ptr)": 8}


def fortran_desc_fields():
    text = open(BIND).read()
    m = re.search(r"type\s*,\s*bind\(C\)\s*::\s*solar_desc\s*\n(.*?)\n\s*end type", text, re.S | re.I)
    assert m, "solar_desc type not found"
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        kind, names = [x.strip() for x in line.split("::")]
        for name in names.split(","):
            fields.append((kind.lower().replace(" ", ""), name.strip()))
    return fields


def c_struct_fields():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    m = re.search(r"typedef struct solar_desc \{(.*?)\} solar_desc;", text, re.S)
    names = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        parts = decl.replace("*", " ").split()
        rest = " ".join(parts[1:]) if parts[0] != "const" else " ".join(parts[2:])
        names += [n.strip() for n in rest.split(",")]
    return names


def expected_layout(fields):
    off, out = 0, []
    for kind, name in fields:
        size = KIND_SIZE[kind]
        off = (off + size - 1) // size * size
        out.append((name, off, size))
        off += size
    total = (off + 7) // 8 * 8
    return out, total


@pytest.fixture(scope="module")
def c_offsets(tmp_path_factory):
    names = c_struct_fields()
    src = ["#include <stddef.h>", "#include <stdio.h>", '#include "solar_gpu.h"', "int main(void) {"]
    for n in names:
        src.append(f'  printf("{n} %zu %zu\\n", offsetof(solar_desc, {n}), sizeof(((solar_desc*)0)->{n}));')
    src.append('  printf("sizeof %zu\\n", sizeof(solar_desc));')
    src.append("  return 0;\n}")
    d = tmp_path_factory.mktemp("layout")
    c = d / "layout.c"
    c.write_text("\n".join(src))
    exe = d / "layout"
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    subprocess.check_call([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)])
    out = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        parts = line.split()
        out[parts[0]] = tuple(int(x) for x in parts[1:])
    return out


def test_fortran_desc_matches_c_header_layout(c_offsets):
    fields = fortran_desc_fields()
    assert [n for _, n in fields] == c_struct_fields()
    layout, total = expected_layout(fields)
    for name, off, size in layout:
        assert c_offsets[name] == (off, size), (name, c_offsets[name], (off, size))
    assert c_offsets["sizeof"] == (total,)


def test_ctypes_mirror_matches_c_header_layout(c_offsets):
    for name, _ in _lib.SolarDesc._fields_:
        f = getattr(_lib.SolarDesc, name)
        assert (f.offset, f.size) == c_offsets[name], name
    assert ctypes.sizeof(_lib.SolarDesc) == c_offsets["sizeof"][0]


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(?:int|void|long long|void\*)\s+\**(solar_\w+)\s*\(([^)]*)\)\s*;", text):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    return protos


def test_every_fortran_interface_names_a_header_function():
    text = open(BIND).read()
    protos = c_prototypes()
    found = 0
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", text, re.I):
        fname, args, cname = m.group(1), m.group(2), m.group(3)
        assert fname == cname, (fname, cname)
        assert cname in protos, cname
        nargs = len([a for a in args.split(",") if a.strip()])
        assert nargs == protos[cname], (cname, nargs, protos[cname])
        found += 1
    assert found >= 15


def test_drop_in_rk4_keeps_the_reference_call_surface():
    text = open(STEP).read()
    assert re.search(r"^SUBROUTINE RK4\s*$", text, re.M)          # timestep.f90:41, no arguments
    body = re.search(r"^SUBROUTINE RK4\s*$(.*?)^END SUBROUTINE RK4", text, re.M | re.S).group(1)
    assert "USE INIT" in body and "solar_gpu_rk4(solar_ctx, 1_c_int)" in body
    assert "time = time + deltat" in body                         # timestep.f90:82


@pytest.mark.skipif(not shutil.which("gfortran"), reason="no Fortran compiler in this image")
def test_fortran_sources_compile(tmp_path):
    subprocess.check_call(["gfortran", "-c", BIND, "-J", str(tmp_path), "-o", str(tmp_path / "bind.o")])
