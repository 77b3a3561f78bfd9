"""The Fortran side (fortran/sharpclaw_cuda.f90) against the C ABI, without a
Fortran compiler (none is installed here): the bind(C) derived types must
have the C structs' fields in the same order with the same types, hence the
same offsets and sizes (checked against offsetof/sizeof of the header
compiled with gcc, and against the ctypes mirror); every bind(C) interface
must name an exported function with the same number of arguments and the
same pointer depth per argument (a dummy without `value` is passed by
reference; type(c_ptr) is itself a pointer); and the drop-in
subroutines must keep the reference's argument lists:

  flux1(q1d,g,dq1d,aux,dt,cfl,t,rp,tfluct,ixy)     src/flux1.f90:2
  flux2(q,g,dq,aux,dt,cfl,t,rp,tfluct)             src/2d/flux2.f90:2
  step(q,g,dq,aux,dt,cfl,t,rp,src,tfluct)          src/1d/step1d.f90:2, src/2d/step2d.f90:2
  sharpclaw(tstart,tend,cfl_maxused,...,b4step)    src/sharpclaw.f90:2-5
"""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from sharpclaw_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "fortran", "sharpclaw_cuda.f90")
HDR = os.path.join(ROOT, "include", "sharpclaw_cuda.h")

SIZES = {"integer(c_int)": 4, "real(c_double)": 8}

REFERENCE_SIGNATURES = {
    "flux1": "q1d,g,dq1d,aux,dt,cfl,t,rp,tfluct,ixy",
    "flux2": "q,g,dq,aux,dt,cfl,t,rp,tfluct",
    "step": "q,g,dq,aux,dt,cfl,t,rp,src,tfluct",
    "sharpclaw": "tstart,tend,cfl_maxused,cfl_last,dt_minused,dt_maxused,dt_last,steps_taken,info,dt_initial,"
                 "dt_max,dt_variable,time_integrator,verbosity,cfl_max,cfl_desired,max_steps,r1,r2,bc,rp,tfluct,"
                 "src,b4step",
}


def _source():
    text = open(F90).read()
    text = re.sub(r"!.*", "", text)                 # comments
    return re.sub(r"&\s*\n\s*", " ", text)          # continuation lines


def fortran_types():
    """{type name: [(field, bytes, count), ...]} of the bind(C) types."""
    out = {}
    for m in re.finditer(r"type\s*,\s*bind\(C\)\s*::\s*(\w+)(.*?)end\s+type", _source(), flags=re.S | re.I):
        fields = []
        for line in m.group(2).splitlines():
            d = re.match(r"\s*(integer\(c_int\)|real\(c_double\))\s*::\s*(.+)", line)
            if not d:
                continue
            for item in d.group(2).split(","):
                item = item.strip()
                a = re.match(r"(\w+)(?:\((\d+)\))?$", item)
                fields.append((a.group(1), SIZES[d.group(1)], int(a.group(2) or 1)))
        out[m.group(1)] = fields
    return out


def c_layout(fields):
    """Offsets of C natural alignment, and the struct size."""
    off, offs, align = 0, [], 1
    for _, size, n in fields:
        off = (off + size - 1) // size * size
        offs.append(off)
        off += size * n
        align = max(align, size)
    return offs, (off + align - 1) // align * align


def test_bind_c_types_match_the_header_layout(tmp_path):
    types = fortran_types()
    assert set(types) == {"scl_params", "scl_run", "scl_result"}
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "sharpclaw_cuda.h"', "int main(void) {"]
    for t, fields in types.items():
        lines.append(f'  printf("{t} size %zu\\n", sizeof({t}));')
        for name, _, _ in fields:
            lines.append(f'  printf("{t} {name} %zu %zu\\n", offsetof({t}, {name}), sizeof((({t}*)0)->{name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        parts = line.split()
        got[(parts[0], parts[1])] = tuple(int(x) for x in parts[2:])
    for t, fields in types.items():
        offs, size = c_layout(fields)
        assert got[(t, "size")] == (size,), t
        ct = getattr(C, t)
        assert ctypes.sizeof(ct) == size, t
        assert [f[0] for f in ct._fields_] == [f[0] for f in fields], t
        for (name, fsize, n), off in zip(fields, offs):
            assert got[(t, name)] == (off, fsize * n), (t, name)
            assert getattr(ct, name).offset == off, (t, name)


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(scl_\w+)\s*\(([^)]*)\)\s*;", text, flags=re.M):
        args = [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        protos[m.group(1)] = args
    return protos


def test_bind_c_interfaces_match_the_header():
    src = _source()
    protos = c_prototypes()
    found = 0
    for m in re.finditer(r"function\s+(scl_\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)(.*?)end\s+function",
                         src, flags=re.S | re.I):
        fname, fargs, cname, body = m.group(1), m.group(2), m.group(3), m.group(4)
        assert fname == cname
        assert cname in protos, f"{cname} is not declared in the header"
        assert hasattr(C.lib(), cname)
        fargs = [a.strip() for a in fargs.split(",") if a.strip()]
        cargs = protos[cname]
        assert len(fargs) == len(cargs), cname
        for fa, ca in zip(fargs, cargs):
            decl = re.search(r"^\s*(.+?)::[^\n]*\b" + fa + r"\b", body, flags=re.M)
            assert decl, (cname, fa)
            # pointer depth: a c_ptr is a pointer itself; a dummy without
            # `value` is passed by reference
            attrs = decl.group(1).lower()
            depth = (1 if "c_ptr" in attrs else 0) + (0 if "value" in attrs else 1)
            assert depth == ca.count("*"), (cname, fa, ca)
        found += 1
    assert found >= 12


def test_drop_in_routines_keep_the_reference_signatures():
    src = _source()
    for name, args in REFERENCE_SIGNATURES.items():
        m = re.search(r"^\s*subroutine\s+" + name + r"\s*\(([^)]*)\)", src, flags=re.M | re.I)
        assert m, name
        got = ",".join(a.strip() for a in m.group(1).split(","))
        assert got == args, name
