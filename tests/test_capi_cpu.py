"""C ABI checks that need no GPU: the library loads, exports every function
declared in include/*.h, and rejects invalid parameters before touching CUDA."""
import ctypes
import os
import re

import pytest

import sharpclaw_b200 as S
from sharpclaw_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(scl_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = C.lib()
    decl = declared_functions()
    assert len(decl) >= 14
    for name in decl:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(decl) == {n for n, _, _ in C.SIGNATURES}


def test_version_string():
    assert b"sm_100a" in C.lib().scl_version()


@pytest.mark.parametrize("change,code", [
    (dict(mbc=2), C.SCL_E_INVALID),
    (dict(mx=2), C.SCL_E_INVALID),
    (dict(lim_type=0), C.SCL_E_UNSUPPORTED),                                   # char_decomp 2
    (dict(lim_type=0, char_decomp=0, mthlim=(7, 1, 1, 1)), C.SCL_E_UNSUPPORTED),  # needs mbc = 4
    (dict(lim_type=0, char_decomp=0, mthlim=(5, 1, 1, 1)), C.SCL_E_INVALID),      # polyrecon.f90 stops
    (dict(lim_type=3), C.SCL_E_INVALID),
    (dict(src_term=1), C.SCL_E_UNSUPPORTED),                                    # SW1D hooks only
    (dict(src_term=5), C.SCL_E_INVALID),
    (dict(rp=S.RP_SW1D, meqn=None, mwaves=None, char_decomp=0, src_term=2), C.SCL_E_INVALID),  # maux 0
    (dict(rp=S.RP_ACOUSTICS_CONST, meqn=None, mwaves=None, char_decomp=0, rho=0.0), C.SCL_E_INVALID),
    (dict(lim_type=1, char_decomp=3), C.SCL_E_UNSUPPORTED),
    (dict(lim_type=1, mthlim=(1, 6, 1, 1)), C.SCL_E_INVALID),
    (dict(char_decomp=4), C.SCL_E_UNSUPPORTED),
    (dict(mthbc=(0, 0)), C.SCL_E_INVALID),                                      # user bc without bc_user
    (dict(bc_user=2), C.SCL_E_INVALID),
    (dict(bc_user=1, mthbc=(0, 1)), C.SCL_E_UNSUPPORTED),                        # the wall needs aux rho
    (dict(rp=S.RP_SW2D, meqn=None, mwaves=None, my=8, dy=0.1, mthbc=(0, 1, 1, 1), bc_user=1), C.SCL_E_UNSUPPORTED),
    (dict(mthbc=(2, 1)), C.SCL_E_INVALID),
    (dict(time_integrator=5), C.SCL_E_INVALID),
    (dict(tfluct_solver=1), C.SCL_E_INVALID),   # Euler has no tfluct plugin
    (dict(meqn=2), C.SCL_E_INVALID),
    (dict(rp=S.RP_ADVECTION, meqn=None, mwaves=None, char_decomp=0, tfluct_solver=1, mthbc=(3, 3)),
     C.SCL_E_INVALID),
])
def test_invalid_params_rejected_without_gpu(change, code):
    base = dict(rp=S.RP_EULER, mx=100, dx=0.01, mthbc=(1, 1), char_decomp=2, tfluct_solver=0)
    base.update(change)
    p = S.ClawParams(**base)
    cp = p.to_c(C.FP64)
    h = ctypes.c_void_p()
    rc = C.lib().scl_create(ctypes.byref(cp), ctypes.byref(h))
    assert rc == code
    assert not h.value
    assert len(C.lib().scl_last_error()) > 0


def test_params_shapes():
    p = S.ClawParams(rp=S.RP_SW2D, mx=10, my=7, dx=0.1, dy=0.1)
    assert p.shape() == (3, 13, 16)
    assert p.meqn == 3 and p.mwaves == 3 and p.ndim == 2 and p.efix == 0
    p = S.ClawParams(rp=S.RP_EULER, mx=10, dx=0.1)
    assert p.shape() == (3, 16) and p.efix == 1


def test_header_is_plain_c_and_links(tmp_path):
    """include/sharpclaw_cuda.h is the boundary a C, C++ or Fortran caller
    binds: it compiles as C99, every declared function links against the
    library, and a C program calls it (scl_version, scl_create rejecting bad
    parameters, scl_format_frame writing a frame: no GPU involved)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = declared_functions()
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "sharpclaw_cuda.h"\n'
        "int main(void) {\n"
        "  void* fns[] = {" + ", ".join("(void*)&" + n for n in names) + "};\n"
        '  printf("%s %d\\n", scl_version(), (int)(sizeof(fns) / sizeof(fns[0])));\n'
        "  scl_params p; memset(&p, 0, sizeof(p));\n"
        "  scl_handle* h = 0;\n"
        "  int rc = scl_create(&p, &h);\n"
        '  printf("%d %s\\n", rc, scl_last_error());\n'
        "  p.ndim = 1; p.mx = 4; p.meqn = 1; p.mwaves = 1; p.mbc = 3; p.dx = 0.25; p.rp = SCL_RP_ADVECTION;\n"
        "  p.lim_type = 2; p.tfluct_solver = 1; p.mthbc[0] = p.mthbc[1] = 2; p.time_integrator = 3;\n"
        "  double q[10] = {0, 0, 0, 1, 2, 3, 4, 0, 0, 0};\n"
        '  int rf = scl_format_frame(&p, q, 0, 0.5, 7, "' + str(tmp_path) + '", 0);\n'
        '  printf("%d\\n", rf);\n'
        "  return (rc == SCL_E_INVALID && h == 0 && rf == SCL_OK) ? 0 : 1;\n}\n")
    libdir = os.path.dirname(C.LIB_PATH)
    exe = tmp_path / "caller"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-o", str(exe), "-L", libdir, "-lsharpclaw_b200", "-Wl,-rpath," + libdir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    first = r.stdout.splitlines()[0]
    assert "sm_100a" in first and first.endswith(" %d" % len(names))
    frame = (tmp_path / "fort.q0007").read_text()
    assert "0.10000000E+01" in frame and "0.40000000E+01" in frame


def test_noalloc_refuses_a_host_array():
    """scl_rk_step_noalloc takes caller-owned device memory; given a host
    (numpy) array it launches nothing and returns an error status instead of
    letting a kernel dereference host memory.  Without a GPU the call stops at
    'no usable CUDA device'; the GPU test checks SCL_E_INVALID there."""
    import numpy as np
    import torch
    p = S.ClawParams(rp=S.RP_EULER, mx=64, dx=0.1, mthbc=(1, 1), char_decomp=2, tfluct_solver=0,
                     time_integrator=3)
    cp = p.to_c(C.FP64)
    q = np.ones((3, 70))
    cfl = ctypes.c_double(0.0)
    rc = C.lib().scl_rk_step_noalloc(ctypes.byref(cp), ctypes.c_void_p(q.ctypes.data), None, 1e-3,
                                     ctypes.byref(cfl), None)
    assert rc in (C.SCL_E_CUDA, C.SCL_E_INVALID)
    msg = C.lib().scl_last_error()
    if not torch.cuda.is_available():
        assert b"no usable CUDA device" in msg
    else:
        assert rc == C.SCL_E_INVALID and b"q_dev" in msg
    assert np.all(q == 1.0)
