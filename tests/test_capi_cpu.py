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
    (dict(mthbc=(0, 0)), C.SCL_E_INVALID),
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
