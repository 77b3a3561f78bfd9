"""ctypes binding of ``libsharpclaw_b200.so`` (the C ABI in include/sharpclaw_cuda.h).

The library is built in-tree (``python -m sharpclaw_b200.build``); loading
fails loudly when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsharpclaw_b200.so")

SCL_OK, SCL_E_INVALID, SCL_E_CUDA, SCL_E_UNSUPPORTED, SCL_E_NONFINITE, SCL_E_TIMEOUT, SCL_E_IO = \
    0, -1, -2, -3, -4, -5, -6
RP_ADVECTION, RP_EULER, RP_SW2D, RP_ACOUSTICS1D, RP_ACOUSTICS2D, RP_ADVECTION2D, RP_SW1D = 1, 2, 3, 4, 5, 6, 7
SRC_NONE, SRC_RADIAL_SW, SRC_BATHYMETRY_SW = 0, 1, 2
RP_SWF_BATHY, RP_SWF_RADIAL, RP_SWF_KAPPA = 8, 9, 10
RP_ACOUSTICS_CONST, RP_ACOUSTICS_FWAVE = 11, 12
RP_TRAFFIC, RP_ADVECTION_CONS, RP_STEGOTON = 13, 14, 15
B4STEP_NONE, B4STEP_SWIRL, B4STEP_TIME_REVERSAL = 0, 1, 2
BC_USER_NONE, BC_USER_OSCILLATING_WALL = 0, 1
RUN_AUTO, RUN_GRAPH, RUN_RESIDENT = 0, 1, 2
FP64, FP64_STRICT, MIXED, FP32 = 0, 1, 2, 3
INFO_DT_NOT_DIVIDING, INFO_CFL_DESIRED_GT_MAX, INFO_TOO_MANY_STEPS, INFO_CFL_FIXED_DT, INFO_NONFINITE = 2, 3, 11, 12, 20
STATUS_NONFINITE, STATUS_TIMEOUT, STATUS_BOUNDS = 1, 2, 4

PRECISIONS = {"fp64": FP64, "fp64_strict": FP64_STRICT, "mixed": MIXED, "fp32": FP32}


class scl_params(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("mx", ctypes.c_int), ("my", ctypes.c_int),
        ("meqn", ctypes.c_int), ("mwaves", ctypes.c_int), ("mbc", ctypes.c_int),
        ("maux", ctypes.c_int), ("mcapa", ctypes.c_int),
        ("lim_type", ctypes.c_int), ("char_decomp", ctypes.c_int), ("tfluct_solver", ctypes.c_int),
        ("mthbc", ctypes.c_int * 4),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("xlower", ctypes.c_double), ("ylower", ctypes.c_double),
        ("rp", ctypes.c_int), ("efix", ctypes.c_int),
        ("u", ctypes.c_double), ("gamma", ctypes.c_double), ("grav", ctypes.c_double),
        ("time_integrator", ctypes.c_int), ("precision", ctypes.c_int),
        ("mthlim", ctypes.c_int * 4),
        ("src_term", ctypes.c_int),
        ("rho", ctypes.c_double), ("bulk", ctypes.c_double),
        ("bc_user", ctypes.c_int), ("wall", ctypes.c_double * 6),
    ]


class scl_run(ctypes.Structure):
    _fields_ = [
        ("tstart", ctypes.c_double), ("tend", ctypes.c_double),
        ("dt_initial", ctypes.c_double), ("dt_max", ctypes.c_double),
        ("cfl_max", ctypes.c_double), ("cfl_desired", ctypes.c_double),
        ("max_steps", ctypes.c_int), ("dt_variable", ctypes.c_int),
    ]


class scl_result(ctypes.Structure):
    _fields_ = [
        ("tend", ctypes.c_double), ("cfl_maxused", ctypes.c_double), ("cfl_last", ctypes.c_double),
        ("dt_minused", ctypes.c_double), ("dt_maxused", ctypes.c_double), ("dt_last", ctypes.c_double),
        ("steps_taken", ctypes.c_int), ("info", ctypes.c_int), ("rejected", ctypes.c_int),
        ("status", ctypes.c_int),
    ]


# (name, restype, argtypes) of every entry point declared in include/sharpclaw_cuda.h
_dp = ctypes.POINTER(ctypes.c_double)
_h = ctypes.c_void_p
SIGNATURES = [
    ("scl_version", ctypes.c_char_p, []),
    ("scl_last_error", ctypes.c_char_p, []),
    ("scl_create", ctypes.c_int, [ctypes.POINTER(scl_params), ctypes.POINTER(ctypes.c_void_p)]),
    ("scl_destroy", ctypes.c_int, [_h]),
    ("scl_set_q", ctypes.c_int, [_h, _dp]),
    ("scl_get_q", ctypes.c_int, [_h, _dp]),
    ("scl_set_aux", ctypes.c_int, [_h, _dp]),
    ("scl_step_dq", ctypes.c_int, [_h, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp]),
    ("scl_flux1", ctypes.c_int, [_h, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp]),
    ("scl_rk_step", ctypes.c_int, [_h, ctypes.c_double, ctypes.c_double, _dp]),
    ("scl_sharpclaw", ctypes.c_int, [_h, ctypes.POINTER(scl_run), ctypes.POINTER(scl_result)]),
    ("scl_sharpclaw_device", ctypes.c_int, [_h, ctypes.POINTER(scl_run), _dp, ctypes.POINTER(scl_result)]),
    ("scl_time_steps", ctypes.c_int, [_h, ctypes.POINTER(scl_run), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_float), ctypes.POINTER(scl_result)]),
    ("scl_time_stages", ctypes.c_int, [_h, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(ctypes.c_longlong)]),
    ("scl_kernels_per_step", ctypes.c_int, [_h]),
    ("scl_set_run_mode", ctypes.c_int, [_h, ctypes.c_int]),
    ("scl_last_run", ctypes.c_int, [_h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]),
    ("scl_select_tiles", ctypes.c_int, [_h, ctypes.c_int]),
    ("scl_set_b4step", ctypes.c_int, [_h, ctypes.c_int, ctypes.c_double]),
    ("scl_write_frame", ctypes.c_int, [_h, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    ("scl_wait_frames", ctypes.c_int, [_h]),
    ("scl_format_frame", ctypes.c_int, [ctypes.POINTER(scl_params), _dp, _dp, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_char_p, ctypes.c_int]),
    ("scl_tiles", ctypes.c_int, [_h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_float)]),
    ("scl_rk_step_noalloc", ctypes.c_int, [ctypes.POINTER(scl_params), ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_double, _dp, ctypes.c_void_p]),
    ("scl_batch_create", ctypes.c_int, [ctypes.POINTER(scl_params), ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("scl_batch_destroy", ctypes.c_int, [_h]),
    ("scl_batch_set_q", ctypes.c_int, [_h, _dp]),
    ("scl_batch_get_q", ctypes.c_int, [_h, _dp]),
    ("scl_batch_set_aux", ctypes.c_int, [_h, _dp]),
    ("scl_batch_run", ctypes.c_int, [_h, ctypes.POINTER(scl_run), ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_float)]),
    ("scl_batch_launches", ctypes.c_longlong, [_h]),
    ("scl_batch_select", ctypes.c_int, [_h, ctypes.c_int]),
    ("scl_batch_tuning", ctypes.c_int, [_h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]),
    ("scl_adjoint_step", ctypes.c_int, [_h, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_double]),
    ("scl_stream", ctypes.c_void_p, [_h]),
    ("scl_set_totals", ctypes.c_int, [_h, ctypes.c_int]),
    ("scl_conserved_totals", ctypes.c_int, [_h, _dp, _dp, _dp]),
    ("scl_test_wait_timeout", ctypes.c_int, [_h, ctypes.c_int]),
]

_lib = None


def lib() -> ctypes.CDLL:
    """Load the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m sharpclaw_b200.build` "
                "(the CUDA path has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class SharpClawError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().scl_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != SCL_OK:
        raise SharpClawError(code, where)
