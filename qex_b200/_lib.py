"""ctypes binding of ``libqexstag.so`` (the C ABI in ``include/qexstag.h``).

The library is built in-tree by :mod:`qex_b200.build`.  Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libqexstag.so"

OK = 0
NOT_CONVERGED = 1
ERR_ARG = -1
ERR_CUDA = -2
ERR_NAN = -3
ERR_TIMEOUT = -4
ERR_ALLOC = -5
ERR_STATE = -6
ERR_IO = -7
GAUGE_SCIDAC, GAUGE_ILDG, GAUGE_MILC = 1, 2, 3

MEM_HOST = 0
MEM_DEVICE = 1
EVEN, ODD, ALL = 0, 1, 2
SLOPPY_NONE, SLOPPY_SINGLE, SLOPPY_HALF = 0, 1, 2


class SolverParamsC(C.Structure):
    _fields_ = [
        ("r2req", C.c_double),
        ("maxits", C.c_int),
        ("sloppy", C.c_int),
        ("delta", C.c_double),
        ("verbosity", C.c_int),
        ("use_prev_soln", C.c_int),
        ("reserved", C.c_int * 6),
    ]


class SolverStatsC(C.Structure):
    _fields_ = [
        ("calls", C.c_int),
        ("iterations", C.c_int),
        ("outer_iterations", C.c_int),
        ("reliable_updates", C.c_int),
        ("seconds", C.c_double),
        ("flops", C.c_double),
        ("r2", C.c_double),
        ("kernel_launches", C.c_longlong),
    ]


class Fat7CoefsC(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("one_link", "three_staple", "five_staple", "seven_staple", "lepage")]


class HisqCoefsC(C.Structure):
    _fields_ = [
        ("fat7first", Fat7CoefsC),
        ("fat7second", Fat7CoefsC),
        ("naik", C.c_double),
        ("reunit_eps", C.c_double),
    ]


class GaugeCoefsC(C.Structure):
    _fields_ = [("plaq", C.c_double), ("rect", C.c_double)]


class GaugeInfoC(C.Structure):
    _fields_ = [
        ("format", C.c_int),
        ("dims", C.c_int * 4),
        ("precision", C.c_int),
        ("has_checksum", C.c_int),
        ("file_checksum", C.c_uint * 2),
        ("data_checksum", C.c_uint * 2),
        ("date", C.c_char * 64),
        ("file_metadata", C.c_char * 256),
        ("record_metadata", C.c_char * 256),
    ]


P = C.c_void_p
D = C.c_double
I = C.c_int
DP = C.POINTER(C.c_double)
PP = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); every symbol declared in include/qexstag.h
SIGNATURES = {
    "qexstag_init": (I, [I]),
    "qexstag_finalize": (I, []),
    "qexstag_set_stream": (I, [P]),
    "qexstag_last_error": (C.c_char_p, []),
    "qexstag_synchronize": (I, []),
    "qexstag_layout_create": (I, [C.POINTER(C.c_int), C.POINTER(P)]),
    "qexstag_layout_destroy": (I, [P]),
    "qexstag_layout_index": (I, [P, C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
    "qexstag_layout_shift_table": (I, [P, I, I, I, P]),
    "qexstag_links_create": (I, [P, I, P, I, D, C.POINTER(P)]),
    "qexstag_links_destroy": (I, [P]),
    "qexstag_links_recon12": (I, [P]),
    "qexstag_links_update": (I, [P, P, I]),
    "qexstag_links_rephase": (I, [P]),
    "qexstag_links_rephase_all": (I, [P]),
    "qexstag_links_create_milc": (I, [P, P, P, D, C.POINTER(C.c_void_p)]),
    "qexstag_links_update_milc": (I, [P, P, P]),
    "qexstag_links_get_milc": (I, [P, P, P]),
    "qexstag_stagD2": (I, [P, I, P, P, D, D, I]),
    "qexstag_stagD": (I, [P, I, P, P, D, D, D, I]),
    "qexstag_stagDN": (I, [P, I, I, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), D, I]),
    "qexstag_D": (I, [P, P, P, D, I]),
    "qexstag_Ddag": (I, [P, P, P, D, I]),
    "qexstag_stagD2ee": (I, [P, P, P, D, I]),
    "qexstag_stagD2oo": (I, [P, P, P, D, I]),
    "qexstag_stagD2ee_noalloc": (I, [P, P, P, D]),
    "qexstag_solveEE": (I, [P, P, P, D, P, P, I]),
    "qexstag_solveOO": (I, [P, P, P, D, P, P, I]),
    "qexstag_solve": (I, [P, P, P, D, P, P, I]),
    "qexstag_solve_multishift": (I, [P, I, PP, P, DP, P, P, I]),
    "qexstag_cgm_ee": (I, [P, D, I, DP, I, PP, PP, P, P, DP, I]),
    "qexstag_solve_batched": (I, [I, PP, DP, PP, PP, P, C.POINTER(C.c_int), DP, C.POINTER(C.c_int), P, I]),
    "qexstag_force": (I, [P, P, P, D, P, P, I]),
    "qexstag_ferm_force": (I, [P, P, P, I]),
    "qexstag_force_solve": (I, [P, P, P, D, P, P, I]),
    "qexstag_ferm_outer": (I, [P, P, P, I]),
    "qexstag_bench_schur": (I, [P, I, I, D, DP]),
    "qexstag_fat7_coefs_set_hisq": (None, [P, D, D]),
    "qexstag_hisq_coefs_init": (None, [P, D, D]),
    "qexstag_smear_create": (I, [P, C.POINTER(P)]),
    "qexstag_smear_destroy": (I, [P]),
    "qexstag_fat7": (I, [P, P, P, P, P, P, D, I]),
    "qexstag_project_u": (I, [P, P, P, D, I]),
    "qexstag_hisq_smear": (I, [P, P, P, P, P, I]),
    "qexstag_links_hisq": (I, [P, P, P, P, I]),
    "qexstag_fat7_deriv": (I, [P, P, P, P, P, P, P, P, D, I]),
    "qexstag_project_u_deriv": (I, [P, P, P, P, P, D, I]),
    "qexstag_hisq_deriv": (I, [P, P, P, P, P, P, I]),
    "qexstag_hisq_force": (I, [P, P, P, P, P, P, D, P, P, I]),
    "qexstag_gauge_file_info": (I, [C.c_char_p, P]),
    "qexstag_gauge_read": (I, [P, C.c_char_p, P, I, P]),
    "qexstag_gauge_write": (I, [P, C.c_char_p, P, I, I, I, C.c_char_p, C.c_char_p]),
    "qexstag_gauge_coefs_rect": (None, [P, D, D]),
    "qexstag_gauge_action": (I, [P, P, P, I, DP]),
    "qexstag_gauge_force": (I, [P, P, P, P, I]),
    "qexstag_link_update": (I, [P, P, P, D, I]),
    "qexstag_momenta_update": (I, [P, P, P, D, I]),
    "qexstag_momenta_heatbath": (I, [P, P, C.c_ulonglong, C.c_ulonglong, I]),
    "qexstag_kinetic_action": (I, [P, P, I, DP]),
    "qexstag_domain_create": (I, [C.POINTER(C.c_int), I, I, I, C.POINTER(P)]),
    "qexstag_domain_create_zt": (I, [C.POINTER(C.c_int), C.POINTER(C.c_int), I, I, C.POINTER(P)]),
    "qexstag_domain_destroy": (I, [P]),
    "qexstag_domain_local_dims": (I, [P, C.POINTER(C.c_int)]),
    "qexstag_domain_recon12": (I, [P]),
    "qexstag_domain_connect_local": (I, [PP, I]),
    "qexstag_nccl_unique_id": (I, [P]),
    "qexstag_domain_connect_nccl": (I, [P, P]),
    "qexstag_domain_connect_host": (I, [P, P]),
    "qexstag_domain_links": (I, [PP, I, PP, I]),
    "qexstag_domain_stagD2ee": (I, [PP, I, PP, PP, D, I]),
    "qexstag_domain_solveEE": (I, [PP, I, PP, PP, D, P, P, I]),
    "qexstag_barrier_selftest": (I, [I, D]),
}

_lib = None


def load() -> C.CDLL:
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m qex_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class QexStagError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: status {code}: {msg}")
        self.code = code


def check(code: int, where: str, allow_not_converged: bool = True) -> int:
    if code == OK or (allow_not_converged and code == NOT_CONVERGED):
        return code
    msg = load().qexstag_last_error().decode()
    raise QexStagError(code, where, msg)
