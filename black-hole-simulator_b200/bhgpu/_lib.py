"""ctypes binding of libbhgpu.so (the C ABI declared in include/bhgpu.h).

There is no fallback: if the CUDA library is missing or cannot be loaded,
importing bhgpu raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbhgpu.so")

BH_OK, BH_EINVAL, BH_ECUDA, BH_ERANGE = 0, -1, -2, -3
BH_ERR_DOMAIN = 1
BH_MINMOD, BH_VANLEER, BH_MC, BH_PPM = 0, 1, 2, 3
BH_FP64, BH_FP64_FMA, BH_MIXED = 0, 1, 2
_vp = C.c_void_p


class BhParams(C.Structure):
    _fields_ = [("M", C.c_double), ("a", C.c_double), ("Q", C.c_double), ("gamma", C.c_double),
                ("limiter", C.c_int32), ("maxiter", C.c_int32), ("tol", C.c_double),
                ("cM", C.c_double), ("ca", C.c_double), ("cQ", C.c_double),
                ("precision", C.c_int32), ("reserved", C.c_int32)]


class BhPool(C.Structure):
    _fields_ = [("npatch", C.c_int32), ("U", _vp), ("W", _vp), ("dU", _vp), ("F", _vp), ("Bf", _vp),
                ("EMF", _vp), ("rth", _vp), ("pgeo", _vp), ("nbr", _vp), ("all", _vp),
                ("leaves", _vp), ("nleaf", C.c_int32), ("err", _vp), ("leafmask", _vp), ("status", _vp),
                ("aux", _vp), ("Wd", _vp), ("nall", C.c_int32)]


class BhAnalysisParams(C.Structure):
    _fields_ = [("hrz", C.c_double), ("rs", C.c_double), ("rho_min_full", C.c_double),
                ("rho_min_bundle", C.c_double)]


BH_NQ = 20


class BhError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"bhgpu: CUDA library {LIB_PATH} is missing; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = C.CDLL(LIB_PATH)
    P, PP = C.POINTER(BhParams), C.POINTER(BhPool)
    i32, i64, dbl = C.c_int32, C.c_int64, C.c_double
    sig = {
        "bh_abi_version": ([], C.c_int),
        "bh_read_error": ([PP, C.POINTER(i32), _vp], C.c_int),
        "bh_clear_error": ([PP, _vp], C.c_int),
        "bh_metric_comp": ([P, _vp, _vp, i64, _vp, _vp], C.c_int),
        "bh_ptoc": ([P, _vp, _vp, _vp, i64, _vp, _vp, _vp], C.c_int),
        "bh_ctop": ([P, _vp, _vp, _vp, i64, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "bh_hlld": ([P, _vp, _vp, _vp, _vp, _vp, _vp, i32, i64, _vp, _vp, _vp], C.c_int),
        "bh_geometry": ([PP, _vp], C.c_int),
        "bh_reconfp": ([P, PP, i32, i32, _vp, _vp, _vp], C.c_int),
        "bh_fluxcomp": ([P, PP, _vp], C.c_int),
        "bh_emfcomp": ([PP, _vp], C.c_int),
        "bh_bfupdate": ([PP, _vp, _vp], C.c_int),
        "bh_f2cb": ([P, PP, _vp], C.c_int),
        "bh_maxdivb": ([PP, _vp, _vp], C.c_int),
        "bh_div_source": ([P, PP, _vp, _vp, _vp], C.c_int),
        "bh_ghosts": ([P, PP, _vp, i32, _vp], C.c_int),
        "bh_prims": ([P, PP, _vp], C.c_int),
        "bh_ghosts_prims": ([P, PP, _vp], C.c_int),
        "bh_ghosts_prims_static": ([P, PP, _vp], C.c_int),
        "bh_update": ([P, PP, _vp, i32, _vp], C.c_int),
        "bh_floors": ([P, PP, _vp], C.c_int),
        "bh_dtcomp": ([P, PP, dbl, _vp, _vp], C.c_int),
        "bh_regrid_flags": ([P, PP, _vp, _vp, _vp], C.c_int),
        "bh_analysis": ([P, PP, C.POINTER(BhAnalysisParams), _vp, _vp, _vp], C.c_int),
        "bh_torus_init": ([P, PP, dbl, dbl, _vp, _vp], C.c_int),
        "bh_refine": ([P, PP, _vp, i32, _vp], C.c_int),
        "bh_ccrstr": ([P, PP, _vp, i32, _vp], C.c_int),
        "bh_b_init": ([P, PP, _vp, i32, _vp], C.c_int),
        "bh_rkstg": ([P, PP, _vp, i32, _vp, _vp, i32, _vp], C.c_int),
        "bh_step": ([P, PP, dbl, _vp, _vp, _vp, i32, _vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


lib = _load()


def check(rc: int, what: str):
    if rc != BH_OK:
        raise BhError(f"{what} failed with code {rc}")
