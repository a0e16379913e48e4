"""ctypes front end of libhostcheck.so: the kernels' per-item functions run
on the CPU (see hostcheck.cu).  Test code only."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(HERE, "libhostcheck.so")
# the same items with the reciprocal-reuse quotients of the FMA and mixed
# variants (BH_RCP), still without contraction
LIB_RCP = os.path.join(HERE, "libhostcheck_rcp.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def build(rcp: bool = False):
    lib = LIB_RCP if rcp else LIB
    src = os.path.join(HERE, "hostcheck.cu")
    csrc = os.path.join(REPO, "black-hole-simulator_b200", "csrc")
    deps = [src] + [os.path.join(csrc, f) for f in os.listdir(csrc)] + [os.path.join(REPO, "include", "bhgpu.h")]
    if os.path.exists(lib) and all(os.path.getmtime(lib) >= os.path.getmtime(d) for d in deps):
        return lib
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-I" + os.path.join(REPO, "include"),
           "-I" + csrc] + (["-DBH_RCP"] if rcp else []) + [src, "-o", lib]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return lib


def _d(a):
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


class HostKernels:
    def __init__(self, M, a, Q, gamma, limiter, maxiter=500, tol=1e-10, rcp=False):
        lib = build(rcp)
        import sys
        sys.path.insert(0, os.path.join(REPO, "black-hole-simulator_b200"))
        from bhgpu._lib import BhParams, BhPool
        self.BhPool = BhPool
        self.L = C.CDLL(lib)
        self.P = BhParams(M, a, Q, gamma, limiter, maxiter, tol, 1.0, 0.0, 0.0)
        self.L.hc_dtcomp.restype = C.c_double
        self.L.hc_step.restype = C.c_double
        self.L.hc_dtcomp.argtypes = [C.c_void_p, C.c_void_p, C.c_double]
        self.L.hc_step.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        self.L.hc_bfupdate.argtypes = [C.c_void_p, C.c_double]
        self.L.hc_update.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int]
        self.L.hc_rkstg.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_int]

    def pool(self, hp, reuse=True, aux=True):
        """bh_pool over the numpy arrays of an oracle.HostPool; reuse=False
        leaves the status scratch unset (ghost cells recompute con2prim),
        aux=False the per-cell flux scratch (faces compute its values)."""
        self._all = np.arange(hp.npatch, dtype=np.int32)
        self._leaves = np.nonzero(hp.leaf)[0].astype(np.int32)
        self._leafmask = np.ascontiguousarray(hp.leaf, np.uint8)
        self._status = np.full((hp.npatch, 8000), 7, np.uint8)
        self._aux = np.full((hp.npatch, 6, 8000), np.nan)
        err = np.zeros(1, np.int32)
        self._err = err
        return self.BhPool(hp.npatch, _d(hp.U), _d(hp.W), _d(hp.dU), _d(hp.F), _d(hp.Bf), _d(hp.EMF), _d(hp.rth),
                           _d(hp.pgeo), _d(hp.nbr), _d(self._all), _d(self._leaves), len(self._leaves), _d(err),
                           _d(self._leafmask), _d(self._status) if reuse else None,
                           _d(self._aux) if aux else None, _d(hp.Wd))

    def call(self, name, *args):
        return getattr(self.L, name)(C.byref(self.P), *args)
