"""CPU checkers for the GPU block update -- TEST INFRASTRUCTURE ONLY.

Two checkers share one ctypes front end and one numpy "pool" layout:

* ``Oracle``  -- ``liboracle.so``, the plain-C restatement in bh_oracle.c.
  It travels with the repository and is the checker on any host.
* ``RefSolver`` -- ``_ref/libbhref.so``, the reference solver's own C++
  sources compiled by oracle/Makefile plus the harness in ref_shim.cpp.
  It pins the restatement (bit for bit) and is the CPU baseline.

Only tests, the smoke check and the benchmark's CPU-baseline leg import
this package; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NC, NF, NE, NMC = 8000, 8400, 8820, 120
NQ = 20   # raw integrals of orc_analysis (ORC_NQ)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


def _ptr(a, t=_dp):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays handed to the checkers must be C-contiguous"
    return a.ctypes.data_as(t)


class OrcParams(C.Structure):
    _fields_ = [("M", C.c_double), ("a", C.c_double), ("Q", C.c_double), ("gamma", C.c_double),
                ("limiter", C.c_int32), ("maxiter", C.c_int32), ("tol", C.c_double),
                ("cM", C.c_double), ("ca", C.c_double), ("cQ", C.c_double)]


class OrcPool(C.Structure):
    _fields_ = [("npatch", C.c_int32), ("U", _dp), ("W", _dp), ("dU", _dp), ("F", _dp),
                ("Bf", _dp), ("EMF", _dp), ("rth", _dp), ("pgeo", _dp), ("nbr", _ip),
                ("leaf", _u8p), ("lvl", _ip), ("ijk", _ip), ("Wd", _dp)]


class HostPool:
    """numpy arrays of one patch pool in the shared SoA layout."""

    def __init__(self, tables: dict):
        n = len(tables["lvl"])
        self.npatch = n
        self.U = np.zeros((n, 8, NC))
        self.W = np.zeros((n, 8, NC))
        self.dU = np.zeros((n, 8, NC))
        self.F = np.zeros((n, 3, 8, NF))
        self.Bf = np.zeros((n, 3, NF))
        self.EMF = np.zeros((n, 3, NE))
        self.rth = np.zeros((n, 2, NC))
        self.Wd = np.zeros((n, 4, NC))      # lor, p, h, b2 as floors / regrid set them
        self.pgeo = np.ascontiguousarray(tables["pgeo"], np.float64)
        self.nbr = np.ascontiguousarray(tables["nbr"], np.int32)
        self.leaf = np.ascontiguousarray(tables["leaf"], np.uint8)
        self.lvl = np.ascontiguousarray(tables["lvl"], np.int32)
        self.ijk = np.ascontiguousarray(tables["ijk"], np.int32)

    def copy(self):
        o = HostPool.__new__(HostPool)
        for k, v in self.__dict__.items():
            o.__dict__[k] = v.copy() if isinstance(v, np.ndarray) else v
        return o

    def cstruct(self) -> OrcPool:
        return OrcPool(self.npatch, _ptr(self.U), _ptr(self.W), _ptr(self.dU), _ptr(self.F),
                       _ptr(self.Bf), _ptr(self.EMF), _ptr(self.rth), _ptr(self.pgeo),
                       _ptr(self.nbr, _ip), _ptr(self.leaf, _u8p), _ptr(self.lvl, _ip),
                       _ptr(self.ijk, _ip), _ptr(self.Wd))


class DomainError(ValueError):
    """The reference throws std::domain_error from its EOS (thermo.cpp:11-31)."""


def reference_root() -> str:
    """Root of the reference checkout: $BH_REFERENCE if set, else the
    Makefile's default (REF ?=), which is the only place that names one."""
    env = os.environ.get("BH_REFERENCE")
    if env:
        return env
    out = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True)
    return out.stdout.strip() if out.returncode == 0 else ""


def build(ref: bool = True, quiet: bool = True):
    """Compile the checkers (the reference harness only if its sources exist)."""
    targets = ["all"]
    root = reference_root() if ref else ""
    if root and os.path.isdir(os.path.join(root, "src", "fluid")):
        targets += ["ref", "REF=" + root]
    out = subprocess.run(["make", "-C", HERE] + targets, capture_output=quiet, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + (out.stderr or ""))


def _params(M, a, Q, gamma, limiter=1, maxiter=500, tol=1e-10):
    # every cell carries a default-constructed metric (M=1, a=0, Q=0), cell.hpp:25
    return OrcParams(M, a, Q, gamma, limiter, maxiter, tol, 1.0, 0.0, 0.0)


class Oracle:
    """ctypes front end of liboracle.so (the C restatement)."""

    def __init__(self, M=0.0, a=0.0, Q=0.0, gamma=4.0 / 3.0, limiter=1, maxiter=500, tol=1e-10, fma=False,
                 noise=False, seed=0):
        """fma=True loads the build with fused multiply-add contraction, and
        noise=True the build whose libm results carry one-ulp noise (pattern
        chosen by seed): the same algorithm with different last-bit rounding
        (see bh_oracle.c).  The noise seed is process-wide; it is set again
        before every call of this object."""
        name = "liboracle_fma.so" if fma else "liboracle_noise.so" if noise else "liboracle.so"
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            build(ref=False)
        self.lib = C.CDLL(path)
        self.P = _params(M, a, Q, gamma, limiter, maxiter, tol)
        self.noise_seed = seed if noise else None
        L = self.lib
        if noise:
            L.orc_set_noise_seed.argtypes = [C.c_uint64]
            _orig = {}
            for fname in ("orc_metric_batch", "orc_ptoc_batch", "orc_ctop_batch", "orc_hlld_batch", "orc_geometry",
                          "orc_fluxcomp_all", "orc_ghosts_all", "orc_prims", "orc_update", "orc_rkstg",
                          "orc_floors_all", "orc_dtcomp", "orc_step", "orc_ct_all", "orc_div_source_all"):
                _orig[fname] = getattr(L, fname)
            self._noise_fns = _orig
        PP, PO = C.POINTER(OrcParams), C.POINTER(OrcPool)
        L.orc_metric_batch.argtypes = [PP, _dp, _dp, C.c_int64, _dp]
        L.orc_ptoc_batch.argtypes = [PP, _dp, _dp, _dp, C.c_int64, _dp, _dp]
        L.orc_ctop_batch.argtypes = [PP, _dp, _dp, _dp, C.c_int64, _dp, _dp, _ip, _ip, _ip]
        L.orc_hlld_batch.argtypes = [PP, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int64, _dp, _dp, _ip]
        L.orc_geometry.argtypes = [PO]
        L.orc_reconfp_all.argtypes = [PP, PO, C.c_int, C.c_int, _dp, _dp]
        L.orc_fluxcomp_all.argtypes = [PP, PO]
        L.orc_emfcomp.argtypes = [PO, C.c_int]
        L.orc_bfupdate.argtypes = [PO, C.c_int, C.c_double]
        L.orc_f2cb.argtypes = [PP, PO, C.c_int]
        L.orc_ct_all.argtypes = [PP, PO, C.c_double]
        L.orc_div_source_all.argtypes = [PP, PO, _dp, _dp]
        L.orc_ghosts_all.argtypes = [PP, PO]
        L.orc_prims.argtypes = [PP, PO]
        L.orc_update.argtypes = [PP, PO, C.c_double, C.c_int]
        L.orc_rkstg.argtypes = [PP, PO, C.c_double, C.c_int]
        L.orc_floors_all.argtypes = [PP, PO]
        L.orc_dtcomp.argtypes = [PP, PO, C.c_double, _dp]
        L.orc_step.argtypes = [PP, PO, C.c_double, _dp]
        L.orc_maxdivb_all.argtypes = [PO, _dp]
        L.orc_regrid_flags.argtypes = [PO, C.c_int, C.c_int]
        L.orc_analysis.argtypes = [PP, PO, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.orc_ctop_guess_batch.argtypes = [PP, _dp, _dp, _dp, C.c_int64, _dp, _dp, _dp, _ip, _ip, _ip, _dp]
        L.orc_b_init.argtypes = [PO, C.c_int]
        L.orc_refine_data.argtypes = [PP, PO, C.c_int, _ip]
        L.orc_ccrstr.argtypes = [PP, PO, C.c_int, _ip]
        for f in ("orc_regrid_flags", "orc_refine_data", "orc_ccrstr"):
            getattr(L, f).restype = C.c_int
        for f in ("orc_ptoc_batch", "orc_fluxcomp_all", "orc_ghosts_all", "orc_prims", "orc_update",
                  "orc_rkstg", "orc_floors_all", "orc_dtcomp", "orc_step"):
            getattr(L, f).restype = C.c_int

    def _chk(self, rc):
        if rc < 0:
            raise DomainError("density is not positive (reference thermo.cpp:11)")

    def __getattribute__(self, name):
        seed = object.__getattribute__(self, "__dict__").get("noise_seed")
        if seed is not None and name in ("metric", "ptoc", "ctop", "hlld", "geometry", "reconfp_all", "fluxcomp",
                                         "emfcomp", "bfupdate", "f2cb", "ct", "div_source", "ghosts", "prims",
                                         "update", "rkstg", "floors", "dtcomp", "step", "maxdivb",
                                         "regrid_flags", "b_init", "refine_data", "ccrstr"):
            object.__getattribute__(self, "lib").orc_set_noise_seed(seed)
        return object.__getattribute__(self, name)

    # ---- stateless physics (SoA [8][n]) -------------------------------
    def metric(self, r, th):
        r = np.ascontiguousarray(r, np.float64); th = np.ascontiguousarray(th, np.float64)
        out = np.zeros((len(r), NMC))
        self.lib.orc_metric_batch(C.byref(self.P), _ptr(r), _ptr(th), len(r), _ptr(out))
        return out

    def ptoc(self, W, r, th):
        W = np.ascontiguousarray(W, np.float64); n = W.shape[1]
        r = np.ascontiguousarray(r, np.float64); th = np.ascontiguousarray(th, np.float64)
        U = np.zeros((8, n)); Wd = np.zeros((4, n))
        self._chk(self.lib.orc_ptoc_batch(C.byref(self.P), _ptr(W), _ptr(r), _ptr(th), n, _ptr(U), _ptr(Wd)))
        return U, Wd

    def ctop(self, U, r, th):
        U = np.ascontiguousarray(U, np.float64); n = U.shape[1]
        r = np.ascontiguousarray(r, np.float64); th = np.ascontiguousarray(th, np.float64)
        W = np.zeros((8, n)); Wd = np.zeros((5, n))
        st = np.zeros(n, np.int32); it = np.zeros(n, np.int32); pa = np.zeros(n, np.int32)
        self.lib.orc_ctop_batch(C.byref(self.P), _ptr(U), _ptr(r), _ptr(th), n, _ptr(W), _ptr(Wd),
                                _ptr(st, _ip), _ptr(it, _ip), _ptr(pa, _ip))
        return W, Wd, st, it, pa

    def hlld(self, WL, WR, UL, UR, r, th, dim=0):
        arrs = [np.ascontiguousarray(x, np.float64) for x in (WL, WR, UL, UR, r, th)]
        n = arrs[0].shape[1]
        F = np.zeros((8, n)); cts = np.zeros(n); st = np.zeros(n, np.int32)
        self.lib.orc_hlld_batch(C.byref(self.P), *[_ptr(x) for x in arrs], dim, n, _ptr(F), _ptr(cts), _ptr(st, _ip))
        return F, cts, st

    # ---- pool level -----------------------------------------------------
    def geometry(self, pool: HostPool):
        s = pool.cstruct(); self.lib.orc_geometry(C.byref(s))

    def reconfp_all(self, pool, dim, lim):
        n = pool.npatch * 17 * 16 * 16
        L = np.zeros((8, n)); R = np.zeros((8, n))
        s = pool.cstruct(); self.lib.orc_reconfp_all(C.byref(self.P), C.byref(s), dim, lim, _ptr(L), _ptr(R))
        return L, R

    def fluxcomp(self, pool):
        s = pool.cstruct(); self._chk(self.lib.orc_fluxcomp_all(C.byref(self.P), C.byref(s)))

    def emfcomp(self, pool):
        s = pool.cstruct()
        for p in range(pool.npatch):
            self.lib.orc_emfcomp(C.byref(s), p)

    def bfupdate(self, pool, dt):
        s = pool.cstruct()
        for p in range(pool.npatch):
            self.lib.orc_bfupdate(C.byref(s), p, dt)

    def f2cb(self, pool):
        s = pool.cstruct()
        for p in range(pool.npatch):
            self.lib.orc_f2cb(C.byref(self.P), C.byref(s), p)

    def ct(self, pool, dt):
        s = pool.cstruct(); self.lib.orc_ct_all(C.byref(self.P), C.byref(s), dt)

    def div_source(self, pool):
        d = np.zeros((pool.npatch, 8, NC)); sr = np.zeros((pool.npatch, 8, NC))
        s = pool.cstruct(); self.lib.orc_div_source_all(C.byref(self.P), C.byref(s), _ptr(d), _ptr(sr))
        return d, sr

    def ghosts(self, pool):
        s = pool.cstruct(); self._chk(self.lib.orc_ghosts_all(C.byref(self.P), C.byref(s)))

    def prims(self, pool):
        s = pool.cstruct(); self._chk(self.lib.orc_prims(C.byref(self.P), C.byref(s)))

    def update(self, pool, dt, stage):
        s = pool.cstruct(); self._chk(self.lib.orc_update(C.byref(self.P), C.byref(s), dt, stage))

    def rkstg(self, pool, dt, stage):
        s = pool.cstruct(); self._chk(self.lib.orc_rkstg(C.byref(self.P), C.byref(s), dt, stage))

    def floors(self, pool):
        s = pool.cstruct(); self._chk(self.lib.orc_floors_all(C.byref(self.P), C.byref(s)))

    def dtcomp(self, pool, cfl):
        dt = C.c_double(0); s = pool.cstruct()
        self._chk(self.lib.orc_dtcomp(C.byref(self.P), C.byref(s), cfl, C.byref(dt)))
        return dt.value

    def step(self, pool, cfl):
        dt = C.c_double(0); s = pool.cstruct()
        self._chk(self.lib.orc_step(C.byref(self.P), C.byref(s), cfl, C.byref(dt)))
        return dt.value

    def ctop_guess(self, U, r, th, xi0=None):
        """ctop with Newton started from xi0 [n] (None or NaN: the midpoint);
        returns (W, Wd, status, iters, path, pre) with pre [7][n] = D, tau,
        Ssq, Bsq, SB, xi_l, xi_h of the preamble."""
        U = np.ascontiguousarray(U, np.float64); n = U.shape[1]
        r = np.ascontiguousarray(r, np.float64); th = np.ascontiguousarray(th, np.float64)
        x = None if xi0 is None else np.ascontiguousarray(xi0, np.float64)
        W = np.zeros((8, n)); Wd = np.zeros((5, n)); pre = np.zeros((7, n))
        st = np.zeros(n, np.int32); it = np.zeros(n, np.int32); pa = np.zeros(n, np.int32)
        self.lib.orc_ctop_guess_batch(C.byref(self.P), _ptr(U), _ptr(r), _ptr(th), n, _ptr(x) if x is not None else None,
                                      _ptr(W), _ptr(Wd), _ptr(st, _ip), _ptr(it, _ip), _ptr(pa, _ip), _ptr(pre))
        return W, Wd, st, it, pa, pre

    def analysis(self, pool, hrz, rs, rho_min_full=0.01, rho_min_bundle=0.005):
        """Raw integrals of analysis::analyser (quantitatives.cpp), summed in
        the reference's order, in the ORC_Q_* order of bh_oracle.h, and the
        sums of the absolute values of their terms."""
        out = np.zeros(NQ); absout = np.zeros(NQ); s = pool.cstruct()
        self.lib.orc_analysis(C.byref(self.P), C.byref(s), hrz, rs, rho_min_full, rho_min_bundle, _ptr(out),
                              _ptr(absout))
        return out, absout

    # AMR regrid pieces (grid.cpp:573-835)
    def regrid_flags(self, pool):
        """Per-patch flags of amrtree::regrid's cell loop (bit 0 refine, bit 1
        erase) for the leaf patches; 0 for the others."""
        s = pool.cstruct()
        return np.array([self.lib.orc_regrid_flags(C.byref(s), p, int(pool.lvl[p])) if pool.leaf[p] else 0
                         for p in range(pool.npatch)], np.int32)

    def b_init(self, pool, p):
        s = pool.cstruct(); self.lib.orc_b_init(C.byref(s), p)

    def refine_data(self, pool, p, kids):
        k = np.ascontiguousarray(kids, np.int32); s = pool.cstruct()
        self._chk(self.lib.orc_refine_data(C.byref(self.P), C.byref(s), p, _ptr(k, _ip)))

    def ccrstr(self, pool, p, kids):
        k = np.ascontiguousarray(kids, np.int32); s = pool.cstruct()
        self._chk(self.lib.orc_ccrstr(C.byref(self.P), C.byref(s), p, _ptr(k, _ip)))

    def maxdivb(self, pool):
        out = np.zeros(pool.npatch); s = pool.cstruct()
        self.lib.orc_maxdivb_all(C.byref(s), _ptr(out))
        return out


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libbhref.so"))


class RefSolver:
    """The reference solver itself (an ``amrtree`` owned by the harness)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            path = os.path.join(HERE, "_ref", "libbhref.so")
            if not os.path.exists(path):
                raise FileNotFoundError("reference harness not built (oracle/Makefile ref)")
            L = C.CDLL(path)
            v = C.c_void_p
            L.ref_new.restype = v
            L.ref_new.argtypes = [_dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
            L.ref_free.argtypes = [v]
            L.ref_npatch.argtypes = [v]
            L.ref_patch_info.argtypes = [v, _dp, _ip, _ip, _u8p]
            L.ref_nbhd.argtypes = [v, C.c_int, C.c_int, C.c_int]
            L.ref_geom.argtypes = [v, _dp]
            L.ref_put.argtypes = [v, _dp, _dp, _dp]
            L.ref_get.argtypes = [v, _dp, _dp, _dp, _dp, _dp, _dp]
            L.ref_refine.argtypes = [v, C.c_int]
            L.ref_flatten.argtypes = [v, C.c_int]
            L.ref_regrid.argtypes = [v]
            L.ref_derived.argtypes = [v, _dp]
            L.ref_batch.argtypes = [v, C.c_double, _dp]
            L.ref_torus_init.argtypes = [v, _dp]
            L.ref_bundle.argtypes = [v, C.c_double, _dp]
            L.ref_metric_batch.argtypes = [C.c_double] * 3 + [_dp, _dp, C.c_int64, _dp]
            L.ref_ptoc_batch.argtypes = [C.c_double] * 4 + [_dp, _dp, _dp, C.c_int64, _dp, _dp]
            L.ref_ctop_batch.argtypes = [C.c_double] * 4 + [_dp, _dp, _dp, C.c_int64, _dp, _dp, _ip]
            L.ref_hlld_batch.argtypes = [C.c_double] * 4 + [_dp] * 6 + [C.c_int, C.c_int64, _dp, _dp, _ip]
            L.ref_reconfp_all.argtypes = [v, C.c_int, C.c_int, _dp, _dp]
            L.ref_fluxcomp_all.argtypes = [v, C.c_int]
            L.ref_emfcomp_all.argtypes = [v]
            L.ref_bfupdate_all.argtypes = [v, C.c_double]
            L.ref_f2cb_all.argtypes = [v]
            L.ref_maxdivb_all.argtypes = [v, _dp]
            L.ref_div_source_all.argtypes = [v, _dp, _dp]
            L.ref_ghosts_all.argtypes = [v, _ip]
            L.ref_prims.argtypes = [v]
            L.ref_update.argtypes = [v, C.c_double, C.c_int]
            L.ref_dtcomp.argtypes = [v, C.c_double, _dp]
            L.ref_floors_all.argtypes = [v, C.c_int]
            L.ref_rkstg.argtypes = [v, C.c_double, C.c_int, _ip, C.c_int]
            L.ref_step.argtypes = [v, C.c_double, _ip, C.c_int, _dp]
            L.ref_step_native.argtypes = [v, C.c_double, _dp]
            cls._lib = L
        return cls._lib

    def __init__(self, dom_l, dom_h, nqlt, M=0.0, a=0.0, Q=0.0, gamma=4.0 / 3.0):
        L = self.lib()
        lo = np.array(dom_l, np.float64); hi = np.array(dom_h, np.float64)
        self.M, self.a, self.Q, self.gamma = M, a, Q, gamma
        self.h = L.ref_new(_ptr(lo), _ptr(hi), nqlt, M, a, Q, gamma)

    def __del__(self):
        if getattr(self, "h", None) and self._lib is not None:
            self._lib.ref_free(self.h)
            self.h = None

    def _chk(self, rc):
        if rc == -1:
            raise DomainError("reference threw std::domain_error")
        if rc < -1:
            raise RuntimeError("reference threw")

    @property
    def npatch(self):
        return self.lib().ref_npatch(self.h)

    def patch_info(self):
        n = self.npatch
        pgeo = np.zeros((n, 6)); lvl = np.zeros(n, np.int32); ijk = np.zeros((n, 3), np.int32)
        leaf = np.zeros(n, np.uint8)
        self.lib().ref_patch_info(self.h, _ptr(pgeo), _ptr(lvl, _ip), _ptr(ijk, _ip), _ptr(leaf, _u8p))
        return dict(pgeo=pgeo, lvl=lvl, ijk=ijk, leaf=leaf)

    def nbhd(self, p, dim, side):
        return self.lib().ref_nbhd(self.h, p, dim, side)

    def geom(self):
        rth = np.zeros((self.npatch, 2, NC)); self.lib().ref_geom(self.h, _ptr(rth)); return rth

    def put(self, pool: HostPool):
        self.lib().ref_put(self.h, _ptr(pool.U), _ptr(pool.W), _ptr(pool.Bf))

    def get(self, pool: HostPool):
        self.lib().ref_get(self.h, _ptr(pool.U), _ptr(pool.W), _ptr(pool.dU), _ptr(pool.F),
                           _ptr(pool.Bf), _ptr(pool.EMF))

    def refine(self, p):
        self._chk(self.lib().ref_refine(self.h, p))

    def flatten(self, p):
        self._chk(self.lib().ref_flatten(self.h, p))

    def regrid(self):
        """amrtree::regrid; the patch count changes (npatch, patch_info)."""
        self._chk(self.lib().ref_regrid(self.h))

    def derived(self):
        out = np.zeros((self.npatch, 4, NC)); self.lib().ref_derived(self.h, _ptr(out)); return out

    def torus_init(self):
        """main()'s initial data (Fishbone-Moncrief torus + A_phi field);
        returns (status, interior rho_max after fm_init)."""
        m = C.c_double(0)
        rc = self.lib().ref_torus_init(self.h, C.byref(m))
        self._chk(rc if rc < 0 else 0)
        return rc, m.value

    def batch(self, t):
        out = np.zeros(17); self.lib().ref_batch(self.h, t, _ptr(out)); return out

    def bundle(self, t):
        out = np.zeros(6); self.lib().ref_bundle(self.h, t, _ptr(out)); return out

    # stateless
    def metric(self, r, th):
        r = np.ascontiguousarray(r, np.float64); th = np.ascontiguousarray(th, np.float64)
        out = np.zeros((len(r), NMC))
        self.lib().ref_metric_batch(self.M, self.a, self.Q, _ptr(r), _ptr(th), len(r), _ptr(out))
        return out

    def ptoc(self, W, r, th):
        W = np.ascontiguousarray(W, np.float64); n = W.shape[1]
        U = np.zeros((8, n)); Wd = np.zeros((4, n))
        self._chk(self.lib().ref_ptoc_batch(self.M, self.a, self.Q, self.gamma, _ptr(W),
                                            _ptr(np.ascontiguousarray(r, np.float64)),
                                            _ptr(np.ascontiguousarray(th, np.float64)), n, _ptr(U), _ptr(Wd)))
        return U, Wd

    def ctop(self, U, r, th):
        U = np.ascontiguousarray(U, np.float64); n = U.shape[1]
        W = np.zeros((8, n)); Wd = np.zeros((5, n)); st = np.zeros(n, np.int32)
        self.lib().ref_ctop_batch(self.M, self.a, self.Q, self.gamma, _ptr(U),
                                  _ptr(np.ascontiguousarray(r, np.float64)),
                                  _ptr(np.ascontiguousarray(th, np.float64)), n, _ptr(W), _ptr(Wd), _ptr(st, _ip))
        return W, Wd, st

    def hlld(self, WL, WR, UL, UR, r, th, dim=0):
        arrs = [np.ascontiguousarray(x, np.float64) for x in (WL, WR, UL, UR, r, th)]
        n = arrs[0].shape[1]
        F = np.zeros((8, n)); cts = np.zeros(n); st = np.zeros(n, np.int32)
        self.lib().ref_hlld_batch(self.M, self.a, self.Q, self.gamma, *[_ptr(x) for x in arrs], dim, n,
                                  _ptr(F), _ptr(cts), _ptr(st, _ip))
        return F, cts, st

    # pool level (the harness's amrtree holds the state; put/get copy it)
    def reconfp_all(self, dim, lim):
        n = self.npatch * 17 * 16 * 16
        L = np.zeros((8, n)); R = np.zeros((8, n))
        self.lib().ref_reconfp_all(self.h, dim, lim, _ptr(L), _ptr(R))
        return L, R

    def fluxcomp(self, lim):
        self._chk(self.lib().ref_fluxcomp_all(self.h, lim))

    def emfcomp(self):
        self.lib().ref_emfcomp_all(self.h)

    def bfupdate(self, dt):
        self.lib().ref_bfupdate_all(self.h, dt)

    def f2cb(self):
        self.lib().ref_f2cb_all(self.h)

    def maxdivb(self):
        out = np.zeros(self.npatch); self.lib().ref_maxdivb_all(self.h, _ptr(out)); return out

    def div_source(self):
        d = np.zeros((self.npatch, 8, NC)); s = np.zeros((self.npatch, 8, NC))
        self._chk(self.lib().ref_div_source_all(self.h, _ptr(d), _ptr(s)))
        return d, s

    def ghosts(self, nbr=None):
        nb = None if nbr is None else np.ascontiguousarray(nbr, np.int32)
        self._chk(self.lib().ref_ghosts_all(self.h, _ptr(nb, _ip) if nb is not None else None))

    def prims(self):
        self._chk(self.lib().ref_prims(self.h))

    def update(self, dt, stage):
        self._chk(self.lib().ref_update(self.h, dt, stage))

    def dtcomp(self, cfl):
        dt = C.c_double(0); self._chk(self.lib().ref_dtcomp(self.h, cfl, C.byref(dt))); return dt.value

    def floors(self, native=False):
        self._chk(self.lib().ref_floors_all(self.h, 1 if native else 0))

    def rkstg(self, dt, stage, nbr, lim):
        nb = np.ascontiguousarray(nbr, np.int32)
        self._chk(self.lib().ref_rkstg(self.h, dt, stage, _ptr(nb, _ip), lim))

    def step(self, cfl, nbr, lim):
        nb = np.ascontiguousarray(nbr, np.int32); dt = C.c_double(0)
        self._chk(self.lib().ref_step(self.h, cfl, _ptr(nb, _ip), lim, C.byref(dt)))
        return dt.value

    def step_native(self, cfl=0.4):
        dt = C.c_double(0); self._chk(self.lib().ref_step_native(self.h, cfl, C.byref(dt))); return dt.value
