"""ctypes front end of liboracle_fixed.so -- the CPU oracle of the corrected
("fixed") scheme (bh_fixed.c).  TEST INFRASTRUCTURE ONLY: used by the tests,
the smoke check and the bench's CPU leg as the checker of the CUDA kernels.

``FxHost`` holds the same arrays as ``bhgpu.fixed.FxGrid`` in host memory
(FP64) with the same block layout, so states move between them by plain
copies.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GB = 3   # ghost layers of every block's box (bh_fixed.c GB)
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lib = None


class FxoParams(C.Structure):
    _fields_ = [("M", C.c_double), ("a", C.c_double), ("gamma", C.c_double), ("cfl", C.c_double),
                ("rho_floor", C.c_double), ("u_floor", C.c_double), ("sigma_max", C.c_double),
                ("W_max", C.c_double), ("r_exc", C.c_double), ("tol", C.c_double), ("maxiter", C.c_int32),
                ("limiter", C.c_int32), ("precision", C.c_int32), ("reserved", C.c_int32)]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle_fixed.so")
        if not os.path.exists(path):
            raise FileNotFoundError("oracle not built (make -C oracle)")
        L = C.CDLL(path)
        P = C.POINTER(FxoParams)
        v, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.fxo_step.argtypes = [P, i32, v, v, i64] + [v] * 9 + [C.c_int]
        L.fxo_prims.argtypes = [P, i32, v, v, i64] + [v] * 8 + [C.c_int, C.c_int]
        L.fxo_ghosts.argtypes = [i32, v, v, i64, v, v, v, C.c_int, C.c_int, C.c_int]
        L.fxo_ghost_pass.argtypes = [i32, v, v, i64, v, v, v, C.c_int, C.c_int, C.c_int]
        L.fxo_emf_raw.argtypes = [i32, v, i64, v, v]
        L.fxo_emf_fix.argtypes = [i32, v, v, i64, v]
        L.fxo_emf.argtypes = [i32, v, v, i64, v, v, C.c_int]
        L.fxo_fluxes.argtypes = [P, i32, v, i64, v, v, v, v, C.c_int]
        L.fxo_update.argtypes = [P, i32, v, i64, v, v, v, v, v, v, v, v, C.c_int]
        L.fxo_divb.argtypes = [i32, v, i64, v, v]
        L.fxo_metric_batch.argtypes = [P, i64, v, v, v, v]
        L.fxo_deriv_batch.argtypes = [P, i64, v, v, v, v]
        L.fxo_cons_flux_batch.argtypes = [P, i64, v, v, v, C.c_int, v, v, v, v, v]
        L.fxo_hll_batch.argtypes = [P, i64, v, v, v, C.c_int, v, v, v]
        L.fxo_ppm_batch.argtypes = [i64, v, v, v]
        L.fxo_source_batch.argtypes = [P, i64, v, v, v, v, v]
        L.fxo_c2p_batch.argtypes = [P, i64, v, v, v, v, v, v, v, v, v]
        L.fxo_fm_batch.argtypes = [d, d, d, d, d, i64, v, v, v, v]
        L.fxo_fm_potential.argtypes = [d, d, d, d, d]
        L.fxo_fm_potential.restype = d
        L.fxo_fm_ell.argtypes = [d, d]
        L.fxo_fm_ell.restype = d
        L.fxo_torus_init.argtypes = [P, i32, v, i64, v, v, v, d, d, d, d, d, C.c_uint64, v, C.c_int]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def params(fx) -> FxoParams:
    """The oracle's parameter struct from a bhgpu.fixed.FxParams-like object
    (any object with the same attributes; limiter 0/1/2/3 or its name)."""
    lim = {"minmod": 0, "vanleer": 1, "mc": 2, "ppm": 3}.get(fx.limiter, fx.limiter)
    r_exc = fx.r_exc
    if r_exc is None:
        r_exc = 1.2 * (fx.M + np.sqrt(fx.M * fx.M - fx.a * fx.a)) if fx.M > 0 else 0.0
    return FxoParams(fx.M, fx.a, fx.gamma, fx.cfl, fx.rho_floor, fx.u_floor, fx.sigma_max, fx.W_max, r_exc, fx.tol,
                     fx.maxiter, int(lim), 0, 0)


class FxHost:
    """Host copy of a block grid (the oracle's state)."""

    def __init__(self, blocks: np.ndarray, nbr: np.ndarray, prm: FxoParams, nactive=None, maxlevel=None):
        """nactive: step blocks[:nactive] only (the rest are neighbours'
        copies); maxlevel: of the whole domain (default: of these blocks)"""
        self.blocks = np.ascontiguousarray(blocks)
        self.nbr = np.ascontiguousarray(nbr, np.int32)
        self.prm = prm
        self.nactive = len(self.blocks) if nactive is None else int(nactive)
        self.N = int(sum((int(n) + 2 * GB + 1) ** 3 for n in blocks["n"]))
        N = self.N
        self.U = np.zeros((8, N))
        self.U1 = np.zeros((8, N))
        self.W = np.zeros((8, N))
        self.Bf = np.zeros((3, N))
        self.Bf1 = np.zeros((3, N))
        self.F = np.zeros((3, 8, N))
        self.E = np.zeros((3, N))
        self.maxlevel = int(self.blocks["level"].max()) if maxlevel is None else int(maxlevel)
        self.dt = np.zeros(2)
        self.count = np.zeros(4, np.int32)

    @property
    def ghost_depth(self) -> int:
        """ghost layers the fill covers: 3 for PPM's stencil, else 2"""
        return 3 if self.prm.limiter == 3 else 2

    def _g(self):
        return (C.byref(self.prm), self.nactive, _p(self.blocks), _p(self.nbr), self.N)

    def step(self):
        lib().fxo_step(*self._g(), _p(self.U), _p(self.U1), _p(self.W), _p(self.Bf), _p(self.Bf1), _p(self.F),
                       _p(self.E), _p(self.dt), _p(self.count), self.maxlevel)

    def prims(self, stage=0, with_dt=False):
        lib().fxo_prims(*self._g(), _p(self.U), _p(self.U1), _p(self.W), _p(self.Bf), _p(self.Bf1), _p(self.F),
                        _p(self.dt), _p(self.count), stage, int(with_dt))

    def ghosts(self, stage=0):
        lib().fxo_ghosts(self.nactive, _p(self.blocks), _p(self.nbr), self.N, _p(self.W), _p(self.Bf),
                         _p(self.Bf1), stage, self.maxlevel, self.ghost_depth)

    def ghost_pass(self, stage, pass_):
        lib().fxo_ghost_pass(self.nactive, _p(self.blocks), _p(self.nbr), self.N, _p(self.W), _p(self.Bf),
                             _p(self.Bf1), stage, pass_, self.ghost_depth)

    def fluxes(self, stage=0):
        lib().fxo_fluxes(C.byref(self.prm), self.nactive, _p(self.blocks), self.N, _p(self.W), _p(self.Bf),
                         _p(self.Bf1), _p(self.F), stage)

    def emf(self):
        lib().fxo_emf(self.nactive, _p(self.blocks), _p(self.nbr), self.N, _p(self.F), _p(self.E),
                      self.maxlevel)

    def emf_raw(self):
        """the edge EMFs of the active blocks, uncorrected"""
        lib().fxo_emf_raw(self.nactive, _p(self.blocks), self.N, _p(self.F), _p(self.E))

    def update(self, stage=0):
        """edge EMFs from the fluxes (corrected at level changes), then the update"""
        self.emf()
        self._update(stage)

    def update_from_emf(self, stage=0):
        """the level-change correction of E (raw EMFs of every block it reads
        already in E), then the update"""
        if self.maxlevel > 0:
            lib().fxo_emf_fix(self.nactive, _p(self.blocks), _p(self.nbr), self.N, _p(self.E))
        self._update(stage)

    def _update(self, stage):
        lib().fxo_update(C.byref(self.prm), self.nactive, _p(self.blocks), self.N, _p(self.U), _p(self.U1),
                         _p(self.W), _p(self.Bf), _p(self.Bf1), _p(self.F), _p(self.E), _p(self.dt), stage)

    def divb(self) -> float:
        out = np.zeros(len(self.blocks))
        lib().fxo_divb(self.nactive, _p(self.blocks), self.N, _p(self.Bf), _p(out))
        return float(out.max())

    def torus_init(self, r_in=6.0, r_max=12.0, kappa=1e-3, beta=100.0, noise=0.04, seed=1):
        out = np.zeros(4)
        lib().fxo_torus_init(C.byref(self.prm), len(self.blocks), _p(self.blocks), self.N, _p(self.U), _p(self.W),
                             _p(self.Bf), r_in, r_max, kappa, beta, noise, seed, _p(out), self.maxlevel)
        return {"ell": out[0], "rho_max_raw": out[1], "field_scale": out[2], "beta": out[3]}

    def interior(self, arr: np.ndarray) -> np.ndarray:
        n = int(self.blocks["n"][0])
        S = n + 2 * GB + 1
        out = []
        for b in self.blocks:
            box = arr[..., int(b["off"]):int(b["off"]) + S ** 3].reshape(arr.shape[:-1] + (S, S, S))
            out.append(box[..., GB:GB + n, GB:GB + n, GB:GB + n])
        return np.stack(out, axis=-4)


# ---- batch physics ------------------------------------------------------
def metric(prm, x, y, z):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    out = np.zeros((len(x), 22))
    lib().fxo_metric_batch(C.byref(prm), len(x), _p(x), _p(y), _p(z), _p(out))
    return out


def deriv(prm, x, y, z):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    out = np.zeros((len(x), 12))
    lib().fxo_deriv_batch(C.byref(prm), len(x), _p(x), _p(y), _p(z), _p(out))
    return out


def cons_flux(prm, x, y, z, dd, w):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    w = np.ascontiguousarray(w, np.float64)
    n = len(x)
    u, F, lm, lp = np.zeros((8, n)), np.zeros((8, n)), np.zeros(n), np.zeros(n)
    lib().fxo_cons_flux_batch(C.byref(prm), n, _p(x), _p(y), _p(z), dd, _p(w), _p(u), _p(F), _p(lm), _p(lp))
    return u, F, lm, lp


def hll(prm, x, y, z, dd, wL, wR):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    wL, wR = np.ascontiguousarray(wL, np.float64), np.ascontiguousarray(wR, np.float64)
    F = np.zeros((8, len(x)))
    lib().fxo_hll_batch(C.byref(prm), len(x), _p(x), _p(y), _p(z), dd, _p(wL), _p(wR), _p(F))
    return F


def ppm(a):
    """PPM face states (L, R) of the faces whose cells p-3 .. p+2 are a[6][n]"""
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[1]
    L, R = np.zeros(n), np.zeros(n)
    lib().fxo_ppm_batch(n, _p(a), _p(L), _p(R))
    return L, R


def source(prm, x, y, z, w):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    w = np.ascontiguousarray(w, np.float64)
    S = np.zeros((8, len(x)))
    lib().fxo_source_batch(C.byref(prm), len(x), _p(x), _p(y), _p(z), _p(w), _p(S))
    return S


def con2prim(prm, x, y, z, U, B, wo):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    U, B, wo = (np.ascontiguousarray(v, np.float64) for v in (U, B, wo))
    n = len(x)
    w, st, it = np.zeros((8, n)), np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib().fxo_c2p_batch(C.byref(prm), n, _p(x), _p(y), _p(z), _p(U), _p(B), _p(wo), _p(w), _p(st), _p(it))
    return w, st, it


def fm(a, gamma, kappa, r_in, r_max, x, y, z):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
    out = np.zeros((len(x), 6))
    lib().fxo_fm_batch(a, gamma, kappa, r_in, r_max, len(x), _p(x), _p(y), _p(z), _p(out))
    return out


def fm_potential(a, ell, r, s2, c2):
    return lib().fxo_fm_potential(a, ell, r, s2, c2)


def fm_ell(a, r):
    return lib().fxo_fm_ell(a, r)
