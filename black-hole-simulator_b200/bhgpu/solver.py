"""Python host API of the GPU block update, named after the reference's
C++ entry points (src/fluid of Fjoerde/black-hole-simulator).

PyTorch provides the device buffers and the stream; every operation is one
or more launches of the hand-written sm_100a kernels in libbhgpu.so
through its C ABI.  Nothing here computes physics on the host.

Error behaviour: the reference throws std::domain_error when a density
<= 0 reaches its EOS (thermo.cpp:11-31).  The kernels record that in a
device error word; ``check=True`` (the default for the stateful calls)
synchronises, reads it and raises :class:`DomainError`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import BH_ERR_DOMAIN, BH_FP64, BH_FP64_FMA, BH_MC, BH_MIXED, BH_MINMOD, BH_VANLEER, BhParams, BhPool, check, lib
from .mesh import NC, NE, NF, Quilt

__all__ = ["Metric", "State", "Conserved", "hlld", "AmrTree", "RK2Integrator", "StepGraph", "DomainError",
           "BH_MINMOD", "BH_VANLEER", "BH_MC"]

_LIMITERS = {"minmod": BH_MINMOD, "vanleer": BH_VANLEER, "mc": BH_MC, "mclim": BH_MC}
# arithmetic variants: "fp64" keeps the reference's separate roundings (the
# parity form); "fp64-fma" contracts multiply-add pairs
PRECISIONS = {"fp64": BH_FP64, "fp64-fma": BH_FP64_FMA, "mixed": BH_MIXED}


class DomainError(ValueError):
    """A non-positive density reached the EOS (reference: std::domain_error)."""


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _p(t: torch.Tensor | None):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "bhgpu buffers must be contiguous CUDA tensors"
    return C.c_void_p(t.data_ptr())


def _dev(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, np.float64), device=device)


class Metric:
    """metric(M, a, Q) -- Kerr(-Newman)-Schild (metric.hpp:23-53)."""

    def __init__(self, M: float = 1.0, a: float = 0.0, Q: float = 0.0):
        self.M, self.a, self.Q = float(M), float(a), float(Q)

    def comp(self, r, th, device="cuda"):
        """metric::comp at n points: [n][120] in the member order of
        struct metriccomp (g, g_inv, Gamma, sqrtdetg, gam, gam_inv,
        sqrtdetgam, alpha, beta)."""
        r, th = _dev(r, device), _dev(th, device)
        out = torch.empty((r.numel(), 120), dtype=torch.float64, device=device)
        P = _params(self, State())
        check(lib.bh_metric_comp(C.byref(P), _p(r), _p(th), r.numel(), _p(out), _stream()), "metric::comp")
        return out


class State:
    """Ideal-gas EOS, state(gm) (state.hpp:9-20)."""

    def __init__(self, gm: float = 5.0 / 3.0):
        self.gamma = float(gm)


def _params(mtr: Metric, stt: State, limiter=BH_VANLEER, maxiter=500, tol=1e-10, precision="fp64") -> BhParams:
    # every cell carries a default-constructed metric() = (M=1, a=0, Q=0)
    # (cell.hpp:25, metric.hpp:30); the kernels use it where the reference
    # evaluates c.mtr
    prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    return BhParams(mtr.M, mtr.a, mtr.Q, stt.gamma, int(limiter), int(maxiter), float(tol), 1.0, 0.0, 0.0, prec, 0)


class Conserved:
    """conserved(mtr, stt) -- prim <-> cons (cons.hpp:62-80), batched.

    Arrays are SoA: W, U are [8][n] in the reference member order
    (rho, eps, v0, v1, v2, B0, B1, B2) and (D, S0, S1, S2, tau, B0, B1, B2).
    """

    def __init__(self, mtr: Metric, stt: State):
        self.mtr, self.stt = mtr, stt

    def ptoc(self, W, r, th, check_domain=True):
        """conserved::ptoc (conserved.cpp:17-73) -> (U [8][n], lor/p/h/b2 [4][n])."""
        W, r, th = _dev(W, "cuda"), _dev(r, "cuda"), _dev(th, "cuda")
        n = W.shape[1]
        U = torch.empty((8, n), dtype=torch.float64, device="cuda")
        Wd = torch.empty((4, n), dtype=torch.float64, device="cuda")
        P = _params(self.mtr, self.stt)
        check(lib.bh_ptoc(C.byref(P), _p(W), _p(r), _p(th), n, _p(U), _p(Wd), _stream()), "conserved::ptoc")
        if check_domain and n and bool((W[0] <= 0).any()):
            raise DomainError("density is not positive (thermo.cpp:11)")
        return U, Wd

    def ctop(self, U, r, th, maxiter: int = 500, tol: float = 1e-10, check_domain=True):
        """conserved::ctop (conserved.cpp:135-285) for n cells.

        Returns (W [8][n], p/T/h/lor/b2 [5][n], status [n], iters [n],
        path [n]); status 1 = recovered, 0 = the reference returns false,
        -1 = the reference throws (raised as DomainError if check_domain).
        """
        U, r, th = _dev(U, "cuda"), _dev(r, "cuda"), _dev(th, "cuda")
        n = U.shape[1]
        W = torch.empty((8, n), dtype=torch.float64, device="cuda")
        Wd = torch.empty((5, n), dtype=torch.float64, device="cuda")
        st = torch.empty(n, dtype=torch.int32, device="cuda")
        it = torch.empty(n, dtype=torch.int32, device="cuda")
        pa = torch.empty(n, dtype=torch.int32, device="cuda")
        P = _params(self.mtr, self.stt, maxiter=maxiter, tol=tol)
        check(lib.bh_ctop(C.byref(P), _p(U), _p(r), _p(th), n, _p(W), _p(Wd), _p(st), _p(it), _p(pa), _stream()),
              "conserved::ctop")
        if check_domain and n and bool((st < 0).any()):
            raise DomainError("density is not positive (thermo.cpp:11)")
        return W, Wd, st, it, pa


def hlld(WL, WR, UL, UR, mtr: Metric, r, th, stt: State, dim: int = 0):
    """hlld(WL, WR, UL, UR, mtr, r, th, stt, dim) (hlld.hpp:19), batched:
    returns (F [8][n] in cons order, ctspeed [n])."""
    arrs = [_dev(x, "cuda") for x in (WL, WR, UL, UR, r, th)]
    n = arrs[0].shape[1]
    F = torch.empty((8, n), dtype=torch.float64, device="cuda")
    cts = torch.empty(n, dtype=torch.float64, device="cuda")
    P = _params(mtr, stt)
    check(lib.bh_hlld(C.byref(P), *[_p(x) for x in arrs], int(dim), n, _p(F), _p(cts), _stream()), "hlld")
    return F, cts


class AmrTree:
    """The patch quilt and its device state -- grid::amrtree (grid.hpp:114-145).

    ``AmrTree(dom_l, dom_h, nqlt, M, a, Q, gm)`` builds nqlt^3 level-0
    patches of 16^3 cells (+2 ghost layers) like the reference constructor
    (grid.cpp:177-206), fills every cell with the floor state and its
    conserved variables, and keeps all per-patch arrays on the GPU in the
    reference's per-patch index order:

        U, W, dU : [npatch, 8, 8000]   F : [npatch, 3, 8, 8400]
        Bf : [npatch, 3, 8400]         EMF : [npatch, 3, 8820]
        rth : [npatch, 2, 8000]        (cell-centre r, theta)

    ``periodic`` wraps the level-0 neighbour search; ``limiter`` selects the
    slope limiter of the flux reconstruction (the reference's fluxcomp
    always uses van Leer, recon.hpp:41); ``precision`` selects the
    arithmetic variant ("fp64" reproduces the reference's roundings,
    "fp64-fma" contracts multiply-add pairs, "mixed" computes the face
    fluxes and the geometric source in FP32 and everything else in FP64).
    """

    def __init__(self, dom_l, dom_h, nqlt: int, M: float = 1.0, a: float = 0.0, Q: float = 0.0,
                 gm: float = 5.0 / 3.0, periodic: bool = False, limiter="vanleer", quilt: Quilt | None = None,
                 device="cuda", init_floor: bool = True, precision: str = "fp64"):
        self.mtr = Metric(M, a, Q)
        self.stt = State(gm)
        self.precision = precision
        self.limiter = _LIMITERS[limiter] if isinstance(limiter, str) else int(limiter)
        self.quilt = quilt if quilt is not None else Quilt(dom_l, dom_h, nqlt, periodic)
        self.device = torch.device(device)
        self._alloc()
        if init_floor:
            self._init_floor()

    # ------------------------------------------------------------------
    def _alloc(self):
        n = len(self.quilt)
        d, f64 = self.device, torch.float64
        self.U = torch.zeros((n, 8, NC), dtype=f64, device=d)
        self.W = torch.zeros((n, 8, NC), dtype=f64, device=d)
        self.dU = torch.zeros((n, 8, NC), dtype=f64, device=d)
        self.F = torch.zeros((n, 3, 8, NF), dtype=f64, device=d)
        self.Bf = torch.zeros((n, 3, NF), dtype=f64, device=d)
        self.EMF = torch.zeros((n, 3, NE), dtype=f64, device=d)
        # derived fields (lor, p, h, b2) of the primitives floors and regrid leave
        self.Wd = torch.zeros((n, 4, NC), dtype=f64, device=d)
        self.err = torch.zeros(1, dtype=torch.int32, device=d)
        self.dt = torch.zeros(1, dtype=f64, device=d)
        self._bind()

    def _bind(self):
        """Per-patch tables, scratch and the bh_pool of the current quilt and
        state arrays; cell geometry (patch::cell_init)."""
        T = self.quilt.tables()
        self.tables = T
        n = len(T["lvl"])
        self.npatch = n
        d, f64 = self.device, torch.float64
        self.rth = torch.zeros((n, 2, NC), dtype=f64, device=d)
        self.pgeo = torch.as_tensor(T["pgeo"], device=d)
        self.nbr = torch.as_tensor(T["nbr"], device=d)
        self.lvl = torch.as_tensor(T["lvl"], device=d)
        self.all = torch.arange(n, dtype=torch.int32, device=d)
        leaves = np.nonzero(T["leaf"])[0].astype(np.int32)
        self.leaves = torch.as_tensor(leaves, device=d)
        self.leafmask = torch.as_tensor(np.ascontiguousarray(T["leaf"], np.uint8), device=d)
        # scratch: con2prim outcome of every interior cell in the current stage
        self.status = torch.zeros((n, NC), dtype=torch.uint8, device=d)
        # scratch of the flux computation: per-cell logarithms and metric
        self.aux = torch.zeros((n, 6, NC), dtype=f64, device=d)
        waves = self.quilt.ghost_waves(T["nbr"], T["leaf"])
        self.nwave = len(waves)
        off = np.zeros(self.nwave + 1, np.int32)
        for w, lst in enumerate(waves):
            off[w + 1] = off[w] + len(lst)
        self._wave_off = off
        self.waves = torch.as_tensor(np.concatenate(waves) if waves else np.zeros(0, np.int32), device=d)
        self.pool = BhPool(n, _p(self.U), _p(self.W), _p(self.dU), _p(self.F), _p(self.Bf), _p(self.EMF),
                           _p(self.rth), _p(self.pgeo), _p(self.nbr), _p(self.all), _p(self.leaves),
                           len(leaves), _p(self.err), _p(self.leafmask), _p(self.status), _p(self.aux),
                           _p(self.Wd))
        check(lib.bh_geometry(C.byref(self.pool), _stream()), "patch::cell_init")

    # ---- initial data ----------------------------------------------------
    def torus_init(self, r_max: float | None = None, r_in: float | None = None) -> dict:
        """The initial data of the reference's main() (main.cpp:89-160) on the
        device: floor state, Fishbone-Moncrief torus (init::fm_init,
        initconds.cpp:228-591; the reference fixes r_max = 12 M, r_in = 4.5 M),
        face B from the curl of A_phi (init::B_pot_init, :594-667), U = ptoc(W).
        Returns l0, W_in, ln h at r_max, the torus density maximum before
        normalisation and the interior density maximum; raises where main()
        stops (no density above 1e-14)."""
        M = self.mtr.M
        r_max = 12.0 * M if r_max is None else float(r_max)
        r_in = 4.5 * M if r_in is None else float(r_in)
        out = np.zeros(5)
        P = self.params()
        rc = lib.bh_torus_init(C.byref(P), C.byref(self.pool), r_max, r_in, out.ctypes.data_as(C.c_void_p),
                               _stream())
        if rc == -3:
            raise RuntimeError("Density initialisation threw back an error: rho_max is zero after "
                               "Fishbone-Moncrief torus initialisation attempt!")
        check(rc, "torus initial data")
        return dict(zip(("l0", "W_in", "lnh_max", "rho_max_torus", "rho_max"), out.tolist()))

    # ---- AMR -------------------------------------------------------------
    def regrid(self, check_domain: bool = True, flags=None):
        """amrtree::regrid (grid.cpp:722-835) on the device.

        The refinement test of every leaf patch runs on the GPU
        (bh_regrid_flags); the quilt bookkeeping -- which patches refine or
        flatten and the order of the new quilt -- runs on the host from
        those flags (Quilt.regrid); the pool is extended by the new children
        (zeroed, as the reference value-initialises a new patch), refine
        (bh_refine) and ccrstr (bh_ccrstr) fill them, and the flattened
        children leave the pool.  ``flags`` (per patch, bit 0 refine, bit 1
        erase) replaces the reference's refinement test with the caller's.
        Returns the plan (bhgpu.mesh.RegridPlan)."""
        P = self.params()
        if flags is None:
            fl = torch.zeros(self.npatch, dtype=torch.uint8, device=self.device)
            check(lib.bh_regrid_flags(C.byref(P), C.byref(self.pool), _p(self.lvl), _p(fl), _stream()),
                  "amrtree::regrid")
            flags = fl.cpu().numpy()
        plan = self.quilt.regrid(np.asarray(flags))
        if not plan.changed:
            return plan
        d, grow = self.device, plan.n_ext - plan.n_old

        def ext(t):
            return torch.cat([t, t.new_zeros((grow,) + tuple(t.shape[1:]))]) if grow else t
        U, W, dU, F, Bf, EMF, Wd = (ext(x) for x in (self.U, self.W, self.dU, self.F, self.Bf, self.EMF, self.Wd))
        rth = torch.zeros((plan.n_ext, 2, NC), dtype=torch.float64, device=d)
        pgeo = torch.as_tensor(plan.ext_pgeo, device=d)
        all_ = torch.arange(plan.n_ext, dtype=torch.int32, device=d)
        pool = BhPool(plan.n_ext, _p(U), _p(W), _p(dU), _p(F), _p(Bf), _p(EMF), _p(rth), _p(pgeo), None,
                      _p(all_), None, 0, _p(self.err), None, None, None, _p(Wd))
        s = _stream()
        check(lib.bh_geometry(C.byref(pool), s), "patch::cell_init")
        if plan.refined:
            rows = torch.as_tensor(np.array([[p] + kids for p, kids in plan.refined], np.int32), device=d)
            check(lib.bh_refine(C.byref(P), C.byref(pool), _p(rows), len(plan.refined), s), "amrtree::refine")
        if plan.flattened:
            rows = torch.as_tensor(np.array([[p] + kids for p, kids in plan.flattened], np.int32), device=d)
            check(lib.bh_ccrstr(C.byref(P), C.byref(pool), _p(rows), len(plan.flattened), s), "amrtree::ccrstr")
        keep = torch.as_tensor(plan.keep, device=d)
        self.U, self.W, self.dU, self.F, self.Bf, self.EMF, self.Wd = (
            x.index_select(0, keep).contiguous() for x in (U, W, dU, F, Bf, EMF, Wd))
        self._bind()
        if check_domain:
            self.check()
        return plan

    def params(self, maxiter=500, tol=1e-10) -> BhParams:
        return _params(self.mtr, self.stt, self.limiter, maxiter, tol, self.precision)

    def _init_floor(self):
        """Every cell starts at amrtree::pvfs and its ptoc (grid.cpp:193-205)."""
        r = self.rth[:, 0]
        rf = 1.0 / torch.sqrt(torch.clamp(r, min=1e-10)) ** 3
        self.W.zero_()
        self.W[:, 0] = 1e-7 * rf
        self.W[:, 1] = 1e-5 * rf
        self.prim_to_cons()

    def prim_to_cons(self, cells: torch.Tensor | None = None):
        """U = conserved::ptoc(W) on every cell (all 20^3 incl. ghosts)."""
        n = self.npatch * NC
        W = self.W.permute(1, 0, 2).reshape(8, n).contiguous()
        r = self.rth[:, 0].reshape(-1).contiguous()
        th = self.rth[:, 1].reshape(-1).contiguous()
        U = torch.empty((8, n), dtype=torch.float64, device=self.device)
        P = self.params()
        check(lib.bh_ptoc(C.byref(P), _p(W), _p(r), _p(th), n, _p(U), None, _stream()), "conserved::ptoc")
        self.U.copy_(U.reshape(8, self.npatch, NC).permute(1, 0, 2))

    # ---- error word ----------------------------------------------------
    def read_error(self) -> int:
        return int(self.err.item())

    def clear_error(self):
        self.err.zero_()

    def check(self):
        e = self.read_error()
        if e & BH_ERR_DOMAIN:
            self.clear_error()
            raise DomainError("Thermodynamic calculations threw back an error: the density is not positive!")

    # ---- patch-level operations (reference names) ------------------------
    def ghosts(self, check_domain=True):
        """amrtree::ghosts (grid.cpp:524-571) on every leaf, wave by wave."""
        P = self.params()
        off = self._wave_off
        for w in range(self.nwave):
            lst = self.waves[off[w]:off[w + 1]]
            check(lib.bh_ghosts(C.byref(P), C.byref(self.pool), _p(lst), int(off[w + 1] - off[w]), _stream()),
                  "amrtree::ghosts")
        if check_domain:
            self.check()

    def prims(self, check_domain=True):
        """ctop on every cell of every leaf with floor fallback (integrator.cpp:288-310)."""
        P = self.params()
        check(lib.bh_prims(C.byref(P), C.byref(self.pool), _stream()), "rkstg reconstruction")
        if check_domain:
            self.check()

    def fluxcomp(self, check_domain=True):
        """patch::fluxcomp (grid.cpp:255-329) on every patch."""
        P = self.params()
        check(lib.bh_fluxcomp(C.byref(P), C.byref(self.pool), _stream()), "patch::fluxcomp")
        if check_domain:
            self.check()

    def reconfp(self, dim: int, limiter=None):
        """reconfp (reconstruction.cpp:40-97) at all flux faces of direction
        dim: (L, R), each [8][npatch*4352] in fluxcomp's loop order."""
        lim = self.limiter if limiter is None else (_LIMITERS[limiter] if isinstance(limiter, str) else limiter)
        n = self.npatch * 17 * 16 * 16
        L = torch.empty((8, n), dtype=torch.float64, device=self.device)
        R = torch.empty((8, n), dtype=torch.float64, device=self.device)
        P = self.params()
        check(lib.bh_reconfp(C.byref(P), C.byref(self.pool), dim, lim, _p(L), _p(R), _stream()), "reconfp")
        return L, R

    def emfcomp(self):
        """constrans::emfcomp (transport.cpp:11-36)."""
        check(lib.bh_emfcomp(C.byref(self.pool), _stream()), "constrans::emfcomp")

    def bfupdate(self, dt):
        """constrans::Bfupdate (transport.cpp:38-58); dt a float or a device scalar."""
        dtd = self._dt_tensor(dt)
        check(lib.bh_bfupdate(C.byref(self.pool), _p(dtd), _stream()), "constrans::Bfupdate")

    def f2cb(self):
        """constrans::f2cB (transport.cpp:60-75)."""
        P = self.params()
        check(lib.bh_f2cb(C.byref(P), C.byref(self.pool), _stream()), "constrans::f2cB")

    def maxdivb(self) -> torch.Tensor:
        """constrans::maxdivB (transport.cpp:77-89) per patch."""
        out = torch.empty(self.npatch, dtype=torch.float64, device=self.device)
        check(lib.bh_maxdivb(C.byref(self.pool), _p(out), _stream()), "constrans::maxdivB")
        return out

    def floors(self, check_domain=True):
        """patch::floors (grid.cpp:331-358) on every patch."""
        P = self.params()
        check(lib.bh_floors(C.byref(P), C.byref(self.pool), _stream()), "patch::floors")
        if check_domain:
            self.check()

    def div_source(self):
        """rk2integrator::div_flux and ::source at every interior cell."""
        dv = torch.zeros_like(self.U)
        sv = torch.zeros_like(self.U)
        P = self.params()
        check(lib.bh_div_source(C.byref(P), C.byref(self.pool), _p(dv), _p(sv), _stream()),
              "rk2integrator::div_flux/source")
        return dv, sv

    def update(self, dt, stage: int):
        """f2cB + conserved update of rkstg (integrator.cpp:325-347)."""
        P = self.params()
        check(lib.bh_update(C.byref(P), C.byref(self.pool), _p(self._dt_tensor(dt)), int(stage), _stream()),
              "rkstg update")

    def _dt_tensor(self, dt) -> torch.Tensor:
        if isinstance(dt, torch.Tensor):
            return dt.reshape(1).to(device=self.device, dtype=torch.float64).contiguous()
        t = torch.empty(1, dtype=torch.float64, device=self.device)
        t.fill_(float(dt))
        return t

    # ---- state exchange --------------------------------------------------
    def load(self, U=None, W=None, Bf=None, dU=None, Wd=None):
        for name, x in (("U", U), ("W", W), ("Bf", Bf), ("dU", dU), ("Wd", Wd)):
            if x is not None:
                getattr(self, name).copy_(torch.as_tensor(np.asarray(x), dtype=torch.float64))

    def data_write(self, path: str, t: float = 0.0, step: int = 0, derived: bool = False):
        """Grid data for the renderer (the reference's data_write switch,
        main.cpp:40-43, whose writer data.hpp never defines): the leaf
        patches' interior primitives and geometry in one snapshot file
        (bhgpu.snapshot)."""
        from . import snapshot
        snapshot.from_tree(self, path, t=t, step=step, derived=derived)

    def host(self, names=("U", "W", "Bf")):
        return {k: getattr(self, k).cpu().numpy() for k in names}


class RK2Integrator:
    """integ::rk2integrator (rk2.hpp:17-30): Heun RK2 with CFL number cfl."""

    def __init__(self, cfl: float = 0.4):
        self.cfl = float(cfl)

    @staticmethod
    def dtcomp(tree: AmrTree, cfl: float, check_domain=True) -> torch.Tensor:
        """rk2integrator::dtcomp (integrator.cpp:156-189) -> device scalar."""
        P = tree.params()
        check(lib.bh_dtcomp(C.byref(P), C.byref(tree.pool), float(cfl), _p(tree.dt), _stream()),
              "rk2integrator::dtcomp")
        if check_domain:
            tree.check()
        return tree.dt

    @staticmethod
    def div_flux_source(tree: AmrTree):
        return tree.div_source()

    def rkstg(self, tree: AmrTree, dt, stg: int, check_domain=True):
        """rk2integrator::rkstg (integrator.cpp:191-260)."""
        P = tree.params()
        dtd = tree._dt_tensor(dt)
        off = tree._wave_off
        offp = off.ctypes.data_as(C.c_void_p)
        check(lib.bh_rkstg(C.byref(P), C.byref(tree.pool), _p(dtd), int(stg), _p(tree.waves), offp,
                           tree.nwave, _stream()), "rk2integrator::rkstg")
        if check_domain:
            tree.check()

    def step(self, tree: AmrTree, sync: bool = True, check_domain: bool = True):
        """rk2integrator::step (integrator.cpp:262-275): dtcomp, two stages,
        floors.  Returns dt (a float if sync, else the device scalar)."""
        P = tree.params()
        off = tree._wave_off
        check(lib.bh_step(C.byref(P), C.byref(tree.pool), self.cfl, _p(tree.dt), _p(tree.waves),
                          off.ctypes.data_as(C.c_void_p), tree.nwave, _stream()), "rk2integrator::step")
        if check_domain:
            tree.check()
        return float(tree.dt.item()) if sync else tree.dt


class StepGraph:
    """rk2integrator::step recorded once into a CUDA graph and replayed.

    The step's 21 launches (dtcomp, two stages, floors) read dt from device
    memory and never synchronise with the host, so the whole step is one
    graph; ``before`` (optional) is recorded in front of it, e.g. a copy
    that resets the state.  Replays run on the current stream.  The domain
    error word is left to the caller (``tree.check()``).
    """

    def __init__(self, tree: AmrTree, integrator: RK2Integrator, before=None, warmup: int = 1):
        self.tree, self.integrator, self.before = tree, integrator, before
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self._body()
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()

    def _body(self):
        if self.before is not None:
            self.before()
        self.integrator.step(self.tree, sync=False, check_domain=False)

    def replay(self):
        self.graph.replay()
        return self.tree.dt
