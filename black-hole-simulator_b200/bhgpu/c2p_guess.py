"""The learned con2prim initial guess (bh_mlp.cu, bh_ctop_guess).

conserved::ctop (conserved.cpp:135-285) starts Newton at the midpoint of
its bracket.  C2PGuess trains a 6 -> 64 -> 64 -> 2 network on the GPU, with
the library's own forward/backward/Adam kernels, on (conserved state, xi)
pairs the solver's FP64 con2prim produces, and then starts Newton at the
network's xi where that lies inside the bracket.  Newton, the Brent
fallback and the acceptance tests stay the reference's: the guess changes
the iteration count, not what is accepted.  Features: log D, asinh(tau/D),
log(1 + S^2/D^2), log(1 + B^2/D), asinh(S.B/D^1.5), log r (the preamble's
quantities); outputs log(xi/D) and log W.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import BhParams, check, lib
from .solver import Conserved, _dev, _p, _params, _stream

NI, NH, NO = 6, 64, 2
NPARAM = NH * NI + NH + NH * NH + NH + NO * NH + NO   # 4738
ONORM = NPARAM


class BhMlp(C.Structure):
    _fields_ = [("w", C.c_void_p), ("wb", C.c_void_p), ("adam_m", C.c_void_p), ("adam_v", C.c_void_p),
                ("step", C.c_int64)]


def _sig():
    vp, i64 = C.c_void_p, C.c_int64
    P = C.POINTER(BhParams)
    lib.bh_ctop_pre.argtypes = [P, vp, vp, vp, i64, vp, vp]
    lib.bh_ctop_guess.argtypes = [P, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp]
    lib.bh_mlp_guess.argtypes = [C.POINTER(BhMlp), vp, vp, i64, vp, vp]
    lib.bh_mlp_train_step.argtypes = [C.POINTER(BhMlp), vp, vp, vp, i64, C.c_float, vp, vp, vp]
    lib.bh_mlp_sync_bf16.argtypes = [C.POINTER(BhMlp), vp]
    lib.bh_ctop_learned.argtypes = [P, C.POINTER(BhMlp), vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.bh_wait_selftest.argtypes = [vp, vp]
    for f in ("bh_ctop_pre", "bh_ctop_guess", "bh_mlp_guess", "bh_mlp_train_step", "bh_mlp_sync_bf16",
              "bh_ctop_learned", "bh_wait_selftest"):
        getattr(lib, f).restype = C.c_int


_sig()


def wait_selftest() -> int:
    """Run the tensor-core kernels' bounded wait on an mbarrier nothing
    arrives on; returns the device error word it leaves (BH_ERR_TIMEOUT = 2)."""
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    check(lib.bh_wait_selftest(_p(err), _stream()), "bh_wait_selftest")
    return int(err.item())


class C2PGuess:
    def __init__(self, cn: Conserved, seed: int = 0, device="cuda"):
        self.cn = cn
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        w = np.zeros(NPARAM + 2 * NI, np.float32)
        o = 0
        for shape, scale in (((NH, NI), 1 / np.sqrt(NI)), ((NH,), 0.0), ((NH, NH), 1 / np.sqrt(NH)), ((NH,), 0.0),
                             ((NO, NH), 1 / np.sqrt(NH)), ((NO,), 0.0)):
            k = int(np.prod(shape))
            w[o:o + k] = rng.normal(size=k) * scale
            o += k
        w[ONORM + NI:] = 1.0
        self.w = torch.as_tensor(w, device=self.device)
        self.wb = torch.zeros(NPARAM, dtype=torch.bfloat16, device=self.device)
        self.m = torch.zeros(NPARAM, dtype=torch.float32, device=self.device)
        self.v = torch.zeros(NPARAM, dtype=torch.float32, device=self.device)
        self.s = BhMlp(_p(self.w), _p(self.wb), _p(self.m), _p(self.v), 0)
        check(lib.bh_mlp_sync_bf16(C.byref(self.s), _stream()), "bh_mlp_sync_bf16")

    def _P(self):
        return _params(self.cn.mtr, self.cn.stt)

    def preamble(self, U, r, th) -> torch.Tensor:
        """[5][n] D, tau, Ssq, Bsq, SB of con2prim's preamble."""
        U, r, th = _dev(U, "cuda"), _dev(r, "cuda"), _dev(th, "cuda")
        n = U.shape[1]
        pre = torch.empty((5, n), dtype=torch.float64, device=self.device)
        P = self._P()
        check(lib.bh_ctop_pre(C.byref(P), _p(U), _p(r), _p(th), n, _p(pre), _stream()), "ctop preamble")
        return pre

    @staticmethod
    def features(pre: torch.Tensor, r: torch.Tensor) -> torch.Tensor:
        D, tau, Ssq, Bsq, SB = pre
        return torch.stack([torch.log(D), torch.asinh(tau / D), torch.log1p(Ssq / (D * D)), torch.log1p(Bsq / D),
                            torch.asinh(SB / (D * torch.sqrt(D))), torch.log(r)]).float()

    def train(self, U, r, th, steps: int = 2000, batch: int = 8192, lr: float = 3e-3, seed: int = 0):
        """Train on the cells whose FP64 con2prim succeeds; returns the loss
        history (mean squared error per cell, every 100 steps)."""
        U, r, th = _dev(U, "cuda"), _dev(r, "cuda"), _dev(th, "cuda")
        W, Wd, st, it, pa = self.cn.ctop(U, r, th, check_domain=False)
        pre = self.preamble(U, r, th)
        xi = Wd[2] * W[0] * Wd[3] * Wd[3]
        tgt = torch.stack([torch.log(xi / pre[0]), torch.log(Wd[3])]).float()
        x = self.features(pre, r)
        good = (st == 1) & torch.isfinite(tgt).all(0) & torch.isfinite(x).all(0)
        idx = torch.nonzero(good).flatten()
        xs = x[:, idx]
        self.w[ONORM:ONORM + NI] = xs.mean(1)
        self.w[ONORM + NI:] = 1.0 / (xs.std(1) + 1e-12)
        self.w[NPARAM - NO] = tgt[0, idx].mean()
        self.w[NPARAM - 1] = tgt[1, idx].mean()
        check(lib.bh_mlp_sync_bf16(C.byref(self.s), _stream()), "bh_mlp_sync_bf16")
        g = torch.Generator(device=self.device)
        g.manual_seed(seed)
        nb = min(batch, idx.numel())
        scratch = torch.empty((4 * NH + 9) * nb + NPARAM, dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        hist = []
        for s in range(steps):
            sel = idx[torch.randint(0, idx.numel(), (nb,), generator=g, device=self.device)]
            pb, rb, tb = pre[:, sel].contiguous(), r[sel].contiguous(), tgt[:, sel].contiguous()
            lr_s = lr * 0.5 * (1 + np.cos(np.pi * s / steps)) + 1e-5
            check(lib.bh_mlp_train_step(C.byref(self.s), _p(pb), _p(rb), _p(tb), nb, C.c_float(lr_s), _p(scratch),
                                        _p(loss), _stream()), "bh_mlp_train_step")
            if s % 100 == 0 or s == steps - 1:
                hist.append(float(loss.item()) / nb)
        return hist

    def gradient(self, pre, r, target):
        """The device's loss and gradient (no step) -- for checking against
        the CPU restatement."""
        n = pre.shape[1]
        scratch = torch.empty((4 * NH + 9) * n + NPARAM, dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        check(lib.bh_mlp_train_step(C.byref(self.s), _p(pre), _p(r), _p(target), n, C.c_float(0.0), _p(scratch),
                                    _p(loss), _stream()), "bh_mlp_train_step")
        return float(loss.item()), scratch[-NPARAM:].double().cpu().numpy()

    def guess(self, pre, r) -> torch.Tensor:
        n = pre.shape[1]
        xi0 = torch.empty(n, dtype=torch.float64, device=self.device)
        check(lib.bh_mlp_guess(C.byref(self.s), _p(pre), _p(r), n, _p(xi0), _stream()), "bh_mlp_guess")
        return xi0

    def ctop(self, U, r, th):
        """conserved::ctop started from the network's guess: (W, Wd, status,
        iters, path) as Conserved.ctop."""
        U, r, th = _dev(U, "cuda"), _dev(r, "cuda"), _dev(th, "cuda")
        return self.ctop_from(U, r, th, self.guess(self.preamble(U, r, th), r))

    def ctop_from(self, U, r, th, xi0):
        """conserved::ctop with Newton started from the given xi0 (bh_ctop_guess)."""
        U, r, th, xi0 = _dev(U, "cuda"), _dev(r, "cuda"), _dev(th, "cuda"), _dev(xi0, "cuda")
        n = U.shape[1]
        W = torch.empty((8, n), dtype=torch.float64, device=self.device)
        Wd = torch.empty((5, n), dtype=torch.float64, device=self.device)
        st = torch.empty(n, dtype=torch.int32, device=self.device)
        it = torch.empty(n, dtype=torch.int32, device=self.device)
        pa = torch.empty(n, dtype=torch.int32, device=self.device)
        P = self._P()
        check(lib.bh_ctop_guess(C.byref(P), _p(U), _p(r), _p(th), n, _p(xi0), _p(W), _p(Wd), _p(st), _p(it), _p(pa),
                                _stream()), "ctop with guess")
        return W, Wd, st, it, pa

    def ctop_learned(self, U, r, th, want_xi0: bool = False, err: torch.Tensor | None = None):
        """The same as ctop() with the network on the tensor cores: one
        kernel for the metric, the preamble and the network, one for Newton
        (bh_ctop_learned).  Returns (W, Wd, status, iters, path) and, with
        want_xi0, the starting points.  err: a device int32 word of the
        caller's that the call sets to BH_ERR_TIMEOUT if a tensor-core wait
        ran out, left for the caller to check (the call then does not
        synchronise); without it the call checks its own word and raises."""
        U, r, th = _dev(U, "cuda"), _dev(r, "cuda"), _dev(th, "cuda")
        n = U.shape[1]
        W = torch.empty((8, n), dtype=torch.float64, device=self.device)
        Wd = torch.empty((5, n), dtype=torch.float64, device=self.device)
        st = torch.empty(n, dtype=torch.int32, device=self.device)
        it = torch.empty(n, dtype=torch.int32, device=self.device)
        pa = torch.empty(n, dtype=torch.int32, device=self.device)
        xi0 = torch.empty(n, dtype=torch.float64, device=self.device)
        own = err is None
        if own:
            err = torch.zeros(1, dtype=torch.int32, device=self.device)
        P = self._P()
        check(lib.bh_ctop_learned(C.byref(P), C.byref(self.s), _p(U), _p(r), _p(th), n,
                                  _p(xi0), _p(W), _p(Wd), _p(st), _p(it), _p(pa),
                                  _p(err), _stream()), "ctop with the tensor-core guess")
        if own and int(err.item()) != 0:
            raise RuntimeError(f"bh_ctop_learned: device error word {int(err.item())} (tensor-core wait ran out)")
        out = (W, Wd, st, it, pa)
        return out + (xi0,) if want_xi0 else out
