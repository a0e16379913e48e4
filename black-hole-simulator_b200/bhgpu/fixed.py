"""The corrected ("fixed") scheme: Valencia GRMHD in Cartesian Kerr-Schild.

The reference's own scheme (``src/fluid``) stops in the first step of a Kerr
torus (``physics/thermo.cpp:10-11`` reached from ``conserved.cpp:205``); this
mode keeps its structure -- ``rk2integrator::step`` = dt, two RK stages of
con2prim, ghost fill, face fluxes, constrained transport and update
(``solver/integrator.cpp:191-275``) -- with the defects corrected (listed in
``csrc/bh_fixed_phys.cuh``).  Host side only: the block table, the
27-neighbour table and the work lists are built here in numpy; the device
buffers are torch tensors; every computation runs in ``libbhgpu.so``.

Layout (``include/bhgpu.h``, bh_fx_grid): cubic blocks of n^3 interior cells,
each stored per array as an (n+7)^3 box (cells -3 .. n+3 per axis).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from bhgrid.blocks import (BLOCK_DTYPE, CHUNK, TILE_MIN, box_size, flux_items, ghost_depth,  # noqa: F401
                           interior as _interior, leveled_blocks, uniform_blocks, work_items)

from ._lib import BH_FP64, BH_FP64_FMA, BH_MIXED, BH_MC, BH_MINMOD, BH_PPM, BH_VANLEER, BhError, check, lib

_vp, _d, _i32, _i64 = C.c_void_p, C.c_double, C.c_int32, C.c_int64
GHOST = 2
QSLOTS = 7           # BH_FX_QSLOTS
PRECISIONS = {"fp64": BH_FP64, "fp64-fma": BH_FP64_FMA, "mixed": BH_MIXED}
LIMITERS = {"minmod": BH_MINMOD, "vanleer": BH_VANLEER, "mc": BH_MC, "ppm": BH_PPM}


class BhFxParams(C.Structure):
    _fields_ = [("M", _d), ("a", _d), ("gamma", _d), ("cfl", _d), ("rho_floor", _d), ("u_floor", _d),
                ("sigma_max", _d), ("W_max", _d), ("r_exc", _d), ("tol", _d), ("maxiter", _i32),
                ("limiter", _i32), ("precision", _i32), ("flags", _i32)]


class BhFxGrid(C.Structure):
    _fields_ = [("nblock", _i32), ("blocks", _vp), ("nbr", _vp), ("items_cell", _vp), ("nitem_cell", _i32),
                ("items_pos", _vp), ("nitem_pos", _i32), ("items_ghost", _vp), ("nitem_ghost", _i32),
                ("ncell", _i64), ("U", _vp), ("U1", _vp), ("W", _vp), ("Bf", _vp), ("Bf1", _vp), ("F", _vp),
                ("dt", _vp), ("count", _vp), ("err", _vp), ("E", _vp), ("maxlevel", _i32), ("queue_ctas", _i32), ("queue", _vp),
                ("items_flux", _vp), ("nitem_flux", _i32), ("ghost_depth", _i32)]


class BhFxTorus(C.Structure):
    _fields_ = [("r_in", _d), ("r_max", _d), ("kappa", _d), ("beta", _d), ("noise", _d), ("seed", C.c_uint64)]


_sig = {
    "bh_fx_step": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _vp],
    "bh_fx_prims": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _i32, _i32, _vp],
    "bh_fx_ghosts": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _i32, _vp],
    "bh_fx_fluxes": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _i32, _vp],
    "bh_fx_update": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _i32, _vp],
    "bh_fx_pack_state": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _vp, _vp, _i32, _vp],
    "bh_fx_ghost_pass": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _i32, _i32, _vp],
    "bh_fx_emf": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _vp],
    "bh_fx_update_from_emf": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _i32, _vp],
    "bh_fx_divb": [C.POINTER(BhFxGrid), _vp, _vp],
    "bh_fx_torus_init": [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), C.POINTER(BhFxTorus), _vp, _vp, _vp],
}
for _name, _args in _sig.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = C.c_int


def horizon_radius(M: float, a: float) -> float:
    return M + math.sqrt(M * M - a * a)


@dataclass
class FxParams:
    """Physics and numerics of the corrected scheme (bh_fx_params).

    The default floors are the Kerr torus configuration's atmosphere.  With
    them the 128^3 torus runs cleanly for ~350 steps; after that a
    floor-density cell above the torus reaches the W_max cap and the run
    (FP64 as well as mixed) loses con2prim in a growing number of cells.
    For longer runs rho_floor=1e-5, u_floor=1e-7 kept 800 steps free of
    con2prim failures with W <= 1.5, as did W_max = 10 or 20."""
    M: float = 1.0
    a: float = 0.9375
    gamma: float = 4.0 / 3.0
    cfl: float = 0.4
    rho_floor: float = 1e-6        # rho >= rho_floor r^-3/2
    u_floor: float = 1e-8          # p / (Gamma - 1) >= u_floor r^-5/2
    sigma_max: float = 100.0
    W_max: float = 50.0
    r_exc: float | None = None     # default: 1.2 r_H
    tol: float = 1e-12
    maxiter: int = 30
    limiter: str = "mc"           # monotonized central: no division per slope
    precision: str = "fp64"
    c2p_fp64: bool = False        # mixed: every cell's con2prim ends with FP64 Newton iterations

    def cstruct(self) -> BhFxParams:
        r_exc = self.r_exc if self.r_exc is not None else (
            1.2 * horizon_radius(self.M, self.a) if self.M > 0 else 0.0)
        return BhFxParams(self.M, self.a, self.gamma, self.cfl, self.rho_floor, self.u_floor, self.sigma_max,
                          self.W_max, r_exc, self.tol, self.maxiter, LIMITERS[self.limiter],
                          PRECISIONS[self.precision], 1 if self.c2p_fp64 else 0)


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class FxGrid:
    """Device buffers of the corrected scheme on a list of blocks.

    ``FxGrid.uniform(lo, hi, N, block)`` builds the uniform N^3 grid over
    [lo, hi]^3; ``block`` = N gives one block (no interior ghost exchange).
    """

    def __init__(self, blocks: np.ndarray, nbr: np.ndarray, params: FxParams, device="cuda", emf_arrays=None,
                 persistent=False, nactive=None, maxlevel=None, tile_min=TILE_MIN):
        """emf_arrays: keep the edge EMFs in arrays (required, and the
        default, when blocks have different levels; otherwise they are
        computed on the fly by the update).  persistent: launch the step
        kernels as persistent CTAs fed by a device work queue.  nactive:
        the kernels work on blocks[:nactive] only (the rest are neighbours'
        copies, as in a sharded grid); maxlevel: the highest level of the
        whole domain (default: of these blocks); tile_min: the smallest
        block the staged flux kernel tiles."""
        self.params = params
        self.blocks_np = blocks
        self.nbr_np = nbr
        self.device = torch.device(device)
        self.ncell = int(sum(box_size(int(n)) for n in blocks["n"]))
        dev = self.device
        self.blocks = torch.from_numpy(blocks.view(np.uint8).copy()).to(dev)
        self.nbr = torch.from_numpy(nbr.copy()).to(dev)
        self.ghost_depth = ghost_depth(params.limiter)
        self.nactive = len(blocks) if nactive is None else int(nactive)
        act = blocks[:self.nactive]
        self.items = {k: torch.from_numpy(work_items(act, k, self.ghost_depth)).to(dev)
                      for k in ("cell", "pos", "ghost")}
        self.items["flux"] = torch.from_numpy(flux_items(act, tile_min)).to(dev)
        wdt = torch.float32 if params.precision == "mixed" else torch.float64
        N = self.ncell
        self.U = torch.zeros((8, N), dtype=torch.float64, device=dev)
        self.U1 = torch.zeros_like(self.U)
        self.W = torch.zeros((8, N), dtype=wdt, device=dev)
        self.Bf = torch.zeros((3, N), dtype=torch.float64, device=dev)
        self.Bf1 = torch.zeros_like(self.Bf)
        self.F = torch.zeros((3, 8, N), dtype=wdt, device=dev)
        self.dt = torch.zeros(2, dtype=torch.float64, device=dev)
        self.count = torch.zeros(4, dtype=torch.int32, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.scratch = torch.zeros(4, dtype=torch.float64, device=dev)
        self.maxlevel = int(blocks["level"].max()) if maxlevel is None else int(maxlevel)
        if emf_arrays is None:
            emf_arrays = self.maxlevel > 0
        self.E = torch.zeros((3, N), dtype=torch.float64, device=dev) if emf_arrays else None
        self.queue = torch.zeros(2 * QSLOTS, dtype=torch.int32, device=dev) if persistent else None
        self._refresh()

    @classmethod
    def uniform(cls, lo: float, hi: float, N: int, block: int, params: FxParams, periodic=False, device="cuda",
                emf_arrays=None, persistent=False):
        blocks, nbr = uniform_blocks(lo, hi, N, block, periodic)
        return cls(blocks, nbr, params, device, emf_arrays, persistent)

    @classmethod
    def leveled(cls, lo: float, hi: float, level: np.ndarray, n0: int, params: FxParams, device="cuda",
                persistent=False, tile_min=TILE_MIN):
        """Equal cubes over [lo, hi]^3 with per-cube levels (n0 2^level cells
        per axis), e.g. bhgrid.blocks.torus_levels()."""
        blocks, nbr = leveled_blocks(lo, hi, level, n0)
        return cls(blocks, nbr, params, device, persistent=persistent, tile_min=tile_min)

    def _refresh(self):
        it = self.items
        self._g = BhFxGrid(self.nactive, _ptr(self.blocks), _ptr(self.nbr),
                           _ptr(it["cell"]), it["cell"].shape[0], _ptr(it["pos"]), it["pos"].shape[0],
                           _ptr(it["ghost"]), it["ghost"].shape[0], self.ncell,
                           _ptr(self.U), _ptr(self.U1), _ptr(self.W), _ptr(self.Bf), _ptr(self.Bf1), _ptr(self.F),
                           _ptr(self.dt), _ptr(self.count), _ptr(self.err), _ptr(self.E), self.maxlevel, 0, _ptr(self.queue),
                           _ptr(it["flux"]), it["flux"].shape[0], self.ghost_depth)
        self._p = self.params.cstruct()

    @property
    def precision(self):
        return self.params.precision

    @property
    def zones(self) -> int:
        return int(sum(int(n) ** 3 for n in self.blocks_np["n"]))

    # ---- the step (rk2integrator::step, solver/integrator.cpp:262-275) ----
    def step(self):
        check(lib.bh_fx_step(C.byref(self._p), C.byref(self._g), _stream()), "bh_fx_step")

    def prims(self, stage=0, with_dt=False):
        check(lib.bh_fx_prims(C.byref(self._p), C.byref(self._g), stage, int(with_dt), _stream()), "bh_fx_prims")

    def ghosts(self, stage=0):
        check(lib.bh_fx_ghosts(C.byref(self._p), C.byref(self._g), stage, _stream()), "bh_fx_ghosts")

    # ---- the state a step reads, packed (bh_fx_pack_state) ----
    def state_nbytes(self) -> int:
        """bytes of the packed state: rows 0-4 of U and W, the blocks' own
        face field"""
        q = self.items["cell"].shape[0] * CHUNK
        nb = self.blocks_np["n"][:self.nactive].astype(np.int64)
        return int(q * (5 * 8 + 5 * self.W.element_size() + 3 * 8) + 8 * 3 * int((nb * nb).sum()))

    def _face_off(self):
        if getattr(self, "_foff", None) is None:
            nb = self.blocks_np["n"][:self.nactive].astype(np.int64)
            off = np.concatenate([[0], np.cumsum(3 * nb * nb)[:-1]]).astype(np.int64)
            self._foff = torch.from_numpy(off).to(self.device)
        return self._foff

    def pack_state(self, buf: torch.Tensor):
        """the state into the device buffer buf (uint8, state_nbytes())"""
        check(lib.bh_fx_pack_state(C.byref(self._p), C.byref(self._g), _ptr(self._face_off()), _ptr(buf), 0,
                                   _stream()), "bh_fx_pack_state")

    def unpack_state(self, buf: torch.Tensor):
        """the grid's U, W rows 0-4 and face field from a packed state"""
        check(lib.bh_fx_pack_state(C.byref(self._p), C.byref(self._g), _ptr(self._face_off()), _ptr(buf), 1,
                                   _stream()), "bh_fx_pack_state")

    def ghost_pass(self, stage, pass_):
        check(lib.bh_fx_ghost_pass(C.byref(self._p), C.byref(self._g), stage, pass_, _stream()), "bh_fx_ghost_pass")

    def emf_raw(self):
        """the edge EMFs of the grid's own blocks into E, uncorrected"""
        check(lib.bh_fx_emf(C.byref(self._p), C.byref(self._g), _stream()), "bh_fx_emf")

    def update_from_emf(self, stage=0):
        check(lib.bh_fx_update_from_emf(C.byref(self._p), C.byref(self._g), stage, _stream()),
              "bh_fx_update_from_emf")

    def fluxes(self, stage=0):
        check(lib.bh_fx_fluxes(C.byref(self._p), C.byref(self._g), stage, _stream()), "bh_fx_fluxes")

    def update(self, stage=0):
        check(lib.bh_fx_update(C.byref(self._p), C.byref(self._g), stage, _stream()), "bh_fx_update")

    def time_step(self) -> float:
        """dt of the last step (device value, synchronises)."""
        return float(self.dt[1].item())

    def divb(self) -> float:
        """max over interior cells of |div B~| / max|B~| of the cell's faces."""
        out = torch.zeros(len(self.blocks_np), dtype=torch.float64, device=self.device)
        check(lib.bh_fx_divb(C.byref(self._g), _ptr(out), _stream()), "bh_fx_divb")
        return float(out.max().item())

    def torus_init(self, r_in=6.0, r_max=12.0, kappa=1e-3, beta=100.0, noise=0.04, seed=1):
        T = BhFxTorus(r_in, r_max, kappa, beta, noise, seed)
        out = (C.c_double * 4)()
        check(lib.bh_fx_torus_init(C.byref(self._p), C.byref(self._g), C.byref(T), _ptr(self.scratch), out,
                                   _stream()), "bh_fx_torus_init")
        return {"ell": out[0], "rho_max_raw": out[1], "field_scale": out[2], "beta": out[3]}

    # ---- host views ----------------------------------------------------
    def interior(self, arr: torch.Tensor) -> np.ndarray:
        """[..., nblock, n, n, n] interior cells of a [..., ncell] array (numpy,
        float64); all blocks must have the same n."""
        return _interior(self.blocks_np, arr.detach().double().cpu().numpy())

    def counters(self) -> dict:
        c = self.count.cpu().numpy()
        return {"c2p_failures": int(c[0]), "floored": int(c[1]), "c2p_fp64_fallback": int(c[2])}

    def reset_counters(self):
        self.count.zero_()

    def copy_state_from(self, other: "FxGrid"):
        """U, W (cast), Bf of another grid with the same blocks."""
        self.U.copy_(other.U)
        self.W.copy_(other.W.to(self.W.dtype))
        self.Bf.copy_(other.Bf)

    # ---- the step as one CUDA graph -----------------------------------------
    def capture(self):
        """Record one step (9 launches) as a CUDA graph on a side stream
        (bh_fx_graph_create); ``replay()`` then runs a step with one launch
        of the graph.  The grid's buffers must not be reallocated while the
        graph lives."""
        self.release_graph()
        s = torch.cuda.Stream(self.device)
        h = C.c_void_p()
        check(lib.bh_fx_graph_create(C.byref(self._p), C.byref(self._g), C.c_void_p(s.cuda_stream), C.byref(h)),
              "bh_fx_graph_create")
        self._graph = h

    def replay(self):
        check(lib.bh_step_graph_replay(self._graph, _stream()), "bh_step_graph_replay")

    def release_graph(self):
        if getattr(self, "_graph", None):
            lib.bh_step_graph_destroy(self._graph)
        self._graph = None

    def __del__(self):
        try:
            self.release_graph()
        except Exception:
            pass


lib.bh_fx_graph_create.argtypes = [C.POINTER(BhFxParams), C.POINTER(BhFxGrid), _vp, C.POINTER(_vp)]
lib.bh_fx_graph_create.restype = C.c_int
lib.bh_step_graph_replay.argtypes = [_vp, _vp]
lib.bh_step_graph_replay.restype = C.c_int
lib.bh_step_graph_destroy.argtypes = [_vp]
lib.bh_step_graph_destroy.restype = C.c_int


class FxHostPipeline:
    """Host-resident torus states stepped through the GPU, copies overlapped.

    A state is what a step reads: the conserved fluid variables (rows 0-4 of
    U), the previous primitives (rows 0-4 of W: con2prim's starting point)
    and the face field Bf, pinned host tensors in the grid layout (U and W
    may carry all 8 rows; only rows 0-4 move).  The cell-centred field (rows
    5-7 of U and W) is recomputed on the device from the face field by the
    step's con2prim, so it is neither uploaded nor downloaded.  Each
    ``submit`` uploads a state into one of the pipeline's device grids on a
    copy stream, advances it ``steps`` RK2 steps on a compute stream and
    downloads it on a second copy stream; consecutive submissions use
    different grids, so the upload of one state, the step of the previous one
    and the download of the one before overlap.  Each result is bit-identical
    to stepping the state alone.  The returned event marks the end of the
    download.
    """

    def __init__(self, grids: list[FxGrid], steps: int = 1):
        if not grids:
            raise ValueError("FxHostPipeline needs at least one device grid")
        if any(g.ncell != grids[0].ncell or g.precision != grids[0].precision for g in grids):
            raise ValueError("the grids of a pipeline must share one layout and variant")
        self.grids, self.steps = list(grids), int(steps)
        dev = grids[0].device
        self.s_in, self.s_run, self.s_out = (torch.cuda.Stream(dev) for _ in range(3))
        self._freed: list[torch.cuda.Event | None] = [None] * len(self.grids)
        self._k = 0
        self._bufs = None

    def submit_packed(self, state_in: torch.Tensor, state_out: torch.Tensor) -> torch.cuda.Event:
        """As submit, for a state packed by FxGrid.pack_state (pinned uint8
        host tensors of state_nbytes()): only the interior cells' values and
        the blocks' own faces cross the host link, unpacked and packed on the
        device by bh_fx_pack_state."""
        if self._bufs is None:
            n = self.grids[0].state_nbytes()
            self._bufs = [torch.empty(n, dtype=torch.uint8, device=g.device) for g in self.grids]
        slot = self._k % len(self.grids)
        self._k += 1
        g, buf = self.grids[slot], self._bufs[slot]
        with torch.cuda.stream(self.s_in):
            if self._freed[slot] is not None:
                self.s_in.wait_event(self._freed[slot])
            buf.copy_(state_in, non_blocking=True)
            loaded = torch.cuda.Event()
            loaded.record(self.s_in)
        with torch.cuda.stream(self.s_run):
            self.s_run.wait_event(loaded)
            g.unpack_state(buf)
            for _ in range(self.steps):
                g.step()
            g.pack_state(buf)
            done = torch.cuda.Event()
            done.record(self.s_run)
        with torch.cuda.stream(self.s_out):
            self.s_out.wait_event(done)
            state_out.copy_(buf, non_blocking=True)
            freed = torch.cuda.Event()
            freed.record(self.s_out)
        self._freed[slot] = freed
        return freed

    def submit(self, U, W, Bf, out_U, out_W, out_Bf) -> torch.cuda.Event:
        slot = self._k % len(self.grids)
        self._k += 1
        g = self.grids[slot]
        with torch.cuda.stream(self.s_in):
            if self._freed[slot] is not None:
                self.s_in.wait_event(self._freed[slot])
            g.U[:5].copy_(U[:5], non_blocking=True)
            g.W[:5].copy_(W[:5], non_blocking=True)
            g.Bf.copy_(Bf, non_blocking=True)
            loaded = torch.cuda.Event()
            loaded.record(self.s_in)
        with torch.cuda.stream(self.s_run):
            self.s_run.wait_event(loaded)
            for _ in range(self.steps):
                g.step()
            done = torch.cuda.Event()
            done.record(self.s_run)
        with torch.cuda.stream(self.s_out):
            self.s_out.wait_event(done)
            out_U[:5].copy_(g.U[:5], non_blocking=True)
            out_W[:5].copy_(g.W[:5], non_blocking=True)
            out_Bf.copy_(g.Bf, non_blocking=True)
            freed = torch.cuda.Event()
            freed.record(self.s_out)
        self._freed[slot] = freed
        return freed

    def synchronize(self):
        for e in self._freed:
            if e is not None:
                e.synchronize()


# ---------------------------------------------------------------------------
# launch-bound autotuning of the scheme's heavy kernels (bh_fx_tune_*)
TUNE_KERNELS = ("c2p", "flux", "update")
TUNE_KNOBS = TUNE_KERNELS + ("stage", "split")   # 1 = the staged flux kernel; the update as two kernels
TUNE_CANDIDATES = (1, 3, 4, 5, 6, 7, 8)
lib.bh_fx_tune_set.argtypes = [_i32, _i32, _i32]
lib.bh_fx_tune_get.argtypes = [_i32, _i32, C.POINTER(_i32)]
lib.bh_fx_tune_set.restype = C.c_int
lib.bh_fx_tune_get.restype = C.c_int


def tune_set(precision: str, kernel: str, ctas: int):
    """kernel in TUNE_KERNELS: resident CTAs per SM (1, 3..8); "stage", "split": 0/1."""
    check(lib.bh_fx_tune_set(PRECISIONS[precision], TUNE_KNOBS.index(kernel), ctas), "bh_fx_tune_set")


def tune_get(precision: str, kernel: str) -> int:
    v = _i32()
    check(lib.bh_fx_tune_get(PRECISIONS[precision], TUNE_KNOBS.index(kernel), C.byref(v)), "bh_fx_tune_get")
    return int(v.value)


def autotune(grid: FxGrid, reps: int = 4, candidates=TUNE_CANDIDATES) -> dict:
    """Choose the launch bounds of con2prim, fluxes and update, and whether
    the flux stencil is staged in shared memory, for the grid's variant: for
    one kernel at a time (the others held), every candidate times `reps` RK2
    steps (CUDA events) from the same saved state; the fastest is kept (the
    flux candidates are the pairs (staged, launch bound), the update's the
    pairs (split in two kernels, launch bound); staging is tried only where
    the grid has blocks of TILE_MIN cells per axis or more).  The
    grid's state is restored.  In the FP64 variant every choice gives the
    same bits (no contraction); in the contracted variants ptxas may pair
    multiply-adds differently under another register budget, which moves
    results by ulps.  Returns {"choice": {knob: value}, "ms": {kernel:
    {candidate: ms per step}}} (flux and update candidates keyed
    "s<stage or split>/<ctas>")."""
    saved = [t.clone() for t in (grid.U, grid.W, grid.Bf)]
    prec = grid.precision
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"choice": {}, "ms": {}}
    tiled = bool((grid.blocks_np["n"] >= TILE_MIN).any())

    def timed(set_fn):
        set_fn()
        for t, s in zip((grid.U, grid.W, grid.Bf), saved):
            t.copy_(s)
        grid.step()
        torch.cuda.synchronize()
        a.record()
        for _ in range(reps):
            grid.step()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    for k in TUNE_KERNELS:
        times = {}
        if k in ("flux", "update"):
            knob = "stage" if k == "flux" else "split"
            for st in ((0, 1) if (tiled or k == "update") else (0,)):
                for c in candidates:
                    times[f"s{st}/{c}"] = timed(lambda: (tune_set(prec, knob, st), tune_set(prec, k, c)))
            best = min(times, key=times.get)
            st, c = best[1:].split("/")
            tune_set(prec, knob, int(st))
            tune_set(prec, k, int(c))
            out["choice"][knob] = int(st)
            out["choice"][k] = int(c)
        else:
            for c in candidates:
                times[c] = timed(lambda: tune_set(prec, k, c))
            best = min(times, key=times.get)
            tune_set(prec, k, best)
            out["choice"][k] = best
        out["ms"][k] = times
    for t, s in zip((grid.U, grid.W, grid.Bf), saved):
        t.copy_(s)
    grid.reset_counters()
    return out
