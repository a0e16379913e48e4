"""The kernels' per-item functions (csrc/bh_items.cuh), compiled for the
host and run in the order the C ABI launches them, equal the oracle bit for
bit.  This pins the kernel logic on a CPU-only host; the GPU tests then
only see the last-bit differences of the device math library."""
import ctypes as C

import numpy as np
import pytest

from helpers import box_case, random_prims, GAMMA
from hostcheck import HostKernels, _d

import oracle
from bhgpu.mesh import Quilt


def eq(a, b):
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("M,a,Q", [(0.0, 0.0, 0.0), (1.0, 0.9375, 0.0), (1.0, 0.9, 0.1)])
def test_physics_items_bitwise(M, a, Q):
    rng = np.random.default_rng(2)
    W, r, th = random_prims(5000, rng)
    orc = oracle.Oracle(M, a, Q, GAMMA)
    hk = HostKernels(M, a, Q, GAMMA, 1)
    n = W.shape[1]
    out = np.zeros((n, 120))
    hk.call("hc_metric", _d(r), _d(th), C.c_int64(n), _d(out))
    assert eq(out, orc.metric(r, th))
    U = np.zeros((8, n)); Wd = np.zeros((4, n))
    hk.call("hc_ptoc", _d(W), _d(r), _d(th), C.c_int64(n), _d(U), _d(Wd))
    Uc, Wdc = orc.ptoc(W, r, th)
    assert eq(U, Uc) and eq(Wd, Wdc)
    Wo = np.zeros((8, n)); Wdo = np.zeros((5, n))
    st = np.zeros(n, np.int32); it = np.zeros(n, np.int32); pa = np.zeros(n, np.int32)
    hk.call("hc_ctop", _d(Uc), _d(r), _d(th), C.c_int64(n), _d(Wo), _d(Wdo), _d(st), _d(it), _d(pa))
    Wc, Wdc5, stc, itc, pac = orc.ctop(Uc, r, th)
    assert eq(st, stc) and eq(it, itc) and eq(pa, pac)
    ok = stc == 1
    assert eq(Wo[:, ok], Wc[:, ok]) and eq(Wdo[:, ok], Wdc5[:, ok])
    WR = W.copy(); WR[0] *= 1.07; WR[2:5] += 0.01
    UR, _ = orc.ptoc(WR, r, th)
    for dim in range(3):
        F = np.zeros((8, n)); cts = np.zeros(n)
        hk.call("hc_hlld", _d(W), _d(WR), _d(Uc), _d(UR), _d(r), _d(th), C.c_int(dim), C.c_int64(n), _d(F), _d(cts))
        Fc, cc, _ = orc.hlld(W, WR, Uc, UR, r, th, dim)
        assert eq(F, Fc) and eq(cts, cc)


CASES = [dict(periodic=True, lim=0, M=0.0, a=0.0, lo=10.0, hi=12.0),
         dict(periodic=False, lim=1, M=0.0, a=0.0, lo=10.0, hi=12.0),
         dict(periodic=True, lim=2, M=1.0, a=0.9375, lo=-6.0, hi=6.0)]


@pytest.mark.parametrize("case", CASES)
def test_kernel_items_bitwise(case):
    q, orc, hp = box_case(2, seed=3, **case)
    hk = HostKernels(case["M"], case["a"], 0.0, GAMMA, case["lim"])
    hh = hp.copy()
    hh.rth[:] = 0
    pool = hk.pool(hh)
    hk.L.hc_geometry(C.byref(pool))
    assert eq(hh.rth, hp.rth)
    lst = np.arange(hp.npatch, dtype=np.int32)
    hk.call("hc_ghosts", C.byref(pool), _d(lst), C.c_int(hp.npatch)); orc.ghosts(hp)
    assert eq(hh.U, hp.U) and eq(hh.W, hp.W)
    hk.call("hc_prims", C.byref(pool), C.c_int(0)); orc.prims(hp)
    assert eq(hh.U, hp.U) and eq(hh.W, hp.W)
    n = hp.npatch * 4352
    for dim in range(3):
        L = np.zeros((8, n)); R = np.zeros((8, n))
        hk.call("hc_reconfp", C.byref(pool), C.c_int(dim), C.c_int(case["lim"]), _d(L), _d(R))
        Lc, Rc = orc.reconfp_all(hp, dim, case["lim"])
        assert eq(L, Lc) and eq(R, Rc)
    hk.call("hc_fluxcomp", C.byref(pool)); orc.fluxcomp(hp)
    assert eq(hh.F, hp.F)
    F_aux = hh.F.copy()                     # the same fluxes without the per-cell scratch
    hh.F[:] = 0
    hk.call("hc_fluxcomp", C.byref(hk.pool(hh, aux=False)))
    assert eq(hh.F, F_aux)
    pool = hk.pool(hh)
    dt = hk.L.hc_dtcomp(C.byref(hk.P), C.byref(pool), 0.4)
    assert dt == orc.dtcomp(hp, 0.4)
    hk.L.hc_emfcomp(C.byref(pool)); orc.emfcomp(hp)
    hk.L.hc_bfupdate(C.byref(pool), dt); orc.bfupdate(hp, dt)
    assert eq(hh.EMF, hp.EMF) and eq(hh.Bf, hp.Bf)
    dv = np.zeros_like(hh.U); sv = np.zeros_like(hh.U)
    hk.call("hc_div_source", C.byref(pool), _d(dv), _d(sv))
    dc, sc = orc.div_source(hp)
    from bhgpu.mesh import interior_mask
    m = interior_mask()
    assert eq(dv[:, :, m], dc[:, :, m]) and eq(sv[:, :, m], sc[:, :, m])
    hk.L.hc_update(C.byref(hk.P), C.byref(pool), dt, 0); orc.f2cb(hp); orc.update(hp, dt, 0)
    assert eq(hh.U, hp.U) and eq(hh.W, hp.W) and eq(hh.dU, hp.dU)
    hk.call("hc_floors", C.byref(pool)); orc.floors(hp)
    assert eq(hh.U, hp.U) and eq(hh.W, hp.W)


@pytest.mark.parametrize("reuse", [True, False])
@pytest.mark.parametrize("case", CASES)
def test_steps_bitwise(case, reuse):
    q, orc, hp = box_case(2, seed=4, **case)
    hk = HostKernels(case["M"], case["a"], 0.0, GAMMA, case["lim"])
    hh = hp.copy()
    pool = hk.pool(hh, reuse=reuse)
    off = np.array([0, hp.npatch], np.int32)
    waves = np.arange(hp.npatch, dtype=np.int32)
    for _ in range(3):
        dt = hk.L.hc_step(C.byref(hk.P), C.byref(pool), 0.4, _d(waves), _d(off), 1)
        assert dt == orc.step(hp, 0.4)
        assert eq(hh.U, hp.U) and eq(hh.W, hp.W) and eq(hh.Bf, hp.Bf) and eq(hh.dU, hp.dU)


def test_refined_quilt_ghost_waves_bitwise():
    """Two refinement levels: the wave-ordered ghost fill with coarse->fine
    prolongation equals the serial quilt-order fill."""
    lo, hi = [10.0] * 3, [12.0] * 3
    q = Quilt(lo, hi, 2)
    q.refine(0); q.refine(9)
    T = q.tables()
    waves = q.ghost_waves(T["nbr"], T["leaf"])
    assert len(waves) >= 2
    orc = oracle.Oracle(0, 0, 0, GAMMA, limiter=0)
    hp = oracle.HostPool(T)
    orc.geometry(hp)
    rng = np.random.default_rng(5)
    hp.W[:, 0] = 1.0 + 0.1 * rng.random(hp.W[:, 0].shape)
    hp.W[:, 1] = 0.3 + 0.05 * rng.random(hp.W[:, 1].shape)
    hp.W[:, 5] = 0.5
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(hp.W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    hk = HostKernels(0, 0, 0, GAMMA, 0)
    hh = hp.copy()
    pool = hk.pool(hh)
    flat = np.concatenate(waves).astype(np.int32)
    off = np.zeros(len(waves) + 1, np.int32)
    off[1:] = np.cumsum([len(w) for w in waves])
    for w in range(len(waves)):
        hk.call("hc_ghosts", C.byref(pool), _d(flat[off[w]:].copy()), C.c_int(int(off[w + 1] - off[w])))
    orc.ghosts(hp)
    assert eq(hh.U, hp.U) and eq(hh.W, hp.W)
    dt = hk.L.hc_step(C.byref(hk.P), C.byref(pool), 0.4, _d(flat), _d(off), len(waves))
    assert dt == orc.step(hp, 0.4)
    assert eq(hh.U, hp.U) and eq(hh.W, hp.W)


def _hc_regrid(hk, hp, quilt, flags=None):
    """bhgpu's device regrid sequence with the host-built kernel items:
    flags, the quilt's plan, refine and ccrstr on the extended pool, the
    kept patches."""
    if flags is None:
        pool = hk.pool(hp)
        flags = np.zeros(hp.npatch, np.uint8)
        hk.L.hc_regrid_flags(C.byref(hk.P), C.byref(pool), _d(np.ascontiguousarray(hp.lvl, np.int32)), _d(flags))
    plan = quilt.regrid(flags)
    ext = oracle.HostPool({"pgeo": plan.ext_pgeo, "lvl": np.zeros(plan.n_ext, np.int32),
                           "ijk": np.zeros((plan.n_ext, 3), np.int32), "leaf": np.zeros(plan.n_ext, np.uint8),
                           "nbr": np.zeros((plan.n_ext, 6, 2), np.int32)})
    for name in ("U", "W", "dU", "F", "Bf", "EMF"):
        getattr(ext, name)[:plan.n_old] = getattr(hp, name)
    pool = hk.pool(ext)
    hk.L.hc_geometry(C.byref(pool))
    for rows, fn in ((plan.refined, "hc_refine"), (plan.flattened, "hc_ccrstr")):
        if rows:
            r = np.ascontiguousarray([[p] + kids for p, kids in rows], np.int32)
            hk.call(fn, C.byref(pool), _d(r), C.c_int(len(rows)))
    new = oracle.HostPool(quilt.tables())
    for name in ("U", "W", "dU", "F", "Bf", "EMF", "rth"):
        getattr(new, name)[:] = getattr(ext, name)[plan.keep]
    return new, plan, flags


def test_regrid_items_bitwise():
    """The regrid kernels' items (flags, refine + B_init, ccrstr + B_init)
    built for the host equal the oracle bit for bit: refinement of the
    floor state around a Schwarzschild hole, and a refined patch of the
    magnetised box flattened again."""
    import copy
    from helpers import oracle_regrid
    lo, hi = [-6.0] * 3, [6.0] * 3
    q = Quilt(lo, hi, 2)
    orc = oracle.Oracle(1.0, 0.0, 0.0, GAMMA, limiter=1)
    hk = HostKernels(1.0, 0.0, 0.0, GAMMA, 1)
    hp = oracle.HostPool(q.tables())
    orc.geometry(hp)
    rf = 1.0 / np.power(np.sqrt(np.maximum(hp.rth[:, 0], 1e-10)), 3.0)    # amrtree::pvfs, the floor state
    hp.W[:, 0] = 1e-7 * rf
    hp.W[:, 1] = 1e-5 * rf
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(hp.W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    qh = copy.deepcopy(q)
    ho, plan_o = oracle_regrid(orc, hp, q)
    hh, plan_h, flags = _hc_regrid(hk, hp, qh)
    assert plan_o.refined == plan_h.refined and len(plan_h.refined) == 8
    assert eq(ho.U, hh.U) and eq(ho.W, hh.W) and eq(ho.Bf, hh.Bf)

    q, orc, hp = box_case(2, seed=5, periodic=False, lim=1)
    hk = HostKernels(0.0, 0.0, 0.0, GAMMA, 1)
    f = np.zeros(8, np.uint8); f[5] = 1
    qh = copy.deepcopy(q)
    hh, _, _ = _hc_regrid(hk, hp, qh, f)
    orig = orc.regrid_flags
    orc.regrid_flags = lambda pool: f
    ho, _ = oracle_regrid(orc, hp, q)
    orc.regrid_flags = orig
    assert eq(ho.U, hh.U) and eq(ho.W, hh.W) and eq(ho.Bf, hh.Bf)
    orc.ghosts(ho); orc.ghosts(hh)
    qh2 = copy.deepcopy(q)
    ho2, plan_o = oracle_regrid(orc, ho, q)
    hh2, plan_h, flags = _hc_regrid(hk, hh, qh2)
    assert plan_o.flattened == plan_h.flattened == [(5, list(range(8, 16)))]
    assert eq(ho2.U, hh2.U) and eq(ho2.W, hh2.W) and eq(ho2.Bf, hh2.Bf)


def test_b_init_indices_stay_in_the_patch():
    """patch::B_init's cell indices, including the out-of-range k = -3 and
    k = 18 of its z-face branch, stay within a patch's 8000 cells."""
    from bhgpu.mesh import cell_index
    G, B = 2, 16
    idx = []
    for i in range(-G, B + G + 1):
        for j in range(-G, B + G):
            for k in range(-G, B + G):
                idx += [cell_index(i - 1, j, k), cell_index(i, j, k)] if -G < i < B + G else \
                       [cell_index(i, j, k)] if i == -G else [cell_index(i - 1, j, k)]
    for i in range(-G, B + G):
        for j in range(-G, B + G):
            for k in range(-G, B + G + 1):
                idx += [cell_index(i, j, k - 1), cell_index(i, j, k)] if -G < k < B + G else \
                       [cell_index(i, j, k)] if i == -G else [cell_index(i, j, k - 1)]
    assert min(idx) >= 0 and max(idx) < 8000


def test_analysis_items_bitwise():
    """The analysis kernel's per-cell integrands built for the host, added in
    the reference's order, equal the oracle's integrals bit for bit."""
    from bhgpu._lib import BhAnalysisParams
    q, orc, hp = box_case(2, seed=4, periodic=False, lim=1, M=1.0, a=0.0, lo=-6.0, hi=6.0)
    orc.step(hp, 0.4)
    hk = HostKernels(1.0, 0.0, 0.0, GAMMA, 1)
    pool = hk.pool(hp)
    out = np.zeros(20)
    A = BhAnalysisParams(2.0, 10.0, 0.01, 0.005)
    hk.L.hc_analysis(C.byref(hk.P), C.byref(pool), C.byref(A), _d(out))
    raw, _ = orc.analysis(hp, 2.0, 10.0)
    assert eq(out, raw)


# ---- the reciprocal-reuse quotients (BH_RCP) of the FMA and mixed variants

def _rel(a, b):
    m = np.isfinite(a) & np.isfinite(b)
    scale = np.abs(b[m]).max()
    return float(np.abs(a[m] - b[m]).max() / scale) if scale > 0 else 0.0


@pytest.mark.parametrize("M,a,Q", [(0.0, 0.0, 0.0), (1.0, 0.9375, 0.0)])
def test_reciprocal_form_physics_close(M, a, Q):
    """ptoc and HLLD with reciprocals in place of repeated divisions stay
    within a few ulps of the reference's quotients (relative to each output
    row's magnitude); con2prim's outcome changes on no more cells than the
    reference's own changes on a one-ulp move of its input, and where both
    recover, the primitives agree to the Newton tolerance's width."""
    rng = np.random.default_rng(2)
    W, r, th = random_prims(5000, rng)
    orc = oracle.Oracle(M, a, Q, GAMMA)
    hk = HostKernels(M, a, Q, GAMMA, 1, rcp=True)
    n = W.shape[1]
    U = np.zeros((8, n)); Wd = np.zeros((4, n))
    hk.call("hc_ptoc", _d(W), _d(r), _d(th), C.c_int64(n), _d(U), _d(Wd))
    Uc, Wdc = orc.ptoc(W, r, th)
    assert np.array_equal(np.isfinite(U), np.isfinite(Uc))
    for v in range(8):
        assert _rel(U[v], Uc[v]) <= 1e-14, v
    WR = W.copy(); WR[0] *= 1.07; WR[2:5] += 0.01
    UR, _ = orc.ptoc(WR, r, th)
    for dim in range(3):
        F = np.zeros((8, n)); cts = np.zeros(n)
        hk.call("hc_hlld", _d(W), _d(WR), _d(Uc), _d(UR), _d(r), _d(th), C.c_int(dim), C.c_int64(n), _d(F), _d(cts))
        Fc, cc, _ = orc.hlld(W, WR, Uc, UR, r, th, dim)
        assert _rel(cts, cc) <= 1e-14
        for v in range(8):
            assert _rel(F[v], Fc[v]) <= 1e-13, (dim, v)
    Wo = np.zeros((8, n)); Wdo = np.zeros((5, n))
    st = np.zeros(n, np.int32); it = np.zeros(n, np.int32); pa = np.zeros(n, np.int32)
    hk.call("hc_ctop", _d(Uc), _d(r), _d(th), C.c_int64(n), _d(Wo), _d(Wdo), _d(st), _d(it), _d(pa))
    Wc, _, stc, _, _ = orc.ctop(Uc, r, th)
    # Brent's success within its 100 iterations is knife-edge for many of
    # these cells: the reference's own outcome flips on a one-ulp move of U
    r2 = np.random.default_rng(5)
    Up = np.where(r2.random(Uc.shape) < 0.5, np.nextafter(Uc, np.inf), np.nextafter(Uc, -np.inf))
    stp = orc.ctop(Up, r, th)[2]
    assert np.mean(st != stc) <= max(1e-3, np.mean(stp != stc))
    ok = (st == 1) & (stc == 1)
    for v in range(8):
        assert _rel(Wo[v, ok], Wc[v, ok]) <= 1e-8, v


@pytest.mark.parametrize("case", [CASES[0], CASES[2]])
def test_reciprocal_form_first_step(case):
    """One step with the reciprocal quotients meets the first-step gate the
    FMA-contracted GPU variant meets against the oracle: 1e-12 relative L-inf
    per conserved field, or 8x the oracle's own response to a one-ulp change
    of its input."""
    from helpers import field_linf, rel_linf, ulp_sensitivity
    q, orc, hp = box_case(2, seed=4, **case)
    sens = ulp_sensitivity(orc, hp, steps=1)
    hk = HostKernels(case["M"], case["a"], 0.0, GAMMA, case["lim"], rcp=True)
    hh = hp.copy()
    pool = hk.pool(hh)
    off = np.array([0, hp.npatch], np.int32)
    waves = np.arange(hp.npatch, dtype=np.int32)
    dt = hk.L.hc_step(C.byref(hk.P), C.byref(pool), 0.4, _d(waves), _d(off), 1)
    dtc = orc.step(hp, 0.4)
    assert abs(dt - dtc) <= 1e-12 * dtc
    assert np.array_equal(np.isfinite(hh.U), np.isfinite(hp.U))
    assert max(field_linf(hh.U, hp.U).values()) <= 1e-12
    for v in range(8):
        assert rel_linf(hh.U[:, v], hp.U[:, v]) <= max(1e-12, 8 * sens[v]), v
