"""GPU parity: every function of the path, called through the C ABI of
libbhgpu.so, against the CPU oracle on the same seeded inputs.

The kernel logic itself is pinned bit for bit on the CPU
(tests/test_hostcheck.py); what remains between GPU and oracle are the
last bits of the device math library (sin, cos, acos, log, exp, pow).
Tolerances written here:

* smooth functions (metric, ptoc, hlld, reconfp, fluxes, CT, sources):
  relative L-infinity <= 1e-12 per variable;
* con2prim: identical status, route and iteration count wherever the
  reference takes its Newton route; the Brent fallback of the reference
  (conserved.cpp:232-285) flips between success and failure under a
  one-ulp change of its input (measured on the oracle itself), so Brent
  cells may differ at most at the oracle's own one-ulp flip rate; with
  exactly representable metric inputs Brent results are identical;
* the first step from a seeded state: relative L-infinity <= 1e-12 per
  conserved field (D, the vector S, tau, the vector B), identical NaN
  masks, and per component within 8x the oracle's own response to a
  one-ulp input perturbation;
* later steps: the reference's own result is only defined up to its
  response to last-bit rounding (its Brent fallback and the blow-up of the
  magnetised box amplify one ulp to O(1) within two steps), measured by
  the oracle built with one-ulp noise on every libm result; the GPU's NaN
  mask and per-variable L1 error stay within 2x / 8x of that envelope."""
import math

import numpy as np
import pytest
import torch

import oracle
from helpers import (GAMMA, box_case, field_linf, gpu_tree, mask_disagreement, rel_l1, rel_linf, random_prims,
                     same_nan, ulp_sensitivity)

pytestmark = pytest.mark.gpu
TOL = 1e-12
METRICS = [(0.0, 0.0, 0.0), (1.0, 0.9375, 0.0), (1.0, 0.9, 0.1)]


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("M,a,Q", METRICS)
def test_metric(M, a, Q):
    import bhgpu
    rng = np.random.default_rng(1)
    _, r, th = random_prims(4000, rng)
    g = _np(bhgpu.Metric(M, a, Q).comp(r, th))
    c = oracle.Oracle(M, a, Q, GAMMA).metric(r, th)
    assert same_nan(g, c)
    for col in range(120):
        assert rel_linf(g[:, col], c[:, col]) <= TOL, col


@pytest.mark.parametrize("M,a,Q", METRICS)
def test_ptoc_hlld(M, a, Q):
    import bhgpu
    rng = np.random.default_rng(2)
    W, r, th = random_prims(20000, rng)
    orc = oracle.Oracle(M, a, Q, GAMMA)
    cn = bhgpu.Conserved(bhgpu.Metric(M, a, Q), bhgpu.State(GAMMA))
    Ug, _ = cn.ptoc(W, r, th)
    Uc, _ = orc.ptoc(W, r, th)
    for v in range(8):
        assert rel_linf(_np(Ug)[v], Uc[v]) <= TOL
    WR = W.copy(); WR[0] *= 1.07; WR[2:5] += 0.01 * rng.normal(size=(3, W.shape[1]))
    UR, _ = orc.ptoc(WR, r, th)
    for dim in (0, 1, 2):
        Fg, cg = bhgpu.hlld(W, WR, Uc, UR, bhgpu.Metric(M, a, Q), r, th, bhgpu.State(GAMMA), dim)
        Fc, cc, _ = orc.hlld(W, WR, Uc, UR, r, th, dim)
        Fg = _np(Fg)
        assert same_nan(Fg, Fc)
        for v in range(8):
            assert rel_linf(Fg[v], Fc[v]) <= TOL, (dim, v)
        assert rel_linf(_np(cg), cc) <= TOL


@pytest.mark.parametrize("M,a,Q", METRICS)
def test_ctop(M, a, Q):
    import bhgpu
    rng = np.random.default_rng(3)
    W, r, th = random_prims(20000, rng)
    orc = oracle.Oracle(M, a, Q, GAMMA)
    Uc, _ = orc.ptoc(W, r, th)
    cn = bhgpu.Conserved(bhgpu.Metric(M, a, Q), bhgpu.State(GAMMA))
    Wg, Wdg, stg, itg, pag = [_np(x) for x in cn.ctop(Uc, r, th)]
    Wc, Wdc, stc, itc, pac = orc.ctop(Uc, r, th)
    newton = pac == 0
    assert newton.sum() > 1000
    assert np.array_equal(pag[newton], pac[newton]) and np.array_equal(itg[newton], itc[newton])
    assert np.array_equal(stg[newton], stc[newton])
    # the oracle's own flip rate under a one-ulp change of theta
    _, _, st1, _, pa1 = orc.ctop(Uc, r, np.nextafter(th, 10.0))
    own = np.mean(st1 != stc)
    assert own > 0, "reference Brent route is ulp-sensitive on these states"
    assert np.mean(stg != stc) <= 1.5 * own + 1e-3
    same = (stg == 1) & (stc == 1) & (pag == pac)
    assert same_nan(Wg[:, same], Wc[:, same])
    for v in range(8):
        assert rel_linf(Wg[v, same], Wc[v, same]) <= TOL, v


def test_ctop_stress_batch_distribution():
    """The con2prim stress batch's own distribution (log-uniform rho in
    [1e-8, 1], W up to 20, sigma up to 100, Kerr a = 0.9375 at r in
    [1.5, 50]) on a 2^16-cell sample: the same gates as test_ctop
    (conserved.cpp:135-285)."""
    import bhgpu
    from bhgpu import configs
    a = 0.9375
    W, r, th = configs.con2prim_batch(1 << 16, seed=4, gamma=GAMMA, a=a)
    orc = oracle.Oracle(1.0, a, 0.0, GAMMA)
    Uc, _ = orc.ptoc(W, r, th)
    cn = bhgpu.Conserved(bhgpu.Metric(1.0, a, 0.0), bhgpu.State(GAMMA))
    Wg, _, stg, itg, pag = [_np(x) for x in cn.ctop(Uc, r, th, check_domain=False)]
    Wc, _, stc, itc, pac = orc.ctop(Uc, r, th)
    newton = pac == 0
    assert newton.sum() > 1000 and (pac >= 2).sum() > 1000, "both routes exercised"
    assert np.array_equal(pag[newton], pac[newton]) and np.array_equal(itg[newton], itc[newton])
    assert np.array_equal(stg[newton], stc[newton])
    _, _, st1, _, _ = orc.ctop(Uc, r, np.nextafter(th, 10.0))
    own = np.mean(st1 != stc)
    assert np.mean(stg != stc) <= 1.5 * own + 1e-3, (np.mean(stg != stc), own)
    same = (stg == 1) & (stc == 1) & (pag == pac)
    assert same.sum() > 1000
    assert same_nan(Wg[:, same], Wc[:, same])
    for v in range(8):
        assert rel_linf(Wg[v, same], Wc[v, same]) <= TOL, v


def test_ctop_brent_route_exact_metric():
    """theta = pi/2 and a flat metric make every metric entry exact on both
    sides; the Brent fallback then gives identical outcomes."""
    import bhgpu
    rng = np.random.default_rng(4)
    W, r, _ = random_prims(20000, rng)
    th = np.full(W.shape[1], math.pi / 2)
    orc = oracle.Oracle(0.0, 0.0, 0.0, GAMMA)
    Uc, _ = orc.ptoc(W, r, th)
    cn = bhgpu.Conserved(bhgpu.Metric(0.0, 0.0, 0.0), bhgpu.State(GAMMA))
    Wg, _, stg, itg, pag = [_np(x) for x in cn.ctop(Uc, r, th)]
    Wc, _, stc, itc, pac = orc.ctop(Uc, r, th)
    assert (pac == 2).sum() > 100, "Brent route exercised"
    assert np.array_equal(stg, stc) and np.array_equal(pag, pac) and np.array_equal(itg, itc)
    ok = stc == 1
    assert same_nan(Wg[:, ok], Wc[:, ok])
    for v in range(8):
        assert rel_linf(Wg[v, ok], Wc[v, ok]) <= TOL


def test_ctop_domain_error_raises():
    import bhgpu
    cn = bhgpu.Conserved(bhgpu.Metric(0, 0, 0), bhgpu.State(GAMMA))
    U = np.zeros((8, 3)); U[0] = [-1.0, 0.0, 1.0]; U[4] = 1.0
    r = np.full(3, 15.0); th = np.ones(3)
    _, _, st, _, _ = cn.ctop(U, r, th, check_domain=False)
    assert list(_np(st)) == [0, -1, 1]
    with pytest.raises(bhgpu.DomainError):
        cn.ctop(U, r, th)


def _cmp_pool(tree, hp, names=("U", "W"), tol=TOL):
    for name in names:
        g = _np(getattr(tree, name)); c = getattr(hp, name)
        assert same_nan(g, c), name
        for v in range(g.shape[1]):
            assert rel_linf(g[:, v], c[:, v]) <= tol, (name, v, rel_linf(g[:, v], c[:, v]))


CASES = [dict(periodic=True, lim=0, M=0.0, a=0.0, lo=10.0, hi=12.0),
         dict(periodic=False, lim=1, M=0.0, a=0.0, lo=10.0, hi=12.0),
         dict(periodic=True, lim=2, M=1.0, a=0.9375, lo=-6.0, hi=6.0)]


@pytest.mark.parametrize("case", CASES)
def test_patch_functions(case):
    """Each stage function on identical input (state re-synchronised from
    the oracle between functions)."""
    import bhgpu
    from bhgpu.mesh import interior_mask
    q, orc, hp = box_case(2, seed=3, **case)
    tree = gpu_tree(q, hp, case["M"], case["a"], case["lim"])
    assert rel_linf(_np(tree.rth), hp.rth) <= 1e-15
    tree.rth.copy_(torch.as_tensor(hp.rth))
    tree.ghosts(); orc.ghosts(hp)
    _cmp_pool(tree, hp)
    tree.load(U=hp.U, W=hp.W)
    tree.prims(); orc.prims(hp)
    _cmp_pool(tree, hp)
    tree.load(U=hp.U, W=hp.W)
    for dim in range(3):
        Lg, Rg = tree.reconfp(dim)
        Lc, Rc = orc.reconfp_all(hp, dim, case["lim"])
        for v in range(8):
            assert rel_linf(_np(Lg)[v], Lc[v]) <= TOL and rel_linf(_np(Rg)[v], Rc[v]) <= TOL
    tree.fluxcomp(); orc.fluxcomp(hp)
    assert same_nan(_np(tree.F), hp.F)
    for d in range(3):
        for v in range(8):
            assert rel_linf(_np(tree.F)[:, d, v], hp.F[:, d, v]) <= TOL, (d, v)
    tree.F.copy_(torch.as_tensor(hp.F))
    dtg = bhgpu.RK2Integrator.dtcomp(tree, 0.4).item()
    dtc = orc.dtcomp(hp, 0.4)
    assert abs(dtg - dtc) <= TOL * dtc
    tree.emfcomp(); orc.emfcomp(hp)
    assert rel_linf(_np(tree.EMF), hp.EMF) <= TOL
    tree.EMF.copy_(torch.as_tensor(hp.EMF))
    tree.bfupdate(dtc); orc.bfupdate(hp, dtc)
    assert rel_linf(_np(tree.Bf), hp.Bf) <= TOL
    tree.Bf.copy_(torch.as_tensor(hp.Bf))
    assert rel_linf(_np(tree.maxdivb()), orc.maxdivb(hp)) <= 1e-9
    dg, sg = tree.div_source()
    dc, sc = orc.div_source(hp)
    inner = interior_mask()
    for v in range(8):
        assert rel_linf(_np(dg)[:, v][:, inner], dc[:, v][:, inner]) <= TOL
        assert rel_linf(_np(sg)[:, v][:, inner], sc[:, v][:, inner]) <= TOL
    tree.update(dtc, 0); orc.f2cb(hp); orc.update(hp, dtc, 0)
    _cmp_pool(tree, hp, ("U", "W", "dU"))
    tree.load(U=hp.U, W=hp.W)
    tree.floors(); orc.floors(hp)
    _cmp_pool(tree, hp)


def _step_gate(tree, hp, sens, label):
    U = _np(tree.U)
    assert same_nan(U, hp.U), label
    f = field_linf(U, hp.U)
    assert max(f.values()) <= TOL, (label, f)
    for v in range(8):
        e = rel_linf(U[:, v], hp.U[:, v])
        assert e <= max(TOL, 8 * sens[v]), (label, v, e, sens[v])
    W = _np(tree.W)
    assert same_nan(W, hp.W), label
    assert rel_linf(_np(tree.Bf), hp.Bf) <= TOL, label


NOISE_SEEDS = range(6)


def _envelope(noisy_states, ref_U):
    """Largest NaN-mask disagreement and per-variable relative L1 error of
    the noisy-oracle realisations against the plain oracle."""
    mask = max(mask_disagreement(h.U, ref_U) for h in noisy_states)
    l1 = np.max([rel_l1(h.U, ref_U) for h in noisy_states], axis=0)
    return mask, l1


def _envelope_gate(gpu_U, ref_U, noisy_states, label):
    """After the first step the reference's result is defined only up to its
    own sensitivity to last-bit rounding: the same algorithm with one-ulp
    noise on every libm result (the noisy oracle, several noise patterns)
    moves it by this much.  The GPU, whose math library differs from the
    host's in the last bit, must stay within a small multiple of it."""
    own_mask, own_l1 = _envelope(noisy_states, ref_U)
    gpu_mask = mask_disagreement(gpu_U, ref_U)
    assert gpu_mask <= 2 * own_mask + 1e-3, (label, gpu_mask, own_mask)
    gpu = rel_l1(gpu_U, ref_U)
    for v in range(8):
        assert gpu[v] <= 8 * own_l1[v] + 1e-13, (label, v, gpu[v], own_l1[v])


def _noisy(case):
    return [oracle.Oracle(case["M"], case["a"], 0.0, GAMMA, limiter=case["lim"], noise=True, seed=k)
            for k in NOISE_SEEDS]


@pytest.mark.parametrize("case", CASES)
def test_free_running_steps(case):
    """Three free-running steps: step 1 meets the strict gate; steps 2-3
    (where the flat-metric box is chaotic in the reference itself) stay
    within the envelope of the noisy oracle, each realisation with its own
    cell geometry as the GPU has its own."""
    import bhgpu
    q, orc, hp = box_case(2, seed=4, **case)
    noisy = _noisy(case)
    hns = [hp.copy() for _ in noisy]
    for o, h in zip(noisy, hns):
        o.geometry(h)
    sens1 = ulp_sensitivity(orc, hp, steps=1)
    tree = gpu_tree(q, hp, case["M"], case["a"], case["lim"])
    rk = bhgpu.RK2Integrator(0.4)
    for s in range(3):
        dtg = rk.step(tree, check_domain=False)
        dtc = orc.step(hp, 0.4)
        for o, h in zip(noisy, hns):
            o.step(h, 0.4)
        if s == 0:
            assert abs(dtg - dtc) <= TOL * dtc
            _step_gate(tree, hp, sens1, "step 1")
        else:
            _envelope_gate(_np(tree.U), hp.U, hns, f"step {s + 1}")


@pytest.mark.parametrize("case", CASES)
def test_stepwise_from_identical_state(case):
    """Three consecutive steps, each started from the oracle's state (cell
    geometry included): each GPU step stays within the envelope of the
    noisy oracle started from the same state, and the first meets the
    strict gate."""
    import bhgpu
    q, orc, hp = box_case(2, seed=4, **case)
    noisy = _noisy(case)
    tree = gpu_tree(q, hp, case["M"], case["a"], case["lim"])
    tree.rth.copy_(torch.as_tensor(hp.rth))
    rk = bhgpu.RK2Integrator(0.4)
    for k in range(3):
        tree.load(U=hp.U, W=hp.W, Bf=hp.Bf, dU=hp.dU)
        hns = [hp.copy() for _ in noisy]
        sens = ulp_sensitivity(orc, hp, steps=1) if k == 0 else None
        dtg = rk.step(tree, check_domain=False)
        dtc = orc.step(hp, 0.4)
        for o, h in zip(noisy, hns):
            o.step(h, 0.4)
        if k == 0:
            assert abs(dtg - dtc) <= TOL * dtc
            _step_gate(tree, hp, sens, "step 1")
        else:
            _envelope_gate(_np(tree.U), hp.U, hns, f"step {k + 1} from the oracle's state")


def test_magnetised_box_64cubed_one_step():
    """The 64^3 magnetised box (4^3 patches of 16^3, periodic, PLM-minmod,
    HLLD, CT, RK2, CFL 0.4, flat metric), one full step."""
    import bhgpu
    q, orc, hp = box_case(4, seed=1, periodic=True, lim=0)
    sens = ulp_sensitivity(orc, hp, steps=1)
    tree = gpu_tree(q, hp, 0.0, 0.0, 0)
    dtg = bhgpu.RK2Integrator(0.4).step(tree)
    dtc = orc.step(hp, 0.4)
    assert abs(dtg - dtc) <= TOL * dtc
    _step_gate(tree, hp, sens, "64^3 one step")
