"""AMR regrid on the device (bh_regrid_flags, bh_refine, bh_ccrstr through
AmrTree.regrid) against the oracle, from identical states: the new quilt
exactly, and U, W, face B within the first-step gate (relative L-infinity
<= 1e-12 per conserved field, identical NaN masks).  Then steps on a
refined quilt: the reference's domain error after a refinement, and one
RK2 step with coarse->fine ghost prolongation in waves."""
import copy

import numpy as np
import pytest

import oracle
from bhgpu.mesh import Quilt
from helpers import GAMMA, box_case, field_linf, oracle_regrid, same_nan

pytestmark = pytest.mark.gpu

PRIMS = {"rho": [0], "eps": [1], "v": [2, 3, 4], "B": [5, 6, 7]}


def tree_for(q, M, a, lim):
    import bhgpu
    return bhgpu.AmrTree(q.dom_l, q.dom_h, q.nqlt, M=M, a=a, Q=0.0, gm=GAMMA, limiter=lim,
                         quilt=copy.deepcopy(q), init_floor=False)


def noise_envelope(hp_in, q_in, M, a, lim, ref_out, seeds=(1, 2, 3)):
    """Per field, the largest relative L-infinity change of the oracle's
    regrid result when every libm result carries one-ulp noise (three noise
    patterns): the band in which the reference's own answer is defined.
    Floor-state tau is a difference of terms ~1e5 times larger than itself,
    so it moves by ~1e-11 under that noise."""
    env = {}
    for s in seeds:
        orc = oracle.Oracle(M, a, 0.0, GAMMA, limiter=lim, noise=True, seed=s)
        hp, _ = oracle_regrid(orc, hp_in.copy(), copy.deepcopy(q_in))
        for name, arr, fields in (("U", hp.U, None), ("W", hp.W, PRIMS), ("Bf", hp.Bf, {"B": [0, 1, 2]})):
            d = field_linf(arr, getattr(ref_out, name), fields) if fields else field_linf(arr, ref_out.U)
            for k, v in d.items():
                env[(name, k)] = max(env.get((name, k), 0.0), v)
    return env


def check_same(tree, q, hp, env=None):
    """Same quilt; U, W, face B within 1e-12 per field, or within 8x the
    noisy-libm envelope where that is wider."""
    T, G = q.tables(), tree.quilt.tables()
    for k in ("pgeo", "lvl", "ijk", "leaf", "nbr"):
        assert np.array_equal(T[k], G[k]), k
    U, W, Bf = (x.cpu().numpy() for x in (tree.U, tree.W, tree.Bf))
    assert same_nan(U, hp.U) and same_nan(W, hp.W)
    for name, d in (("U", field_linf(U, hp.U)), ("W", field_linf(W, hp.W, PRIMS)),
                    ("Bf", field_linf(Bf, hp.Bf, {"B": [0, 1, 2]}))):
        for k, v in d.items():
            bound = max(1e-12, 8 * env.get((name, k), 0.0)) if env else 1e-12
            assert v <= bound, (name, k, v, bound)


def floor_state(q, orc):
    hp = oracle.HostPool(q.tables())
    orc.geometry(hp)
    rf = 1.0 / np.power(np.sqrt(np.maximum(hp.rth[:, 0], 1e-10)), 3.0)    # amrtree::pvfs
    hp.W[:, 0] = 1e-7 * rf
    hp.W[:, 1] = 1e-5 * rf
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(hp.W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    return hp


def test_regrid_refinement_near_the_horizon():
    """Two regrids of the floor state around a Schwarzschild hole: every
    patch refines, then (their halos being unfilled zeros) every child."""
    q = Quilt([-6.0] * 3, [6.0] * 3, 2)
    orc = oracle.Oracle(1.0, 0.0, 0.0, GAMMA, limiter=1)
    hp = floor_state(q, orc)
    tree = tree_for(q, 1.0, 0.0, 1)
    for n_expect in (72, 584):
        tree.load(U=hp.U, W=hp.W, Bf=hp.Bf)
        plan = tree.regrid()
        hp_in, q_in = hp.copy(), copy.deepcopy(q)
        hp, plan_o = oracle_regrid(orc, hp, q)
        assert plan.refined == plan_o.refined and len(q) == n_expect == tree.npatch
        check_same(tree, q, hp, noise_envelope(hp_in, q_in, 1.0, 0.0, 1, hp))


def refined_box():
    """The magnetised box with patch 5 refined by the regrid kernels."""
    q, orc, hp = box_case(2, seed=5, periodic=False, lim=1)
    tree = tree_for(q, 0.0, 0.0, 1)
    tree.load(U=hp.U, W=hp.W, Bf=hp.Bf)
    f = np.zeros(8, np.uint8); f[5] = 1
    tree.regrid(flags=f)
    orig = orc.regrid_flags
    orc.regrid_flags = lambda pool: f
    hp, _ = oracle_regrid(orc, hp, q)
    orc.regrid_flags = orig
    return q, orc, hp, tree


def test_step_after_refinement_reports_the_domain_error():
    """The first step after a refinement meets the new children's unfilled
    (zero) edge and corner ghost cells (A18) in con2prim: the reference
    throws std::domain_error, the device sets BH_ERR_DOMAIN."""
    import bhgpu
    q, orc, hp, tree = refined_box()
    with pytest.raises(oracle.DomainError):
        orc.step(hp.copy(), 0.4)
    with pytest.raises(bhgpu.DomainError):
        bhgpu.RK2Integrator(0.4).step(tree)


def test_step_on_a_refined_quilt():
    """One RK2 step on a two-level quilt (coarse->fine ghost prolongation,
    ghost fill in waves) from a state valid in every cell."""
    import bhgpu
    q, orc, hp, tree = refined_box()
    rng = np.random.default_rng(3)
    hp.W[:] = 0.0
    hp.W[:, 0] = 1.0 + 0.1 * rng.random(hp.W[:, 0].shape)
    hp.W[:, 1] = 0.3 + 0.05 * rng.random(hp.W[:, 1].shape)
    hp.W[:, 5] = 0.5
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(hp.W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    assert tree.nwave > 1
    tree.load(U=hp.U, W=hp.W, Bf=hp.Bf, dU=hp.dU)
    dtg = bhgpu.RK2Integrator(0.4).step(tree)
    dto = orc.step(hp, 0.4)
    assert abs(dtg - dto) <= 1e-12 * dto
    U = tree.U.cpu().numpy()
    assert same_nan(U, hp.U)
    assert max(field_linf(U, hp.U).values()) <= 1e-12


def test_regrid_flattens_a_smooth_refined_patch():
    q, orc, hp, tree = refined_box()
    check_same(tree, q, hp)
    orc.ghosts(hp)                          # the children's halos, as a step fills them
    tree.load(U=hp.U, W=hp.W, Bf=hp.Bf)
    plan = tree.regrid()
    hp, plan_o = oracle_regrid(orc, hp, q)
    assert plan.flattened == plan_o.flattened == [(5, list(range(8, 16)))] and tree.npatch == 8
    check_same(tree, q, hp)
