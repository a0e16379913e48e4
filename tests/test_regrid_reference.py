"""Pins the AMR regrid of the C restatement (refinement flags, refine's
prolongation, ccrstr's restriction, B_init) and the quilt bookkeeping of
bhgpu.mesh to the reference's own amrtree::refine / flatten / regrid
(grid.cpp:573-835), bit for bit.

The tree metric has a = 0 throughout: the reference's regrid calls its
con2prim from inside its own loops, where the uninitialised reads of
conserved.cpp:144-150 cannot be scrubbed, and only for a = 0 are they
multiplied by an exact zero.  Skipped where the reference harness is not
built."""
import numpy as np
import pytest

import oracle
from bhgpu.mesh import Quilt
from helpers import GAMMA, box_case, oracle_regrid

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built")


def eq(a, b):
    return np.array_equal(a, b, equal_nan=True)


def same_pool(hp, ref):
    R = oracle.HostPool(ref.patch_info() | {"nbr": np.zeros((ref.npatch, 6, 2), np.int32)})
    ref.get(R)
    return eq(hp.U, R.U) and eq(hp.W, R.W) and eq(hp.Bf, R.Bf)


def same_tables(q, ref):
    T, info = q.tables(), ref.patch_info()
    return len(q) == ref.npatch and all(eq(info[k], T[k]) for k in ("pgeo", "lvl", "ijk", "leaf"))


def test_refine_prolongation_and_b_init():
    """amrtree::refine of one patch of the magnetised box: children's U, W
    (prolongation with the reference's swapped neighbour order, con2prim and
    its fallback) and their face B (B_init, with its z-face quirk)."""
    q, orc, hp = box_case(2, seed=5, periodic=False, lim=1)
    ref = oracle.RefSolver(q.dom_l, q.dom_h, 2, 0.0, 0.0, 0.0, GAMMA)
    ref.put(hp)
    ref.refine(3)
    flags = np.zeros(len(q), np.int32); flags[3] = 1
    plan = q.regrid(flags)
    assert plan.refined == [(3, list(range(8, 16)))] and not plan.flattened
    ext = oracle.HostPool(q.tables())
    for name in ("U", "W", "Bf"):
        getattr(ext, name)[:8] = getattr(hp, name)
    orc.geometry(ext)
    orc.refine_data(ext, 3, plan.refined[0][1])
    assert same_tables(q, ref)
    assert same_pool(ext, ref)
    assert (ext.Bf[8:, 2] != 0).any() and (ext.W[8:, 0] > 0).any()


def test_regrid_refines_near_the_horizon_twice():
    """Two amrtree::regrid passes on the floor state around a Schwarzschild
    hole.  The first refines every patch (each holds cells inside r = 3);
    in the second, the children's unfilled (zero) halos give every child a
    density gradient above the threshold, so all 64 refine."""
    lo, hi = [-6.0] * 3, [6.0] * 3
    ref = oracle.RefSolver(lo, hi, 2, 1.0, 0.0, 0.0, GAMMA)
    q = Quilt(lo, hi, 2)
    orc = oracle.Oracle(1.0, 0.0, 0.0, GAMMA, limiter=1)
    hp = oracle.HostPool(q.tables())
    orc.geometry(hp)
    ref.get(hp)                           # the reference's own initial state (pvfs, ptoc)
    for n_expect in (72, 584):
        ref.regrid()
        hp, plan = oracle_regrid(orc, hp, q)
        assert len(q) == n_expect and plan.refined and not plan.flattened
        assert same_tables(q, ref)
        assert same_pool(hp, ref)


def test_regrid_flattens_smooth_children():
    """A refined patch whose children carry no gradient is flattened again:
    ccrstr's volume-weighted restriction, con2prim, B_init of the parent,
    and the children removed from the quilt in order."""
    q, orc, hp = box_case(2, seed=5, periodic=False, lim=1)
    ref = oracle.RefSolver(q.dom_l, q.dom_h, 2, 0.0, 0.0, 0.0, GAMMA)
    ref.put(hp)
    ref.refine(5)
    flags = np.zeros(len(q), np.int32); flags[5] = 1
    hp, _ = _apply(orc, hp, q, flags)
    assert same_pool(hp, ref)
    T = q.tables()
    orc.ghosts(hp); ref.ghosts(T["nbr"])     # fill the children's halos as a step would
    assert same_pool(hp, ref)
    flags = orc.regrid_flags(hp)
    assert (flags[8:] == 2).all() and (flags[:8] == 0).all()
    ref.regrid()
    hp, plan = oracle_regrid(orc, hp, q)
    assert plan.flattened == [(5, list(range(8, 16)))] and len(q) == 8
    assert same_tables(q, ref)
    assert same_pool(hp, ref)


def _apply(orc, hp, q, flags):
    """oracle_regrid with given flags instead of the cell loop's."""
    orig = orc.regrid_flags
    orc.regrid_flags = lambda pool: flags
    try:
        return oracle_regrid(orc, hp, q)
    finally:
        orc.regrid_flags = orig
