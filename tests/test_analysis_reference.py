"""analysis::analyser (data/quantitatives.cpp): the C restatement's
integrals, summed in the reference's order, and bhgpu.analysis's
composition of batch_ / bundle_ equal the reference's own analyser bit for
bit on the state its step leaves (the derived primitive fields floors
records included).  a = 0, so the reference's own loops are deterministic.
Skipped where the reference harness is not built."""
import numpy as np
import pytest

import oracle
from bhgpu.analysis import BATCH_FIELDS, BUNDLE_FIELDS, compose_batch, compose_bundle, r_horizon
from bhgpu.mesh import interior_mask
from helpers import GAMMA, box_case

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built")


def eq(a, b):
    return np.array_equal(a, b, equal_nan=True)


def stepped(M=1.0):
    q, orc, hp = box_case(2, seed=4, periodic=False, lim=1, M=M, a=0.0, lo=-6.0, hi=6.0)
    ref = oracle.RefSolver(q.dom_l, q.dom_h, 2, M, 0.0, 0.0, GAMMA)
    ref.put(hp)
    T = q.tables()
    assert orc.step(hp, 0.4) == ref.step(0.4, T["nbr"], 1)
    return q, orc, hp, ref


def test_floors_records_the_reference_derived_fields():
    q, orc, hp, ref = stepped()
    m = interior_mask()
    assert eq(hp.Wd[:, :, m], ref.derived()[:, :, m])
    assert np.isfinite(hp.Wd[:, :, m]).any()


@pytest.mark.parametrize("t", [0.0, 0.75])
def test_batch_and_bundle_bitwise(t):
    q, orc, hp, ref = stepped()
    raw, _ = orc.analysis(hp, r_horizon(1.0, 0.0, 0.0), 10.0)
    assert raw[3] != 0.0 and raw[9] != 0.0 and raw[18] != 0.0, "surface integrals select cells"
    b = compose_batch(raw, t, 1.0, 0.0, 0.0)
    rb = ref.batch(t)
    for i, k in enumerate(BATCH_FIELDS):
        assert eq(b[k], rb[i]), k
    u = compose_bundle(raw, t)
    ru = ref.bundle(t)
    for i, k in enumerate(BUNDLE_FIELDS):
        assert eq(u[k], ru[i]), k
