"""The C restatement (oracle) against fixtures produced by the reference
solver itself (tests/golden/make_golden.py): bit-for-bit on every stored
value.  Runs on any host, with or without the reference sources."""
import os

import numpy as np
import pytest

import oracle
from bhgpu import configs
from bhgpu.mesh import Quilt
from helpers import GAMMA

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz"))
SAMPLE = slice(0, None, 97)


def eq(a, b):
    return np.array_equal(a, b, equal_nan=True)


def checksums(a):
    a = a.reshape(a.shape[0], a.shape[1], -1)
    out = []
    for v in range(a.shape[1]):
        x = a[:, v].reshape(-1)
        f = np.isfinite(x)
        out.append((float(np.sum(x[f])), float((~f).sum())))
    return np.array(out)


@pytest.mark.parametrize("tag,M,a,Q", [("flat", 0.0, 0.0, 0.0), ("kerr", 1.0, 0.9375, 0.0), ("kn", 1.0, 0.9, 0.1)])
def test_physics_golden(tag, M, a, Q):
    orc = oracle.Oracle(M, a, Q, GAMMA)
    W, r, th, WR = G[f"{tag}_W"], G[f"{tag}_r"], G[f"{tag}_th"], G[f"{tag}_WR"]
    assert eq(orc.metric(r[:48], th[:48]), G[f"{tag}_metric"])
    U, Wd = orc.ptoc(W, r, th)
    assert eq(U, G[f"{tag}_U"]) and eq(Wd, G[f"{tag}_Wd"])
    Wc, Wdc, st, _, _ = orc.ctop(U, r, th)
    assert eq(st, G[f"{tag}_ctop_status"])
    ok = st == 1
    assert eq(Wc[:, ok], G[f"{tag}_ctop_W"][:, ok]) and eq(Wdc[:, ok], G[f"{tag}_ctop_Wd"][:, ok])
    UR, _ = orc.ptoc(WR, r, th)
    assert eq(UR, G[f"{tag}_UR"])
    F, cts, _ = orc.hlld(W, WR, U, UR, r, th, 0)
    assert eq(F, G[f"{tag}_F"]) and eq(cts, G[f"{tag}_cts"])


@pytest.mark.parametrize("tag,periodic,lim", [("box_periodic_minmod", True, 0), ("box_outflow_vanleer", False, 1)])
def test_two_steps_golden(tag, periodic, lim):
    q = Quilt([10.0] * 3, [12.0] * 3, 2, periodic=periodic)
    W, Bf = configs.magnetised_box(q, seed=9, gamma=GAMMA)
    orc = oracle.Oracle(0.0, 0.0, 0.0, GAMMA, limiter=lim)
    hp = oracle.HostPool(q.tables())
    orc.geometry(hp)
    hp.W[:] = W; hp.Bf[:] = Bf
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    assert eq(checksums(hp.U), G[f"{tag}_U0_sum"]), "regenerated initial state differs"
    dts = [orc.step(hp, 0.4) for _ in range(2)]
    assert eq(np.array(dts), G[f"{tag}_dt"])
    for name in ("U", "W", "Bf"):
        arr = getattr(hp, name)
        assert eq(checksums(arr), G[f"{tag}_{name}_sum"]), name
        assert eq(arr.reshape(arr.shape[0], arr.shape[1], -1)[:, :, SAMPLE], G[f"{tag}_{name}_sample"]), name
