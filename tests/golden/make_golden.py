"""Generates tests/golden/reference_golden.npz from the reference solver
itself (its sources compiled by oracle/Makefile into oracle/_ref).

    python tests/golden/make_golden.py

Contents: seeded inputs and the reference's outputs for metric::comp,
conserved::ptoc / ctop, hlld, and for whole steps of small patch quilts
(the reference's own rk2integrator::step with outflow ghosts and van Leer;
the restated periodic/minmod step built from the reference's functions),
stored as a strided sample of cells plus exact per-variable checksums.
The initial states are regenerated by the test from the same seed; their
checksums are stored to check that regeneration.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "black-hole-simulator_b200"), os.path.join(REPO, "tests")]

import oracle  # noqa: E402
from bhgpu import configs  # noqa: E402
from bhgpu.mesh import Quilt  # noqa: E402
from helpers import GAMMA, random_prims  # noqa: E402

SAMPLE = slice(0, None, 97)


def checksums(a):
    """Per-variable (sum of finite entries, number of non-finite entries)."""
    a = a.reshape(a.shape[0], a.shape[1], -1) if a.ndim == 3 else a
    out = []
    for v in range(a.shape[1]):
        x = a[:, v].reshape(-1)
        f = np.isfinite(x)
        out.append((float(np.sum(x[f])), float((~f).sum())))
    return np.array(out)


def main():
    g = {}
    for tag, (M, a, Q) in {"flat": (0.0, 0.0, 0.0), "kerr": (1.0, 0.9375, 0.0), "kn": (1.0, 0.9, 0.1)}.items():
        rng = np.random.default_rng(100)
        ref = oracle.RefSolver([10.0] * 3, [12.0] * 3, 1, M, a, Q, GAMMA)
        W, r, th = random_prims(256, rng)
        WR = W.copy(); WR[0] *= 1.1; WR[2:5] += 0.01
        g[f"{tag}_W"], g[f"{tag}_r"], g[f"{tag}_th"], g[f"{tag}_WR"] = W, r, th, WR
        g[f"{tag}_metric"] = ref.metric(r[:48], th[:48])
        U, Wd = ref.ptoc(W, r, th)
        g[f"{tag}_U"], g[f"{tag}_Wd"] = U, Wd
        Wc, Wdc, st = ref.ctop(U, r, th)
        g[f"{tag}_ctop_W"], g[f"{tag}_ctop_Wd"], g[f"{tag}_ctop_status"] = Wc, Wdc, st
        UR, _ = ref.ptoc(WR, r, th)
        F, cts, _ = ref.hlld(W, WR, U, UR, r, th, 0)
        g[f"{tag}_UR"], g[f"{tag}_F"], g[f"{tag}_cts"] = UR, F, cts
    # whole steps on 2^3 patches of the magnetised box
    for tag, periodic, lim in (("box_periodic_minmod", True, 0), ("box_outflow_vanleer", False, 1)):
        q = Quilt([10.0] * 3, [12.0] * 3, 2, periodic=periodic)
        W, Bf = configs.magnetised_box(q, seed=9, gamma=GAMMA)
        ref = oracle.RefSolver([10.0] * 3, [12.0] * 3, 2, 0.0, 0.0, 0.0, GAMMA)
        hp = oracle.HostPool(q.tables())
        hp.rth[:] = ref.geom()
        hp.W[:] = W; hp.Bf[:] = Bf
        for p in range(hp.npatch):
            hp.U[p] = ref.ptoc(W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
        g[f"{tag}_U0_sum"] = checksums(hp.U)   # the test regenerates the state and checks it
        ref.put(hp)
        dts = []
        for _ in range(2):
            dts.append(ref.step(0.4, hp.nbr, lim) if periodic else ref.step_native(0.4))
        ref.get(hp)
        g[f"{tag}_dt"] = np.array(dts)
        for name in ("U", "W", "Bf"):
            arr = getattr(hp, name)
            g[f"{tag}_{name}_sum"] = checksums(arr)
            g[f"{tag}_{name}_sample"] = arr.reshape(arr.shape[0], arr.shape[1], -1)[:, :, SAMPLE].copy()
    np.savez_compressed(os.path.join(HERE, "reference_golden.npz"), **g)
    print("wrote", os.path.join(HERE, "reference_golden.npz"), len(g), "arrays")


if __name__ == "__main__":
    main()
