"""Step the Kerr torus a few times with chosen launch settings: the
workload for a profiler's capture of the corrected scheme's kernels.

    python -m bhgpu.profile_step --precision mixed --grid 128 --steps 2 \\
        --tune c2p=6,flux=8,update=7,stage=1

(run from the package directory, or with it on PYTHONPATH).  Every step is
one torus RK2 step (con2prim, ghost fill, fluxes, update per stage); no
timing is taken, so the numbers a profiler reports are the only output.
``--form faithful`` steps the reference-faithful form instead (FP64, the
magnetised box of (grid/16)^3 patches of 16^3 cells, periodic, minmod).
"""
from __future__ import annotations

import argparse

import torch

from bhgpu.fixed import FxGrid, FxParams, tune_set


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "fp64-fma", "mixed"])
    ap.add_argument("--grid", type=int, default=128, help="cells per axis over [-40, 40]^3")
    ap.add_argument("--block", type=int, default=0, help="cells per block axis (0: one block)")
    ap.add_argument("--limiter", default="mc", choices=["minmod", "vanleer", "mc", "ppm"])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--tune", default="", help="knob=value,...: c2p, flux, update (CTAs per SM), stage (0/1)")
    ap.add_argument("--form", default="fixed", choices=["fixed", "faithful"])
    a = ap.parse_args(argv)
    if a.form == "faithful":
        return faithful(a)
    for kv in filter(None, a.tune.split(",")):
        k, v = kv.split("=")
        tune_set(a.precision, k, int(v))
    g = FxGrid.uniform(-40.0, 40.0, a.grid, a.block or a.grid, FxParams(precision=a.precision, limiter=a.limiter))
    g.torus_init()
    for _ in range(a.steps):
        g.step()
    torch.cuda.synchronize()
    print("ok", a.precision, a.grid, g.counters(), flush=True)


def faithful(a):
    import bhgpu
    from bhgrid import configs
    from bhgrid.mesh import Quilt
    nq = a.grid // 16
    q = Quilt([10.0] * 3, [12.0] * 3, nq, periodic=True)
    tree = bhgpu.AmrTree(q.dom_l, q.dom_h, nq, M=0.0, a=0.0, Q=0.0, gm=4.0 / 3.0, periodic=True, limiter="minmod",
                         quilt=q, init_floor=False, precision="fp64")
    W, Bf = configs.magnetised_box(q, seed=1, gamma=4.0 / 3.0)
    tree.load(W=W, Bf=Bf)
    tree.prim_to_cons()
    rk = bhgpu.RK2Integrator(0.4)
    for _ in range(a.steps):
        rk.step(tree, sync=False, check_domain=False)
    torch.cuda.synchronize()
    print("ok faithful", a.grid, flush=True)


if __name__ == "__main__":
    main()
