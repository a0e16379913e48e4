"""The corrected scheme's block grid sharded over world_size 2 and 3 gloo
process groups on the CPU (bhgpu.fxshard, bhgrid.shard), with the oracle
doing each rank's arithmetic: each rank holds its Morton run of blocks plus
copies of their neighbours (less memory than the whole grid), steps only its
own blocks, and exchanges the copies' boxes between the pieces of a stage.
The owned blocks after the sharded steps must equal the whole grid stepped
in one process, bit for bit -- on one level, across three levels (ghost
fill passes and the EMF correction across ranks), and with PPM's third
ghost layer."""
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(kind):
    from bhgrid.blocks import leveled_blocks, torus_levels, uniform_blocks
    if kind == "uniform":
        return uniform_blocks(-40.0, 40.0, 32, 8)
    return leveled_blocks(-40.0, 40.0, torus_levels(nb=6, r_fine=(14.0, 26.0), seed=3), 4)


def _params(limiter):
    from oracle import fixed as ofx

    class Prm:   # the scheme's defaults (bhgpu.fixed.FxParams) without importing the CUDA library
        M, a, gamma, cfl = 1.0, 0.9375, 4.0 / 3.0, 0.4
        rho_floor, u_floor, sigma_max, W_max, r_exc = 1e-6, 1e-8, 100.0, 50.0, None
        tol, maxiter = 1e-12, 30
    Prm.limiter = limiter
    return ofx.params(Prm)


def _worker(rank, world, port, out_dir, kind, limiter, steps):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "black-hole-simulator_b200"))
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist
    from oracle import fixed as ofx
    from bhgpu.fxshard import ShardedFxGrid
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ.setdefault("OMP_NUM_THREADS", "2")
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        blocks, nbr = _case(kind)
        prm = _params(limiter)
        whole = ofx.FxHost(blocks, nbr, prm)
        whole.torus_init()
        sh = ShardedFxGrid(blocks, nbr, lambda lb, ln, na, ml: ofx.FxHost(lb, ln, prm, nactive=na, maxlevel=ml))
        # unfilled entries of the local arrays: NaN, so that a read of data
        # that did not arrive shows up in the result
        for name in ("U", "U1", "W", "Bf", "Bf1", "F", "E"):
            getattr(sh.grid, name)[:] = np.nan
        for name in ("U", "W", "Bf"):
            sh.scatter(name, getattr(whole, name))
        for _ in range(steps):
            sh.step()
        out = {"U": sh.owned_boxes("U"), "Bf": sh.owned_boxes("Bf"), "dt": sh.grid.dt.copy(),
               "ncell": sh.local.ncell, "whole": whole.N}
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array(out, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,limiter,world", [("uniform", "mc", 2), ("leveled", "mc", 2), ("leveled", "mc", 3),
                                                ("leveled", "ppm", 2)])
def test_sharded_steps_equal_one_process(kind, limiter, world):
    from oracle import fixed as ofx
    from bhgrid.blocks import box_size
    steps = 2
    blocks, nbr = _case(kind)
    whole = ofx.FxHost(blocks, nbr, _params(limiter))
    whole.torus_init()
    for _ in range(steps):
        whole.step()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d, kind, limiter, steps), nprocs=world, join=True,
                           start_method="spawn")
        parts = [np.load(os.path.join(d, f"r{r}.npy"), allow_pickle=True).item() for r in range(world)]
    seen = np.concatenate([sorted(p["U"]) for p in parts])
    assert np.array_equal(np.sort(seen), np.arange(len(blocks)))
    n_int = 0
    for p in parts:
        assert p["ncell"] < p["whole"]                      # a rank holds less than the whole grid
        assert p["dt"][1] == whole.dt[1]
        for g in sorted(p["U"]):
            b = blocks[g]
            n, off = int(b["n"]), int(b["off"])
            S, G = n + 7, 3
            for name, arr in (("U", p["U"][g]), ("Bf", p["Bf"][g])):
                ref = getattr(whole, name)[:, off:off + box_size(n)].reshape(-1, S, S, S)[:, G:G + n, G:G + n, G:G + n]
                got = arr.reshape(-1, S, S, S)[:, G:G + n, G:G + n, G:G + n]
                assert np.array_equal(got, ref), (name, int(g))
            n_int += n ** 3
    assert n_int == sum(int(n) ** 3 for n in blocks["n"])
