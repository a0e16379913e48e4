"""Sharded stepping (bhgpu.shard) on world_size-2 gloo process groups, on
the CPU: the partition, the halo plan and the exchange, with the oracle
doing each rank's arithmetic.  Every rank poisons (NaN) the patches it does
not own before each stage, so whatever its owned patches read from another
rank's patches can only have arrived through the halo exchange; the
owned patches gathered from both ranks must equal the single-process step
bit for bit."""
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from bhgpu.mesh import Quilt
from bhgpu.shard import halo_plan, partition


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_path, steps):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "black-hole-simulator_b200"))
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist
    from helpers import box_case
    from bhgpu.shard import HaloExchange, halo_plan, partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        q, orc, hp = box_case(2, seed=4, periodic=True, lim=0)
        T = q.tables()
        owner = partition(q, world)
        mine = owner == rank
        hx = HaloExchange(halo_plan(T["nbr"], T["leaf"], owner, rank), "cpu", stage_on_host=True)
        U, W = torch.from_numpy(hp.U), torch.from_numpy(hp.W)

        def poison():
            for a in (hp.U, hp.W, hp.dU, hp.Bf, hp.F, hp.EMF):
                a[~mine] = np.nan
        for _ in range(steps):
            poison()
            dt = torch.tensor([orc.dtcomp(hp, 0.4)], dtype=torch.float64)
            dist.all_reduce(dt, op=dist.ReduceOp.MIN)
            for stage in (0, 1):
                hx.exchange(U, W)
                orc.rkstg(hp, float(dt.item()), stage)
                poison()
            orc.floors(hp)
        got = torch.from_numpy(np.where(mine[:, None, None], hp.U, 0.0))
        dist.all_reduce(got)
        if rank == 0:
            np.save(out_path, got.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("steps", [1, 2])
def test_sharded_steps_equal_single_process(steps):
    from helpers import box_case
    q, orc, hp = box_case(2, seed=4, periodic=True, lim=0)
    for _ in range(steps):
        orc.step(hp, 0.4)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "u.npy")
        mp.start_processes(_worker, args=(2, _free_port(), out, steps), nprocs=2, join=True, start_method="spawn")
        got = np.load(out)
    assert np.array_equal(np.isnan(got), np.isnan(hp.U))
    assert np.array_equal(np.nan_to_num(got, nan=7.0), np.nan_to_num(hp.U, nan=7.0))


def test_partition_and_plan_are_consistent():
    q = Quilt([10.0] * 3, [12.0] * 3, 4, periodic=True)
    T = q.tables()
    for world in (2, 3, 8):
        owner = partition(q, world)
        counts = np.bincount(owner, minlength=world)
        assert counts.max() - counts.min() <= 1
        plans = [halo_plan(T["nbr"], T["leaf"], owner, r) for r in range(world)]
        for a in range(world):
            for b, (send, recv) in plans[a].items():
                assert np.array_equal(send, plans[b][a][1]) and np.array_equal(recv, plans[b][a][0])
                assert (owner[send // 8000] == a).all() and (owner[recv // 8000] == b).all()
