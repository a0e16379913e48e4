"""bhgpu.shard.ShardedStepper with the CUDA kernels: two ranks (processes)
on the one GPU of this test, exchanging halos through a gloo group in host
memory -- no kernel of one rank waits on another rank's, the ranks only
meet in host-side collectives.  Two sharded steps of a 4^3-patch periodic
box equal two single-process steps bit for bit: a rank computes its own
patches with the same arithmetic, and a ghost cell copied from another
rank's patch runs its two con2prim passes instead of reusing the source's
outcome, which gives the same primitives."""
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _box():
    import bhgpu
    from bhgpu import configs
    from bhgpu.mesh import Quilt
    q = Quilt([10.0] * 3, [12.0] * 3, 4, periodic=True)
    tree = bhgpu.AmrTree(q.dom_l, q.dom_h, 4, M=0.0, a=0.0, Q=0.0, gm=4.0 / 3.0, periodic=True, limiter="minmod",
                         quilt=q, init_floor=False)
    W, Bf = configs.magnetised_box(q, seed=2, gamma=4.0 / 3.0)
    tree.load(W=W, Bf=Bf)
    tree.prim_to_cons()
    return tree


def _worker(rank, world, port, out_path):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "black-hole-simulator_b200"))
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from bhgpu.shard import ShardedStepper
        tree = _box()
        st = ShardedStepper(tree, 0.4)
        for _ in range(2):
            st.step()
        U = st.gather("U")
        if rank == 0:
            np.save(out_path, U.cpu().numpy())
    finally:
        dist.destroy_process_group()


def test_sharded_steps_equal_single_process_on_the_device():
    import bhgpu
    tree = _box()
    rk = bhgpu.RK2Integrator(0.4)
    for _ in range(2):
        rk.step(tree, check_domain=False)
    want = tree.U.cpu().numpy()
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "u.npy")
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        got = np.load(out)
    assert np.array_equal(np.nan_to_num(got, nan=7.0), np.nan_to_num(want, nan=7.0))
