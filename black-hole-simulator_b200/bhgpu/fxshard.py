"""The corrected scheme's block grid sharded over the ranks of a process
group (one process per GPU).

Each rank steps only the blocks it owns (``bhgrid.shard``: a Morton run of
the equal cubes, balanced by zones) and holds copies of the neighbouring
blocks whose boxes its ghost fill and EMF correction read -- its memory is
its share of the domain plus one layer of neighbouring blocks.  Within a
step the data that crosses ranks is:

    dt[0]   min over ranks after stage 0's con2prim         (all_reduce MIN)
    W, B~   the boxes of the neighbours' copies, before each ghost-fill pass
            (pass 0 reads interiors; pass l's prolongations read the coarse
            blocks' ghosts that pass l-1 filled on their owners)
    E       the copies' edge EMFs before the level-change correction
            (blocks of several levels only)

rk2integrator::step (solver/integrator.cpp:262-275) runs as the same pieces
as ``FxGrid.step`` with these exchanges between them, so each owned block
ends the step with the bits the whole grid stepped in one process gives it.
The exchanges are torch.distributed point-to-point calls: NCCL over NVLink
between GPUs, gloo through host memory in the CPU tests.
"""
from __future__ import annotations

import numpy as np
import torch

from bhgrid.blocks import box_size
from bhgrid.shard import exchange_plan, local_grid, partition_blocks


class ShardedFxGrid:
    """Steps the owned blocks of a local grid (``FxGrid`` built on
    ``bhgrid.shard.local_grid``'s tables with ``nactive`` = the owned
    blocks) in step with the other ranks."""

    def __init__(self, blocks: np.ndarray, nbr: np.ndarray, grid_factory, group=None, owner=None):
        """grid_factory(local_blocks, local_nbr, nactive, maxlevel) returns
        the rank's local grid: an object with arrays W, Bf, Bf1, E (torch
        tensors, or numpy arrays viewed as tensors), dt, and the pieces
        prims, ghost_pass, fluxes, update, emf_raw, update_from_emf (an
        ``FxGrid``)."""
        import torch.distributed as dist
        self.group = group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        self.owner = partition_blocks(blocks, self.world) if owner is None else np.asarray(owner, np.int32)
        self.maxlevel = int(blocks["level"].max())
        self.local = local_grid(blocks, nbr, self.owner, self.rank)
        self.grid = grid_factory(self.local.blocks, self.local.nbr, self.local.nown, self.maxlevel)
        self.global_blocks = blocks
        plan = exchange_plan(blocks, nbr, self.owner, self.rank)
        dev = self._t("W").device
        self._peers = [(p, self._box_index(s, dev), self._box_index(r, dev)) for p, (s, r) in plan.items()]

    def _box_index(self, local_ids, device):
        """flat entries of the boxes of local blocks, per component count"""
        lb = self.local.blocks
        n = self.local.ncell
        one = (np.concatenate([int(lb["off"][b]) + np.arange(box_size(int(lb["n"][b]))) for b in local_ids])
               if len(local_ids) else np.zeros(0, np.int64))
        return {C: torch.as_tensor((np.arange(C)[:, None] * n + one[None, :]).reshape(-1), device=device)
                for C in (3, 8)}

    def _t(self, name):
        a = getattr(self.grid, name)
        return a if isinstance(a, torch.Tensor) else torch.from_numpy(a)

    def _exchange(self, names):
        import torch.distributed as dist
        ops, inbox = [], []
        for name in names:
            a = self._t(name)
            flat = a.view(-1)
            C = a.shape[0]
            for peer, send, recv in self._peers:
                si, ri = send[C], recv[C]
                if si.numel():
                    ops.append(dist.P2POp(dist.isend, flat.index_select(0, si), peer, self.group))
                if ri.numel():
                    buf = torch.empty(ri.numel(), dtype=a.dtype, device=a.device)
                    ops.append(dist.P2POp(dist.irecv, buf, peer, self.group))
                    inbox.append((flat, ri, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for flat, ri, buf in inbox:
            flat.index_copy_(0, ri, buf)

    def step(self):
        """One RK2 step of the owned blocks (every rank calls it)."""
        import torch.distributed as dist
        g = self.grid
        for stage in (0, 1):
            g.prims(stage, with_dt=stage == 0)
            if stage == 0:
                dt = self._t("dt")[:1]
                if dt.device.type == "cuda" and dist.get_backend(self.group) == "gloo":
                    h = dt.cpu()
                    dist.all_reduce(h, op=dist.ReduceOp.MIN, group=self.group)
                    dt.copy_(h)
                else:
                    dist.all_reduce(dt, op=dist.ReduceOp.MIN, group=self.group)
            face = "Bf1" if stage else "Bf"
            for pass_ in range(self.maxlevel + 1):
                self._exchange(("W", face))
                g.ghost_pass(stage, pass_)
            g.fluxes(stage)
            if self.maxlevel > 0:
                g.emf_raw()
                self._exchange(("E",))
                g.update_from_emf(stage)
            else:
                g.update(stage)

    # ---- moving whole-domain states in and out ----------------------------
    def scatter(self, name: str, full):
        """Set array ``name`` of the local grid (owned blocks and copies) from
        the whole-domain array ``full`` ([C][ncell of the global grid])."""
        a = self._t(name)
        f = full if isinstance(full, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(full))
        gb, lb = self.global_blocks, self.local.blocks
        for l, g in enumerate(self.local.glob):
            box = box_size(int(lb["n"][l]))
            go, lo = int(gb["off"][g]), int(lb["off"][l])
            a[:, lo:lo + box].copy_(f[:, go:go + box].to(a.dtype))

    def owned_boxes(self, name: str) -> dict:
        """{global block: its box of array ``name``} of the owned blocks
        (numpy, float64)."""
        a = self._t(name)
        lb = self.local.blocks
        out = {}
        for l in range(self.local.nown):
            box = box_size(int(lb["n"][l]))
            lo = int(lb["off"][l])
            out[int(self.local.glob[l])] = a[:, lo:lo + box].double().cpu().numpy()
        return out
