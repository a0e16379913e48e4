"""One AMR domain sharded over ranks (one process per GPU).

The reference steps its whole quilt in one process (OpenMP over patches,
integrator.cpp:191-275).  Here the leaf patches are split over ranks along
a Morton curve; every rank keeps the whole pool but advances only the
patches it owns, and the only data a rank needs from others within a step
are the interior cells its ghost strips copy from neighbours it does not own
(gh_copy, grid.cpp:390-425) and the time step, a minimum over all leaves
(dtcomp, integrator.cpp:156-189).  So a step is:

    dt = min over ranks of dtcomp(owned leaves)          (all_reduce MIN)
    for stage in 0, 1:
        halo exchange: the source strips of U and W      (point to point)
        rkstg(stage) on the owned patches
    floors on the owned patches

Each exchanged strip is the two interior layers of a patch next to one face
(512 cells, 8 conserved and 8 primitive values each), written into the
receiver's copy of the owner's patch at the same cells, where the ghost
fill reads them.  Con2prim reuse by ghost cells stays within a rank (the
leaf mask handed to the kernels marks owned leaves only).  Coarse-to-fine
prolongation from a patch owned by another rank is not supported: the
partition must keep such pairs together (``halo_plan`` raises otherwise).

The exchange goes through torch.distributed point-to-point calls, so it
runs on NCCL over NVLink between GPUs, and on gloo (host memory) in the
tests, with the same plan.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .mesh import BLOCK, CPN, GHOST, NB_COPY, NB_PROLONG, NC, Quilt


def _morton(ijk, lvl, max_lvl):
    """Morton code of a patch's origin on the finest level's index grid."""
    s = 1 << (max_lvl - lvl)
    x, y, z = (int(c) * s for c in ijk)
    code = 0
    for b in range(21):
        code |= ((x >> b) & 1) << (3 * b + 2) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b)
    return code


def partition(quilt: Quilt, world: int) -> np.ndarray:
    """owner[npatch]: the leaves in Morton order cut into ``world`` runs of
    equal length (all patches have 16^3 cells); a non-leaf patch goes with
    its first child's owner, or rank 0."""
    T = quilt.tables()
    n = len(quilt)
    leaves = [p for p in range(n) if T["leaf"][p]]
    max_lvl = int(T["lvl"].max()) if n else 0
    order = sorted(leaves, key=lambda p: _morton(T["ijk"][p], T["lvl"][p], max_lvl))
    owner = np.zeros(n, np.int32)
    for i, p in enumerate(order):
        owner[p] = min(world - 1, i * world // max(len(order), 1))
    for p in range(n - 1, -1, -1):           # children come after their parents in the quilt
        P = quilt.patches[p]
        if not P.leaf:
            kids = [c for c in P.children if c >= 0]
            owner[p] = owner[kids[0]] if kids else 0
    return owner


def _strip_cells(dim, side):
    """Linear indices of the 512 interior cells a neighbour's ghost strip on
    face (dim, side) of the *receiving* patch copies, in the source patch
    (gh_copy's source layers, grid.cpp:399-422)."""
    start = 0 if side == 1 else BLOCK - GHOST
    out = []
    for gg in range(GHOST):
        for t1 in range(BLOCK):
            for t2 in range(BLOCK):
                ijk = [t1, t2]
                ijk.insert(dim, start + gg)
                i, j, k = ijk
                out.append((i + GHOST) * CPN * CPN + (j + GHOST) * CPN + (k + GHOST))
    return np.array(out, np.int64)


_STRIPS = {(d, s): _strip_cells(d, s) for d in range(3) for s in (-1, 1)}


def halo_plan(nbr: np.ndarray, leaf: np.ndarray, owner: np.ndarray, rank: int):
    """{peer: (send, recv)} of flat cell indices (patch * 8000 + cell): the
    cells of this rank's patches that ``peer``'s ghost strips copy, and the
    cells of ``peer``'s patches this rank's ghost strips copy."""
    n = len(owner)
    need = {}                               # (receiver, source owner) -> set of flat cells
    for p in range(n):
        if not leaf[p]:
            continue
        for s in range(6):
            q, kind = int(nbr[p, s, 0]), int(nbr[p, s, 1])
            if q < 0 or owner[q] == owner[p]:
                continue
            if kind == NB_PROLONG:
                raise NotImplementedError(f"patch {p} (rank {owner[p]}) prolongs from patch {q} (rank {owner[q]}); "
                                          "keep coarse-fine neighbours on one rank")
            if kind != NB_COPY:
                continue
            dim, side = s // 2, (1 if s & 1 else -1)
            cells = q * NC + _STRIPS[(dim, side)]
            need.setdefault((int(owner[p]), int(owner[q])), set()).update(cells.tolist())
    plan = {}
    for (recv_rank, src_rank), cells in need.items():
        idx = np.array(sorted(cells), np.int64)
        if src_rank == rank:
            plan.setdefault(recv_rank, [np.zeros(0, np.int64), np.zeros(0, np.int64)])[0] = idx
        if recv_rank == rank:
            plan.setdefault(src_rank, [np.zeros(0, np.int64), np.zeros(0, np.int64)])[1] = idx
    return {peer: (s, r) for peer, (s, r) in sorted(plan.items())}


class HaloExchange:
    """Moves the planned cells of U and W ([npatch, 8, 8000] each) between
    ranks.  ``stage_on_host`` packs through host memory (gloo); otherwise the
    buffers stay on the arrays' device (NCCL)."""

    def __init__(self, plan: dict, device, stage_on_host: bool = False, group=None):
        self.group = group
        self.host = stage_on_host
        self.device = torch.device(device)
        self.peers = []
        for peer, (send, recv) in plan.items():
            # [8 components] x cells: flat offsets of component v of cell (patch, l) = (patch*8 + v)*NC + l
            def comp_index(flat):
                pt, l = flat // NC, flat % NC
                v = np.arange(8)[:, None]
                return torch.as_tensor(((pt[None, :] * 8 + v) * NC + l[None, :]).reshape(-1), device=self.device)
            self.peers.append((peer, comp_index(send), comp_index(recv), len(send), len(recv)))

    def exchange(self, U: torch.Tensor, W: torch.Tensor):
        import torch.distributed as dist
        Uf, Wf = U.view(-1), W.view(-1)
        ops, inbox = [], []
        for peer, si, ri, ns, nr in self.peers:
            if ns:
                buf = torch.cat([Uf.index_select(0, si), Wf.index_select(0, si)])
                if self.host:
                    buf = buf.cpu()
                ops.append(dist.P2POp(dist.isend, buf, peer, self.group))
            if nr:
                rb = torch.empty(16 * nr, dtype=U.dtype, device="cpu" if self.host else U.device)
                ops.append(dist.P2POp(dist.irecv, rb, peer, self.group))
                inbox.append((ri, rb))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for ri, rb in inbox:
            rb = rb.to(U.device)
            n = ri.numel()
            Uf.index_copy_(0, ri, rb[:n])
            Wf.index_copy_(0, ri, rb[n:])


class ShardedStepper:
    """rk2integrator::step of one AmrTree sharded over the ranks of the
    default process group (every rank holds the same tree and state)."""

    def __init__(self, tree, cfl: float = 0.4, owner: np.ndarray | None = None, group=None):
        import torch.distributed as dist
        from .solver import BhPool, _p
        self.tree, self.cfl, self.group = tree, float(cfl), group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        T = tree.tables
        self.owner = partition(tree.quilt, self.world) if owner is None else np.asarray(owner, np.int32)
        if tree.nwave > 1:
            for p in np.nonzero(T["leaf"])[0]:
                for s in range(6):
                    q, kind = T["nbr"][p, s]
                    if kind == NB_PROLONG and self.owner[q] != self.owner[p]:
                        raise NotImplementedError("coarse-fine neighbours must share a rank")
        mine = self.owner == self.rank
        d = tree.device
        self.all_mine = torch.as_tensor(np.nonzero(mine)[0].astype(np.int32), device=d)
        leaves = np.nonzero(mine & (T["leaf"] != 0))[0].astype(np.int32)
        self.leaves_mine = torch.as_tensor(leaves, device=d)
        self.leafmask_mine = torch.as_tensor((mine & (T["leaf"] != 0)).astype(np.uint8), device=d)
        backend = dist.get_backend(group)
        self.halo = HaloExchange(halo_plan(T["nbr"], T["leaf"], self.owner, self.rank), d,
                                 stage_on_host=(backend == "gloo"), group=group)
        t = tree
        self.pool = BhPool(t.npatch, _p(t.U), _p(t.W), _p(t.dU), _p(t.F), _p(t.Bf), _p(t.EMF), _p(t.rth),
                           _p(t.pgeo), _p(t.nbr), _p(self.all_mine), _p(self.leaves_mine), len(leaves), _p(t.err),
                           _p(self.leafmask_mine), _p(t.status), _p(t.aux), _p(t.Wd), len(self.all_mine))
        # waves restricted to owned leaves (one wave: the fused ghost fill + con2prim)
        off = t._wave_off
        lists = [t.waves[off[w]:off[w + 1]].cpu().numpy() for w in range(t.nwave)]
        lists = [l_[mine[l_]] for l_ in lists]
        self.nwave = len(lists)
        woff = np.zeros(self.nwave + 1, np.int32)
        for w, l_ in enumerate(lists):
            woff[w + 1] = woff[w] + len(l_)
        self._wave_off = woff
        self.waves = torch.as_tensor(np.concatenate(lists).astype(np.int32) if lists else np.zeros(0, np.int32),
                                     device=d)

    def step(self):
        """One RK2 step; returns dt (float)."""
        import torch.distributed as dist
        from .solver import _p, _stream, check, lib
        t = self.tree
        P = t.params()
        s = _stream()
        check(lib.bh_dtcomp(C.byref(P), C.byref(self.pool), self.cfl, _p(t.dt), s), "rk2integrator::dtcomp")
        dt = t.dt.cpu() if dist.get_backend(self.group) == "gloo" else t.dt
        dist.all_reduce(dt, op=dist.ReduceOp.MIN, group=self.group)
        t.dt.copy_(dt)
        offp = self._wave_off.ctypes.data_as(C.c_void_p)
        for stage in (0, 1):
            self.halo.exchange(t.U, t.W)
            check(lib.bh_rkstg(C.byref(P), C.byref(self.pool), _p(t.dt), stage, _p(self.waves), offp, self.nwave, s),
                  "rk2integrator::rkstg")
        check(lib.bh_floors(C.byref(P), C.byref(self.pool), s), "patch::floors")
        return float(t.dt.item())

    def gather(self, name: str = "U") -> torch.Tensor:
        """The full array with every patch taken from its owner (all ranks)."""
        import torch.distributed as dist
        x = getattr(self.tree, name)
        mine = torch.as_tensor(self.owner == self.rank, device=x.device).view(-1, *([1] * (x.dim() - 1)))
        y = torch.where(mine, x, torch.zeros_like(x))
        if dist.get_backend(self.group) == "gloo":
            y = y.cpu()
        dist.all_reduce(y, group=self.group)
        return y
