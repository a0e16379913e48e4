"""A block grid of the corrected scheme cut over ranks (pure numpy).

Each rank owns a run of blocks along a Morton curve of the equal cubes
(balanced by zones) and keeps, besides its own blocks, copies of the blocks
its blocks' ghost fill and EMF correction read: every block in their
27-neighbourhoods.  Its local grid lists the owned blocks first (the work
lists cover only those) and the neighbours' copies after them, each with a
box of its own; so a rank's memory is its blocks plus one layer of
neighbouring blocks, not the whole domain.

The copies are refreshed by whole-box exchanges (bhgpu.fxshard): rank r
sends to rank p the boxes of r's blocks that p keeps as copies, and receives
the boxes of p's blocks that r keeps -- both lists in global block order, so
the two sides agree without a handshake.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .blocks import box_size


def cube_coords(blocks: np.ndarray) -> np.ndarray:
    """[nblock, 3] integer coordinates of the equal cubes (the blocks' lower
    corners over the cube size)."""
    size = blocks["n"] * blocks["dx"]
    lo = blocks["x0"].min(0)
    return np.rint((blocks["x0"] - lo) / size[:, None]).astype(np.int64)


def _morton(c: np.ndarray) -> np.ndarray:
    code = np.zeros(len(c), np.int64)
    for b in range(20):
        for d in range(3):
            code |= ((c[:, d] >> b) & 1) << (3 * b + 2 - d)
    return code


def partition_blocks(blocks: np.ndarray, world: int) -> np.ndarray:
    """owner[nblock]: the cubes in Morton order cut into ``world`` runs of
    nearly equal zone counts (n^3 per block)."""
    order = np.argsort(_morton(cube_coords(blocks)), kind="stable")
    zones = blocks["n"][order].astype(np.int64) ** 3
    # the rank of a block: where the midpoint of its zones falls
    mid = np.cumsum(zones) - zones / 2.0
    rank = np.minimum((mid * world / zones.sum()).astype(np.int64), world - 1)
    owner = np.empty(len(blocks), np.int32)
    owner[order] = rank
    return owner


@dataclass
class LocalGrid:
    blocks: np.ndarray    # local block table: owned blocks, then neighbours' copies (own offsets)
    nbr: np.ndarray       # local 27-neighbour table (rows of the copies: themselves only)
    glob: np.ndarray      # global index of each local block
    nown: int             # the first nown local blocks are owned

    @property
    def ncell(self) -> int:
        return int(sum(box_size(int(n)) for n in self.blocks["n"]))


def local_grid(blocks: np.ndarray, nbr: np.ndarray, owner: np.ndarray, rank: int) -> LocalGrid:
    own = np.nonzero(owner == rank)[0]
    near = np.unique(nbr[own].ravel())
    halo = np.setdiff1d(near[near >= 0], own)
    glob = np.concatenate([own, halo]).astype(np.int64)
    g2l = np.full(len(blocks), -1, np.int64)
    g2l[glob] = np.arange(len(glob))
    lb = blocks[glob].copy()
    sizes = np.array([box_size(int(n)) for n in lb["n"]], np.int64)
    lb["off"] = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    ln = np.full((len(glob), 27), -1, np.int32)
    rows = nbr[own]
    ln[:len(own)] = np.where(rows >= 0, g2l[np.maximum(rows, 0)], -1)
    ln[np.arange(len(own), len(glob)), 13] = np.arange(len(own), len(glob))
    assert (ln[:len(own)][rows >= 0] >= 0).all()
    return LocalGrid(lb, ln, glob, len(own))


def exchange_plan(blocks: np.ndarray, nbr: np.ndarray, owner: np.ndarray, rank: int) -> dict:
    """{peer: (send, recv)}: local indices (in this rank's local grid) of the
    owned blocks whose boxes go to ``peer`` and of the copies whose boxes
    come from it, both in global block order."""
    world = int(owner.max()) + 1
    mine = local_grid(blocks, nbr, owner, rank)
    g2l = {int(g): i for i, g in enumerate(mine.glob)}
    plan = {}
    for peer in range(world):
        if peer == rank:
            continue
        theirs = local_grid(blocks, nbr, owner, peer)
        sent = sorted(int(g) for g in theirs.glob[theirs.nown:] if owner[g] == rank)
        got = sorted(int(g) for g in mine.glob[mine.nown:] if owner[g] == peer)
        if sent or got:
            plan[peer] = (np.array([g2l[g] for g in sent], np.int64), np.array([g2l[g] for g in got], np.int64))
    return plan
