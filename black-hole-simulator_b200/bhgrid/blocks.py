"""Block tables of the corrected scheme's grid (include/bhgpu.h, bh_fx_grid).

Pure numpy: the block table (n, level, offset of the block's (n+5)^3 box,
lower corner, spacing), the 27-neighbour table used by the ghost fill and the
work lists (block, first index) the kernels walk.  The CPU oracle and the GPU
path build their grids from the same tables.
"""
from __future__ import annotations

import numpy as np

CHUNK = 128          # BH_FX_CHUNK: indices per work item (threads per CTA)

BLOCK_DTYPE = np.dtype([("n", "<i4"), ("level", "<i4"), ("off", "<i8"), ("x0", "<f8", 3), ("dx", "<f8")])
assert BLOCK_DTYPE.itemsize == 48


def box_size(n: int) -> int:
    """Entries of one block's box per array: cells -2 .. n+2 per axis."""
    return (n + 5) ** 3


def uniform_blocks(lo: float, hi: float, ncell: int, nblk: int, periodic: bool = False):
    """Block table and 27-neighbour table of a uniform grid of ncell^3 cells
    over the cube [lo, hi]^3 cut into blocks of nblk^3 cells; neighbour
    entry (ox+1)*9 + (oy+1)*3 + (oz+1) is the block at offset (ox, oy, oz),
    -1 outside the domain (outflow) unless periodic."""
    if ncell % nblk or nblk % 8:
        raise ValueError("the grid must be a whole number of blocks whose size is a multiple of 8")
    nb = ncell // nblk
    dx = (hi - lo) / ncell
    blocks = np.zeros(nb ** 3, BLOCK_DTYPE)
    nbr = np.full((nb ** 3, 27), -1, np.int32)
    off = 0
    for bi in range(nb):
        for bj in range(nb):
            for bk in range(nb):
                b = (bi * nb + bj) * nb + bk
                blocks[b]["n"] = nblk
                blocks[b]["off"] = off
                blocks[b]["x0"] = (lo + bi * nblk * dx, lo + bj * nblk * dx, lo + bk * nblk * dx)
                blocks[b]["dx"] = dx
                off += box_size(nblk)
                for ox in (-1, 0, 1):
                    for oy in (-1, 0, 1):
                        for oz in (-1, 0, 1):
                            q = [bi + ox, bj + oy, bk + oz]
                            if periodic:
                                q = [v % nb for v in q]
                            elif not all(0 <= v < nb for v in q):
                                continue
                            nbr[b, (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1)] = (q[0] * nb + q[1]) * nb + q[2]
    return blocks, nbr


def index_count(n: int, kind: str) -> int:
    return {"cell": n ** 3, "pos": (n + 2) ** 3, "ghost": (n + 4) ** 3 - n ** 3}[kind]


def work_items(blocks: np.ndarray, kind: str) -> np.ndarray:
    """(block, first index) pairs of CHUNK consecutive indices of each
    block's index space: 'cell' n^3, 'pos' (n+2)^3, 'ghost' (n+4)^3 - n^3."""
    out = []
    for b, n in enumerate(blocks["n"]):
        starts = np.arange(0, index_count(int(n), kind), CHUNK, dtype=np.int32)
        out.append(np.stack([np.full_like(starts, b), starts], 1))
    return np.concatenate(out).astype(np.int32)


def interior(blocks: np.ndarray, arr: np.ndarray) -> np.ndarray:
    """[..., nblock, n, n, n] interior cells of a [..., ncell] array (all
    blocks of one size)."""
    n = int(blocks["n"][0])
    S = n + 5
    out = []
    for b in blocks:
        box = arr[..., int(b["off"]):int(b["off"]) + S ** 3].reshape(arr.shape[:-1] + (S, S, S))
        out.append(box[..., 2:2 + n, 2:2 + n, 2:2 + n])
    return np.stack(out, axis=-4)
