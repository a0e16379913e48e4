"""Block tables of the corrected scheme's grid (include/bhgpu.h, bh_fx_grid).

Pure numpy: the block table (n, level, offset of the block's (n+7)^3 box,
lower corner, spacing), the 27-neighbour table used by the ghost fill and the
work lists (block, first index) the kernels walk.  The CPU oracle and the GPU
path build their grids from the same tables.
"""
from __future__ import annotations

import numpy as np

CHUNK = 128          # BH_FX_CHUNK: indices per work item (threads per CTA)
GB = 3               # ghost layers of every block's box

BLOCK_DTYPE = np.dtype([("n", "<i4"), ("level", "<i4"), ("off", "<i8"), ("x0", "<f8", 3), ("dx", "<f8")])
assert BLOCK_DTYPE.itemsize == 48


def box_size(n: int) -> int:
    """Entries of one block's box per array: cells -3 .. n+3 per axis."""
    return (n + 2 * GB + 1) ** 3


def ghost_depth(limiter) -> int:
    """Ghost layers the fill covers: 3 for PPM's stencil, else 2."""
    return 3 if limiter in ("ppm", 3) else 2


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


def index_count(n: int, kind: str, depth: int = 2) -> int:
    return {"cell": n ** 3, "pos": (n + 2) ** 3, "ghost": (n + 2 * depth) ** 3 - n ** 3}[kind]


def work_items(blocks: np.ndarray, kind: str, depth: int = 2) -> np.ndarray:
    """(block, first index) pairs of CHUNK consecutive indices of each
    block's index space: 'cell' n^3, 'pos' (n+2)^3, 'ghost' (n+2 depth)^3 -
    n^3 (the shell of the depth ghost layers the fill covers)."""
    out = []
    for b, n in enumerate(blocks["n"]):
        starts = np.arange(0, index_count(int(n), kind, depth), CHUNK, dtype=np.int32)
        out.append(np.stack([np.full_like(starts, b), starts], 1))
    return np.concatenate(out).astype(np.int32)


# tiles of the staged flux kernel: TILE positions (i, j, k) per tile; blocks
# below TILE_MIN cells per axis keep chunks of positions (a tile box of n + 2
# positions per axis wastes up to (ceil((n+2)/T) T / (n+2)) of its threads)
TILE = (4, 4, 8)
TILE_MIN = 64


def flux_items(blocks: np.ndarray, tile_min: int = TILE_MIN) -> np.ndarray:
    """(block, e) work items of the staged flux kernel: e >= 0 is tile e of a
    block with n >= tile_min (tile (ti, tj, tk) -> (ti nj + tj) nk + tk over
    the position box [-1, n]^3), e < 0 the CHUNK positions from -(e + 1) on
    of a smaller block."""
    out = []
    for b, n in enumerate(blocks["n"]):
        n = int(n)
        m = n + 2
        if n >= tile_min:
            nt = -(-m // TILE[0]) * -(-m // TILE[1]) * -(-m // TILE[2])
            e = np.arange(nt, dtype=np.int32)
        else:
            e = -np.arange(0, m ** 3, CHUNK, dtype=np.int32) - 1
        out.append(np.stack([np.full_like(e, b), e], 1))
    return np.concatenate(out).astype(np.int32)


def flux_item_positions(n: int, e: int) -> np.ndarray:
    """Positions (i, j, k) in [-1, n]^3 that item e of a block of n cells
    covers (the kernel's decode; positions beyond n are masked)."""
    m = n + 2
    if e < 0:
        idx = np.arange(-(e + 1), min(-(e + 1) + CHUNK, m ** 3))
        return np.stack([idx // (m * m) - 1, (idx // m) % m - 1, idx % m - 1], 1)
    nj, nk = -(-m // TILE[1]), -(-m // TILE[2])
    o = (-1 + (e // (nj * nk)) * TILE[0], -1 + ((e // nk) % nj) * TILE[1], -1 + (e % nk) * TILE[2])
    g = np.stack(np.meshgrid(*[np.arange(o[d], o[d] + TILE[d]) for d in range(3)], indexing="ij"), -1).reshape(-1, 3)
    return g[(g <= n).all(1)]


def interior(blocks: np.ndarray, arr: np.ndarray) -> np.ndarray:
    """[..., nblock, n, n, n] interior cells of a [..., ncell] array (all
    blocks of one size)."""
    n = int(blocks["n"][0])
    S = n + 2 * GB + 1
    out = []
    for b in blocks:
        box = arr[..., int(b["off"]):int(b["off"]) + S ** 3].reshape(arr.shape[:-1] + (S, S, S))
        out.append(box[..., GB:GB + n, GB:GB + n, GB:GB + n])
    return np.stack(out, axis=-4)


def balanced_levels(level: np.ndarray) -> np.ndarray:
    """Raise cube levels until every pair of cubes that touch (faces, edges
    or corners) differ by at most one level (2:1 balance)."""
    lv = level.copy()
    nb = lv.shape[0]
    changed = True
    while changed:
        changed = False
        for i in range(nb):
            for j in range(nb):
                for k in range(nb):
                    m = lv[max(i - 1, 0):i + 2, max(j - 1, 0):j + 2, max(k - 1, 0):k + 2].max()
                    if lv[i, j, k] < m - 1:
                        lv[i, j, k] = m - 1
                        changed = True
    return lv


def leveled_blocks(lo: float, hi: float, level: np.ndarray, n0: int, periodic: bool = False):
    """Block table and 27-neighbour table of equal cubes over [lo, hi]^3, one
    block per cube, cube (i, j, k) holding (n0 2^level)^3 cells: a
    refinement level changes a cube's resolution, not its extent, so each
    block has exactly one neighbour per offset; levels must be 2:1 balanced."""
    nb = level.shape[0]
    if n0 % 2 or n0 < 4:
        raise ValueError("block sizes must be even and at least 4")
    L = (hi - lo) / nb
    blocks = np.zeros(nb ** 3, BLOCK_DTYPE)
    nbr = np.full((nb ** 3, 27), -1, np.int32)
    off = 0
    for bi in range(nb):
        for bj in range(nb):
            for bk in range(nb):
                b = (bi * nb + bj) * nb + bk
                n = n0 << int(level[bi, bj, bk])
                blocks[b]["n"] = n
                blocks[b]["level"] = level[bi, bj, bk]
                blocks[b]["off"] = off
                blocks[b]["x0"] = (lo + bi * L, lo + bj * L, lo + bk * L)
                blocks[b]["dx"] = L / n
                off += box_size(n)
                for ox in (-1, 0, 1):
                    for oy in (-1, 0, 1):
                        for oz in (-1, 0, 1):
                            q = [bi + ox, bj + oy, bk + oz]
                            if periodic:
                                q = [v % nb for v in q]
                            elif not all(0 <= v < nb for v in q):
                                continue
                            s = (q[0] * nb + q[1]) * nb + q[2]
                            if abs(int(level[q[0], q[1], q[2]]) - int(level[bi, bj, bk])) > 1:
                                raise ValueError("levels are not 2:1 balanced")
                            nbr[b, (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1)] = s
    return blocks, nbr


def torus_levels(nb: int = 8, lo: float = -40.0, hi: float = 40.0, r_fine=(14.0, 26.0), seed: int = 3,
                 jitter: float = 0.25):
    """Seeded uneven level map concentrated near the hole: with radii
    r_fine = (r_1, ..., r_L) in increasing order, a cube whose centre lies
    within r_l gets level L - l + 1 (the innermost the highest), beyond all
    of them level 0; a fraction `jitter` of the cubes moves one level up or
    down at random; then 2:1 balanced."""
    rng = np.random.default_rng(seed)
    L = (hi - lo) / nb
    c = lo + (np.arange(nb) + 0.5) * L
    R = np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2)
    top = len(r_fine)
    lv = np.zeros(R.shape, np.int64)
    for l, r in enumerate(sorted(r_fine, reverse=True)):
        lv = np.where(R < r, l + 1, lv)
    move = rng.random(lv.shape) < jitter
    step = rng.choice([-1, 1], size=lv.shape)
    lv = np.clip(np.where(move, lv + step, lv), 0, top)
    return balanced_levels(lv)
