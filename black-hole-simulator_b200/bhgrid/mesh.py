"""Host-side patch quilt: geometry, neighbour table and ghost-fill order.

This is the mesh bookkeeping of ``grid::amrtree`` (src/fluid/grid/grid.cpp)
restated on the host in numpy.  It never touches cell data: it produces the
small per-patch tables (corners, edge origin and spacing, level, octree
index, leaf flag, neighbour slots) that the CUDA kernels consume.

Floating-point expressions follow the reference's evaluation order so that
patch edges and spacings are bit-identical to the reference's
(``patch::patch``, grid.cpp:19-48; ``amrtree::refine``, grid.cpp:574-600).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BLOCK = 16          # grid.hpp:19
GHOST = 2           # grid.hpp:20
CPN = BLOCK + 2 * GHOST
NC = CPN ** 3                 # cells per patch incl. ghosts
NF = (CPN + 1) * CPN * CPN    # faces per direction
NE = CPN * (CPN + 1) * (CPN + 1)  # edges per direction

# neighbour kinds of amrtree::ghosts (grid.cpp:528-534)
NB_BNDY, NB_COPY, NB_PROLONG = 0, 1, 2


@dataclass
class Patch:
    lvl: int
    ijk: tuple
    cor1: tuple
    cor2: tuple
    parent: int = -1
    children: list = field(default_factory=lambda: [-1] * 8)
    leaf: bool = True

    def edge(self, d: int, i: int) -> float:
        """xedge/yedge/zedge[i] exactly as patch::patch builds them (grid.cpp:24-29)."""
        k = float(i) / BLOCK
        return self.cor1[d] + k * (self.cor2[d] - self.cor1[d])

    def origin_spacing(self):
        e0 = [self.edge(d, 0) for d in range(3)]
        sp = [self.edge(d, 1) - e0[d] for d in range(3)]   # patch::dx (grid.cpp:128-130)
        return e0, sp


@dataclass
class RegridPlan:
    """What one regrid does to the pool, in the indices of the extended
    quilt (the old patches, then the children appended by refinement):

    refined:   (parent, [8 children]) per refined patch
    flattened: (parent, [8 children]) per flattened patch
    keep:      extended indices that remain, in the new quilt order
    ext_pgeo:  [n_ext, 6] corners and spacings of the extended quilt
    """
    n_old: int
    n_ext: int
    ext_pgeo: np.ndarray
    refined: list
    flattened: list
    keep: np.ndarray

    @property
    def changed(self) -> bool:
        return bool(self.refined or self.flattened)


class Quilt:
    """The patch list of ``amrtree`` (``quilt``, grid.hpp:119), in quilt order.

    ``periodic`` wraps same-level neighbour search at the domain edge (the
    reference has only copy-outflow boundaries; periodic wrap is the
    boundary condition of the uniform magnetised-box workload).
    """

    def __init__(self, dom_l, dom_h, nqlt: int, periodic: bool = False):
        self.dom_l = tuple(float(x) for x in dom_l)
        self.dom_h = tuple(float(x) for x in dom_h)
        self.nqlt = int(nqlt)
        self.periodic = bool(periodic)
        self.patches: list[Patch] = []
        px = [(self.dom_h[d] - self.dom_l[d]) / self.nqlt for d in range(3)]  # grid.cpp:180
        for i in range(self.nqlt):
            for j in range(self.nqlt):
                for k in range(self.nqlt):
                    c1 = (self.dom_l[0] + i * px[0], self.dom_l[1] + j * px[1], self.dom_l[2] + k * px[2])
                    c2 = (c1[0] + px[0], c1[1] + px[1], c1[2] + px[2])
                    self.patches.append(Patch(0, (i, j, k), c1, c2))

    def __len__(self):
        return len(self.patches)

    # ------------------------------------------------------------------
    def refine(self, p: int) -> list[int]:
        """Geometry of amrtree::refine (grid.cpp:574-600): eight children
        appended to the quilt in octant order; cell data is not touched."""
        P = self.patches[p]
        if not P.leaf:
            return []
        lo = [P.edge(d, 0) for d in range(3)]
        hi = [P.edge(d, BLOCK) for d in range(3)]
        mid = [(lo[d] + hi[d]) / 2 for d in range(3)]
        kids = []
        for h in range(8):
            ix, iy, iz = (h >> 2) & 1, (h >> 1) & 1, h & 1
            c1 = (mid[0] if ix else lo[0], mid[1] if iy else lo[1], mid[2] if iz else lo[2])
            c2 = (hi[0] if ix else mid[0], hi[1] if iy else mid[1], hi[2] if iz else mid[2])
            cijk = (2 * P.ijk[0] + ix, 2 * P.ijk[1] + iy, 2 * P.ijk[2] + iz)
            self.patches.append(Patch(P.lvl + 1, cijk, c1, c2, parent=p))
            P.children[h] = len(self.patches) - 1
            kids.append(len(self.patches) - 1)
        P.leaf = False
        return kids

    # ------------------------------------------------------------------
    def regrid(self, flags) -> "RegridPlan":
        """Patch bookkeeping of amrtree::regrid (grid.cpp:722-835) given the
        per-patch flags of its cell loop (bit 0: refine, bit 1: erase; the
        flags of non-leaf patches are ignored).

        Leaves flagged for refinement are refined in quilt order, their
        children appended (refine, :574-600); then every leaf flagged for
        erasure whose parent is not a leaf and whose siblings are all leaves
        flattens that parent (:827-834).  The reference keeps raw pointers
        to children that an earlier flatten of the same parent has already
        destroyed; the only consistent reading of its loop is that each
        parent is flattened at most once, which is what happens here.
        Flattened children leave the quilt with the order of the others
        kept (std::remove_if, :722-726).  Returns the plan the data
        operations follow, in the indices of the quilt before removal."""
        flags = np.asarray(flags)
        n_old = len(self.patches)
        rfn = [p for p in range(n_old) if self.patches[p].leaf and flags[p] & 1]
        flt = [p for p in range(n_old) if self.patches[p].leaf and flags[p] & 2]
        refined = [(p, self.refine(p)) for p in rfn]
        ext_pgeo = self._pgeo()
        flattened, removed = [], set()
        for p in flt:
            par = self.patches[p].parent
            if par < 0 or self.patches[par].leaf:
                continue
            kids = self.patches[par].children
            if any(c >= 0 and not self.patches[c].leaf for c in kids):
                continue
            flattened.append((par, list(kids)))
            removed.update(c for c in kids if c >= 0)
            self.patches[par].children = [-1] * 8
            self.patches[par].leaf = True
        keep = np.array([q for q in range(len(self.patches)) if q not in removed], np.int64)
        new_of = {int(q): i for i, q in enumerate(keep)}
        self.patches = [self.patches[q] for q in keep]
        for P in self.patches:
            P.parent = new_of.get(P.parent, -1) if P.parent >= 0 else -1
            P.children = [new_of.get(c, -1) if c >= 0 else -1 for c in P.children]
        return RegridPlan(n_old, len(ext_pgeo), ext_pgeo, refined, flattened, keep)

    def _pgeo(self) -> np.ndarray:
        pgeo = np.zeros((len(self.patches), 6), np.float64)
        for p, P in enumerate(self.patches):
            e0, sp = P.origin_spacing()
            pgeo[p, :3] = e0
            pgeo[p, 3:] = sp
        return pgeo

    # ------------------------------------------------------------------
    def nbhd(self, p: int, dim: int, side: int) -> int:
        """amrtree::nbhd (grid.cpp:361-386): same-level patch first, then the
        coarser one, else -1 (domain boundary)."""
        P = self.patches[p]
        nb = list(P.ijk)
        nb[dim] += side
        if self.periodic and P.lvl == 0:
            nb[dim] %= self.nqlt
        nb = tuple(nb)
        for q, Q in enumerate(self.patches):
            if Q.lvl == P.lvl and Q.ijk == nb:
                return q
        if P.lvl > 0:
            crs = [x // 2 for x in P.ijk]
            crs[dim] += side
            crs = tuple(crs)
            for q, Q in enumerate(self.patches):
                if Q.lvl == P.lvl - 1 and Q.ijk == crs:
                    return q
        return -1

    def tables(self):
        """Per-patch tables consumed by the kernels."""
        n = len(self.patches)
        pgeo = np.zeros((n, 6), np.float64)
        lvl = np.zeros(n, np.int32)
        ijk = np.zeros((n, 3), np.int32)
        leaf = np.zeros(n, np.uint8)
        nbr = np.zeros((n, 6, 2), np.int32)
        for p, P in enumerate(self.patches):
            e0, sp = P.origin_spacing()
            pgeo[p, :3] = e0
            pgeo[p, 3:] = sp
            lvl[p] = P.lvl
            ijk[p] = P.ijk
            leaf[p] = 1 if P.leaf else 0
            for dim in range(3):
                for s, side in enumerate((-1, 1)):
                    q = self.nbhd(p, dim, side)
                    if q < 0:
                        nbr[p, dim * 2 + s] = (-1, NB_BNDY)
                    elif self.patches[q].lvl == P.lvl:
                        nbr[p, dim * 2 + s] = (q, NB_COPY)
                    else:
                        nbr[p, dim * 2 + s] = (q, NB_PROLONG)
        return dict(pgeo=pgeo, lvl=lvl, ijk=ijk, leaf=leaf, nbr=nbr)

    def ghost_waves(self, nbr: np.ndarray, leaf: np.ndarray) -> list[np.ndarray]:
        """Order of the ghost fill.

        The reference fills leaf patches one after another in quilt order
        (integrator.cpp:194-200).  A prolongation reads the coarse
        neighbour's cells including its ghost layer (grid.cpp:449-476), so
        it must see that layer as the serial order would: filled if the
        coarse patch comes earlier in the quilt, not yet filled otherwise.
        Patches are grouped into waves; every dependency goes from a lower
        to a higher quilt index, and each wave can run in parallel.
        """
        n = len(self.patches)
        wave = np.zeros(n, np.int64)
        readers = {q: [] for q in range(n)}
        for p in range(n):
            for s in range(6):
                q, kind = nbr[p, s]
                if kind == NB_PROLONG and leaf[p]:
                    readers[q].append(p)
        for p in range(n):
            if not leaf[p]:
                continue
            deps = []
            for s in range(6):
                q, kind = nbr[p, s]
                if kind == NB_PROLONG and q < p and leaf[q]:
                    deps.append(q)
            deps += [r for r in readers[p] if r < p]
            wave[p] = 1 + max((wave[d] for d in deps), default=-1)
        leaves = [p for p in range(n) if leaf[p]]
        if not leaves:
            return []
        nw = int(max(wave[p] for p in leaves)) + 1
        return [np.array([p for p in leaves if wave[p] == w], np.int32) for w in range(nw)]


def cell_index(i, j, k):
    """patch::lindx (grid.cpp:51-53): i slowest, k fastest, ghosts included."""
    return (i + GHOST) * CPN * CPN + (j + GHOST) * CPN + (k + GHOST)


def xface_index(i, j, k):   # patch::xfc_idx / Bfx_idx (grid.cpp:61-63, 72-74)
    return (i + GHOST) * CPN * CPN + (j + GHOST) * CPN + (k + GHOST)


def yface_index(i, j, k):   # patch::yfc_idx / Bfy_idx (grid.cpp:64-66, 75-77)
    return (i + GHOST) * (CPN + 1) * CPN + (j + GHOST) * CPN + (k + GHOST)


def zface_index(i, j, k):   # patch::zfc_idx / Bfz_idx (grid.cpp:67-69, 78-80)
    return (i + GHOST) * CPN * (CPN + 1) + (j + GHOST) * (CPN + 1) + (k + GHOST)


def interior_mask() -> np.ndarray:
    """Boolean [NC] mask of the 16^3 interior cells of a patch."""
    a = np.arange(CPN) - GHOST
    i, j, k = np.meshgrid(a, a, a, indexing="ij")
    m = (i >= 0) & (i < BLOCK) & (j >= 0) & (j < BLOCK) & (k >= 0) & (k < BLOCK)
    return m.reshape(-1)
