"""Seeded synthetic workloads (host side, numpy).

No dataset is involved anywhere on this path: every input is generated here
from ``numpy.random.default_rng(seed)``.

* ``magnetised_box``: uniform magnetised gas on a uniform patch quilt --
  rho = 1, p = 0.1 (1 + 0.01 N(0,1)), v = 0, B = (0.5, 0.3, 0) + curl A with
  A a sum of random Fourier modes 1 <= |k| <= 4 scaled so the perturbation
  of B has RMS ``amp``; face B is the discrete curl of edge A, so its
  divergence (the stencil of constrans::maxdivB, transport.cpp:77-89) is
  zero to roundoff.  Fields are periodic on the global grid.
* ``con2prim_batch``: independent cells for the con2prim stress test --
  log-uniform rho, Lorentz factor, magnetisation sigma = b^2/rho, isotropic
  directions, Kerr-Schild positions.
"""
from __future__ import annotations

import numpy as np

from .mesh import BLOCK, CPN, GHOST, NC, NF, Quilt


def _global_index(n_cells: int, nqlt: int):
    """Global cell index of every local (patch, i, j, k) incl. ghosts, wrapped."""
    loc = np.arange(CPN) - GHOST
    base = np.arange(nqlt) * BLOCK
    g = (base[:, None] + loc[None, :]) % n_cells   # [nqlt][CPN]
    return g


def _vector_potential(n, L, amp, rng, kmax=4):
    """Edge-sampled periodic vector potential on an n^3 index grid; the
    curl is scaled afterwards to the requested RMS."""
    ks = []
    for kx in range(-kmax, kmax + 1):
        for ky in range(-kmax, kmax + 1):
            for kz in range(0, kmax + 1):
                k2 = kx * kx + ky * ky + kz * kz
                if k2 == 0 or k2 > kmax * kmax:
                    continue
                if kz == 0 and (ky < 0 or (ky == 0 and kx < 0)):
                    continue           # keep one of each +-k pair
                ks.append((kx, ky, kz))
    ks = np.array(ks, np.float64)
    nm = len(ks)
    amps = rng.normal(size=(nm, 3)) / np.maximum(1.0, np.sqrt((ks ** 2).sum(1)))[:, None]
    phase = rng.uniform(0, 2 * np.pi, size=(nm, 3))
    x = np.arange(n) / n   # fractional coordinate of the index grid
    A = np.zeros((3, n, n, n))
    for m in range(nm):
        kx, ky, kz = ks[m] * 2 * np.pi
        px = np.exp(1j * kx * x)[:, None, None]
        py = np.exp(1j * ky * x)[None, :, None]
        pz = np.exp(1j * kz * x)[None, None, :]
        e = px * py * pz
        for c in range(3):
            A[c] += amps[m, c] * np.imag(e * np.exp(1j * phase[m, c]))
    return A


def _curl_faces(A, dx):
    """Face fields from edge potential with the index structure of the CT
    update (transport.cpp:38-58), periodic, divergence-free by construction."""
    Ax, Ay, Az = A
    r = lambda a, ax: np.roll(a, 1, axis=ax)   # a[i-1] along ax
    Bx = (Az - r(Az, 1)) / dx[1] - (Ay - r(Ay, 2)) / dx[2]
    By = (Ax - r(Ax, 2)) / dx[2] - (Az - r(Az, 0)) / dx[0]
    Bz = (Ay - r(Ay, 0)) / dx[0] - (Ax - r(Ax, 1)) / dx[1]
    return Bx, By, Bz


def magnetised_box(quilt: Quilt, seed: int = 1, gamma: float = 4.0 / 3.0, rho0: float = 1.0,
                   p0: float = 0.1, dp: float = 0.01, B0=(0.5, 0.3, 0.0), amp: float = 1e-2):
    """Primitive cell state W [np][8][NC] and face field Bf [np][3][NF].

    Requires a single-level cubic quilt.  Ghost cells and ghost-region
    faces take the periodic image of the global field.
    """
    nq = quilt.nqlt
    assert len(quilt) == nq ** 3, "magnetised_box needs an unrefined quilt"
    n = nq * BLOCK
    rng = np.random.default_rng(seed)
    p = p0 * (1.0 + dp * rng.normal(size=(n, n, n)))
    L = [quilt.dom_h[d] - quilt.dom_l[d] for d in range(3)]
    dx = [L[d] / n for d in range(3)]
    A = _vector_potential(n, L, 1.0, rng)
    dB = _curl_faces(A, dx)
    rms = np.sqrt(np.mean(dB[0] ** 2 + dB[1] ** 2 + dB[2] ** 2) / 3.0)
    scale = amp / rms if rms > 0 else 0.0
    Bface = [B0[c] + scale * dB[c] for c in range(3)]
    # cell-centred B: mean of the two faces bounding the cell (face i is the
    # lower face of cell i, as patch::B_init builds it, grid.cpp:208-251)
    Bcell = [(Bface[c] + np.roll(Bface[c], -1, axis=c)) / 2 for c in range(3)]

    g = _global_index(n, nq)
    npch = len(quilt)
    W = np.zeros((npch, 8, NC))
    Bf = np.zeros((npch, 3, NF))
    eps = p / ((gamma - 1.0) * rho0)
    # faces: per-direction extents (21,20,20), (20,21,20), (20,20,21)
    gf = np.concatenate([g, ((g[:, -1:] + 1) % n)], axis=1)   # one more face index
    for pi_, P in enumerate(quilt.patches):
        i, j, k = P.ijk
        gi, gj, gk = g[i], g[j], g[k]
        sl = np.ix_(gi, gj, gk)
        W[pi_, 0] = rho0
        W[pi_, 1] = eps[sl].reshape(-1)
        for c in range(3):
            W[pi_, 5 + c] = Bcell[c][sl].reshape(-1)
        Bf[pi_, 0] = Bface[0][np.ix_(gf[i], gj, gk)].reshape(-1)
        Bf[pi_, 1] = Bface[1][np.ix_(gi, gf[j], gk)].reshape(-1)
        Bf[pi_, 2] = Bface[2][np.ix_(gi, gj, gf[k])].reshape(-1)
    return W, Bf


def con2prim_batch(n: int, seed: int = 4, gamma: float = 4.0 / 3.0, a: float = 0.9375,
                   rmin: float = 1.5, rmax: float = 50.0):
    """Primitive samples W [8][n] and positions r, theta for the con2prim
    stress batch.  The velocity is set from the Lorentz factor W in the
    Cartesian-component norm v_i v^i with the spatial metric of the
    solver, so the target is physical for that metric."""
    rng = np.random.default_rng(seed)
    rho = 10 ** rng.uniform(-8, 0, n)
    lor = rng.uniform(1.0, 20.0, n)
    sigma = 10 ** rng.uniform(-3, 2, n)
    r = rng.uniform(rmin, rmax, n)
    th = np.arccos(rng.uniform(-1, 1, n))
    # spatial metric of metric::comp (spacetime.cpp:20-34,103-109), M=1, Q=0
    c, s = np.cos(th), np.sin(th)
    Sig = r * r + a * a * c * c
    H = 2 * r / Sig
    g11 = 1 + H
    g13 = -H * a * s * s
    g22 = Sig
    g33 = (r * r + a * a + H * a * a * s * s) * s * s
    def unit():
        v = rng.normal(size=(3, n))
        return v / np.linalg.norm(v, axis=0)
    vh, bh = unit(), unit()
    def norm2(x):
        return g11 * x[0] ** 2 + 2 * g13 * x[0] * x[2] + g22 * x[1] ** 2 + g33 * x[2] ** 2
    v2 = 1.0 - 1.0 / lor ** 2
    v = vh * np.sqrt(v2 / np.maximum(norm2(vh), 1e-300))
    eps = 10 ** rng.uniform(-3, 0, n)
    # |B| such that b^2 ~ sigma rho (b^2 ~ B^2 / W^2 for B perpendicular to v)
    Bmag = np.sqrt(sigma * rho) * lor
    B = bh * (Bmag / np.sqrt(np.maximum(norm2(bh), 1e-300)))
    W = np.zeros((8, n))
    W[0], W[1], W[2:5], W[5:8] = rho, eps, v, B
    return W, r, th
