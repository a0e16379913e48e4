"""Shared set-up for the parity tests: one seeded state loaded identically
into the GPU tree and into the CPU checkers."""
from __future__ import annotations

import numpy as np

import oracle
from bhgpu import configs
from bhgpu.mesh import Quilt

GAMMA = 4.0 / 3.0


def rel_linf(a, b):
    """Per-variable relative L-infinity error over the entries finite in
    both, normalised by the largest reference magnitude of that variable."""
    a = np.asarray(a); b = np.asarray(b)
    m = np.isfinite(a) & np.isfinite(b)
    if not m.any():
        return 0.0
    scale = np.abs(b[m]).max()
    return float(np.abs(a[m] - b[m]).max() / scale) if scale > 0 else float(np.abs(a[m] - b[m]).max())


FIELDS = {"D": [0], "S": [1, 2, 3], "tau": [4], "B": [5, 6, 7]}
PRIM_FIELDS = {"rho": [0], "eps": [1], "v": [2, 3, 4], "B": [5, 6, 7]}


def field_linf(a, b, fields=FIELDS):
    """Relative L-infinity error per conserved field of a [np][8][n] state:
    the vector fields S and B are normalised by their largest component
    magnitude, the scalars by their own.  Entries finite in both only."""
    out = {}
    for name, comps in fields.items():
        x = np.asarray(a)[:, comps]; y = np.asarray(b)[:, comps]
        m = np.isfinite(x) & np.isfinite(y)
        scale = np.abs(y[m]).max() if m.any() else 0.0
        err = np.abs(x[m] - y[m]).max() if m.any() else 0.0
        out[name] = float(err / scale) if scale > 0 else float(err)
    return out


def ulp_sensitivity(orc, hp, steps=1, seed=0):
    """Per-component relative change of the oracle's own result when its
    input state U moves by one ulp (random direction per entry): the
    conditioning floor of the reference for this case."""
    rng = np.random.default_rng(seed)
    base = hp.copy()
    pert = hp.copy()
    pert.U[:] = np.where(rng.random(pert.U.shape) < 0.5, np.nextafter(pert.U, np.inf), np.nextafter(pert.U, -np.inf))
    for _ in range(steps):
        orc.step(base, 0.4)
        orc.step(pert, 0.4)
    return [rel_linf(pert.U[:, v], base.U[:, v]) for v in range(8)]


def perturbed_response(orc, hp, steps, rel=1e-7, seed=0):
    """The reference's own response to a relative input perturbation: the
    oracle run from U and from U (1 + rel N(0,1)) for ``steps`` steps;
    returns (per-variable relative L1 difference, NaN-mask disagreement)."""
    rng = np.random.default_rng(seed)
    base = hp.copy()
    pert = hp.copy()
    pert.U[:] = pert.U * (1.0 + rel * rng.standard_normal(pert.U.shape))
    for _ in range(steps):
        orc.step(base, 0.4)
        orc.step(pert, 0.4)
    return rel_l1(pert.U, base.U), mask_disagreement(pert.U, base.U), base


def rel_l1(a, b):
    """Per-variable relative L1 error over the entries finite in both."""
    out = []
    for v in range(a.shape[1]):
        x = np.asarray(a)[:, v]; y = np.asarray(b)[:, v]
        m = np.isfinite(x) & np.isfinite(y)
        den = np.abs(y[m]).mean() if m.any() else 0.0
        num = np.abs(x[m] - y[m]).mean() if m.any() else 0.0
        out.append(float(num / den) if den > 0 else float(num))
    return out


def mask_disagreement(a, b):
    return float(np.mean(np.isfinite(a) != np.isfinite(b)))


def same_nan(a, b):
    return np.array_equal(np.isfinite(a), np.isfinite(b))


def box_case(nq=2, seed=3, periodic=True, lim=0, M=0.0, a=0.0, lo=10.0, hi=12.0, **box):
    """Magnetised-box state on an nq^3 quilt: (quilt, oracle, host pool);
    ``box`` goes to configs.magnetised_box (B0=(0, 0, 0), amp=0 gives the
    unmagnetised box)."""
    q = Quilt([lo] * 3, [hi] * 3, nq, periodic=periodic)
    orc = oracle.Oracle(M, a, 0.0, GAMMA, limiter=lim)
    hp = oracle.HostPool(q.tables())
    orc.geometry(hp)
    W, Bf = configs.magnetised_box(q, seed=seed, gamma=GAMMA, **box)
    hp.W[:] = W
    hp.Bf[:] = Bf
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    return q, orc, hp


def oracle_regrid(orc, hp, quilt):
    """One amrtree::regrid on the oracle: flags, the quilt's plan, the data
    operations on the extended pool, then the kept patches.  Returns the
    new HostPool (quilt is updated in place) and the plan."""
    flags = orc.regrid_flags(hp)
    plan = quilt.regrid(flags)
    T = quilt.tables()
    ext = oracle.HostPool({"pgeo": plan.ext_pgeo, "lvl": np.zeros(plan.n_ext, np.int32),
                           "ijk": np.zeros((plan.n_ext, 3), np.int32), "leaf": np.zeros(plan.n_ext, np.uint8),
                           "nbr": np.zeros((plan.n_ext, 6, 2), np.int32)})
    for name in ("U", "W", "dU", "F", "Bf", "EMF"):
        getattr(ext, name)[:plan.n_old] = getattr(hp, name)
    orc.geometry(ext)
    for p, kids in plan.refined:
        orc.refine_data(ext, p, kids)
    for p, kids in plan.flattened:
        orc.ccrstr(ext, p, kids)
    new = oracle.HostPool(T)
    for name in ("U", "W", "dU", "F", "Bf", "EMF", "rth"):
        getattr(new, name)[:] = getattr(ext, name)[plan.keep]
    return new, plan


def gpu_tree(q, hp, M=0.0, a=0.0, lim=0, precision="fp64"):
    import bhgpu
    tree = bhgpu.AmrTree(q.dom_l, q.dom_h, q.nqlt, M=M, a=a, Q=0.0, gm=GAMMA, periodic=q.periodic,
                         limiter=lim, quilt=q, init_floor=False, precision=precision)
    tree.load(U=hp.U, W=hp.W, Bf=hp.Bf, dU=hp.dU)
    return tree


def random_prims(n, rng, a=0.0):
    r = rng.uniform(2.0, 40.0, n)
    th = np.arccos(rng.uniform(-0.98, 0.98, n))
    W = np.zeros((8, n))
    W[0] = 10 ** rng.uniform(-3, 0, n)
    W[1] = 10 ** rng.uniform(-2, 0, n)
    W[2:5] = rng.normal(size=(3, n)) * 0.02
    W[5:8] = rng.normal(size=(3, n)) * 0.1
    return W, r, th
