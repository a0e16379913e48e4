"""The launch-bound autotuner (bhgpu.tune) on the device.  The candidates
change only the registers per thread the compiler may use.  In the
reference-faithful variant (no contraction) every choice steps the state to
the same bits.  In the contracted variants ptxas may fuse a different set of
multiply-add pairs under another register budget, which moves results by
ulps: there every choice must agree with the default to the variant's own
rounding level.  autotune picks a candidate, restores the tree's state and
can cache and re-apply its choice."""
import json

import pytest
import torch

pytestmark = pytest.mark.gpu


def box(nq, precision, **kw):
    import bhgpu
    from bhgpu import configs
    from bhgpu.mesh import Quilt
    q = Quilt([10.0] * 3, [12.0] * 3, nq, periodic=True)
    tree = bhgpu.AmrTree(q.dom_l, q.dom_h, nq, M=0.0, a=0.0, Q=0.0, gm=4.0 / 3.0, periodic=True,
                         limiter="minmod", quilt=q, init_floor=False, precision=precision)
    W, Bf = configs.magnetised_box(q, seed=3, **kw)
    tree.load(W=W, Bf=Bf)
    tree.prim_to_cons()
    return tree


def bits(t):
    return t.contiguous().view(torch.int64)


def settings(i):
    from bhgpu import tune
    return {k: tune.candidates(k)[i % len(tune.candidates(k))] for k in tune.KERNELS}


def run_with(tree, precision, choice, U0, W0, B0, steps):
    import bhgpu
    from bhgpu import tune
    for k, c in choice.items():
        tune.set(precision, k, c)
    integ = bhgpu.RK2Integrator(0.4)
    tree.U.copy_(U0); tree.W.copy_(W0); tree.Bf.copy_(B0)
    for _ in range(steps):
        integ.step(tree, check_domain=False)
    torch.cuda.synchronize()
    return tree.U.clone(), tree.W.clone(), tree.Bf.clone()


def test_every_launch_bound_gives_the_same_bits_faithful():
    from bhgpu import tune
    tree = box(2, "fp64")
    U0, W0, B0 = tree.U.clone(), tree.W.clone(), tree.Bf.clone()
    default = tune.current("fp64")
    try:
        ref = run_with(tree, "fp64", default, U0, W0, B0, 2)
        for i in range(4):
            out = run_with(tree, "fp64", settings(i), U0, W0, B0, 2)
            for a, b in zip(ref, out):
                assert torch.equal(bits(a), bits(b)), settings(i)
    finally:
        for k, c in default.items():
            tune.set("fp64", k, c)


@pytest.mark.parametrize("precision,tol", [("fp64-fma", 1e-12), ("mixed", 1e-5)])
def test_every_launch_bound_agrees_to_rounding_contracted(precision, tol):
    """Unmagnetised box (con2prim well conditioned there), two steps: every
    choice within `tol` relative L-infinity of the default's result per
    conserved field, the same NaN mask."""
    from bhgpu import tune
    tree = box(2, precision, B0=(0.0, 0.0, 0.0), amp=0.0)
    U0, W0, B0 = tree.U.clone(), tree.W.clone(), tree.Bf.clone()
    default = tune.current(precision)
    try:
        ref = run_with(tree, precision, default, U0, W0, B0, 2)[0]
        for i in range(4):
            U = run_with(tree, precision, settings(i), U0, W0, B0, 2)[0]
            assert torch.equal(torch.isfinite(U), torch.isfinite(ref))
            for comps in ([0], [1, 2, 3], [4], [5, 6, 7]):
                a, b = U[:, comps], ref[:, comps]
                m = torch.isfinite(b)
                den = b[m].abs().max().item()
                err = (a[m] - b[m]).abs().max().item() / (den if den > 0 else 1.0)
                assert err <= tol, (settings(i), comps, err)
    finally:
        for k, c in default.items():
            tune.set(precision, k, c)


def test_autotune_keeps_the_state_and_caches_its_choice(tmp_path):
    import bhgpu
    from bhgpu import tune
    tree = box(4, "fp64-fma")
    integ = bhgpu.RK2Integrator(0.4)
    before = {n: getattr(tree, n).clone() for n in ("U", "W", "Bf")}
    default = tune.current("fp64-fma")
    path = str(tmp_path / "tune.json")
    try:
        res = tune.autotune(tree, integ, reps=1, cache=path, save=True)
        for n, t in before.items():
            assert torch.equal(bits(getattr(tree, n)), bits(t)), n
        for k, c in res["choice"].items():
            assert c in tune.candidates(k)
            assert set(res["ms"][k]) == set(tune.candidates(k))
            assert res["ms"][k][c] == min(res["ms"][k].values())
        print(res)
        with open(path) as f:
            data = json.load(f)
        assert list(data.values()) == [res["choice"]]
        for k, c in default.items():
            tune.set("fp64-fma", k, c)
        assert tune.load_tuning("fp64-fma", cache=path) == res["choice"]
        assert tune.current("fp64-fma") == res["choice"]
    finally:
        for k, c in default.items():
            tune.set("fp64-fma", k, c)
