"""The step recorded into a CUDA graph and replayed equals the eagerly
launched step bit for bit; the FMA-contracted FP64 variant meets the same
first-step gate against the oracle as the reference-faithful one."""
import numpy as np
import pytest
import torch

from helpers import GAMMA, box_case, field_linf, gpu_tree, rel_linf, same_nan, ulp_sensitivity

pytestmark = pytest.mark.gpu


def test_graph_replay_equals_eager():
    import bhgpu
    q, orc, hp = box_case(2, seed=6, periodic=True, lim=0)
    eager = gpu_tree(q, hp, 0.0, 0.0, 0)
    graphed = gpu_tree(q, hp, 0.0, 0.0, 0)
    rk = bhgpu.RK2Integrator(0.4)
    U0 = graphed.U.clone(); W0 = graphed.W.clone(); B0 = graphed.Bf.clone()

    def reset():
        graphed.U.copy_(U0); graphed.W.copy_(W0); graphed.Bf.copy_(B0)

    g = bhgpu.StepGraph(graphed, rk, before=reset)
    for _ in range(2):                      # replaying restarts from the same state
        g.replay()
    torch.cuda.synchronize()
    rk.step(eager)
    for name in ("U", "W", "Bf", "dU"):
        assert torch.equal(getattr(eager, name).nan_to_num(7.0), getattr(graphed, name).nan_to_num(7.0)), name
    assert float(graphed.dt.item()) == float(eager.dt.item())
    # two steps through a graph without the reset
    g2 = bhgpu.StepGraph(graphed, rk, warmup=0)
    reset()
    e2 = gpu_tree(q, hp, 0.0, 0.0, 0)
    for _ in range(2):
        g2.replay()
        rk.step(e2, check_domain=False)
    torch.cuda.synchronize()
    assert torch.equal(e2.U.nan_to_num(7.0), graphed.U.nan_to_num(7.0))


@pytest.mark.parametrize("case", [dict(periodic=True, lim=0, M=0.0, a=0.0, lo=10.0, hi=12.0),
                                  dict(periodic=True, lim=2, M=1.0, a=0.9375, lo=-6.0, hi=6.0)])
def test_fma_variant_first_step(case):
    import bhgpu
    import oracle
    q, orc, hp = box_case(2, seed=4, **case)
    sens = ulp_sensitivity(orc, hp, steps=1)
    fma = oracle.Oracle(case["M"], case["a"], 0.0, GAMMA, limiter=case["lim"], fma=True)
    hf = hp.copy()
    fma.step(hf, 0.4)
    tree = bhgpu.AmrTree(q.dom_l, q.dom_h, q.nqlt, M=case["M"], a=case["a"], Q=0.0, gm=GAMMA,
                         periodic=q.periodic, limiter=case["lim"], quilt=q, init_floor=False, precision="fp64-fma")
    tree.load(U=hp.U, W=hp.W, Bf=hp.Bf, dU=hp.dU)
    dtg = bhgpu.RK2Integrator(0.4).step(tree)
    dtc = orc.step(hp, 0.4)
    assert abs(dtg - dtc) <= 1e-12 * dtc
    U = tree.U.cpu().numpy()
    assert same_nan(U, hp.U)
    assert max(field_linf(U, hp.U).values()) <= 1e-12
    for v in range(8):
        own = max(sens[v], rel_linf(hf.U[:, v], hp.U[:, v]))
        assert rel_linf(U[:, v], hp.U[:, v]) <= max(1e-12, 8 * own), v


def test_host_pipeline_equals_stepping_alone():
    """Three different host states through a two-tree pipeline (so a tree is
    reused while other copies are in flight) give the states one eager step
    gives each, bit for bit."""
    import bhgpu
    rk = bhgpu.RK2Integrator(0.4)
    states, want = [], []
    for seed in (6, 7, 8):
        q, orc, hp = box_case(2, seed=seed, periodic=True, lim=0)
        t = gpu_tree(q, hp, 0.0, 0.0, 0)
        states.append(tuple(x.cpu().pin_memory() for x in (t.U, t.W, t.Bf)))
        rk.step(t, check_domain=False)
        want.append((t.U.cpu(), t.W.cpu(), t.Bf.cpu()))
    trees = [gpu_tree(q, hp, 0.0, 0.0, 0) for _ in range(2)]
    pipe = bhgpu.HostPipeline(trees, rk)
    outs = [tuple(torch.empty_like(x).pin_memory() for x in s) for s in states]
    for s, o in zip(states, outs):
        pipe.submit(*s, *o)
    pipe.synchronize()
    for o, w in zip(outs, want):
        for a, b in zip(o, w):
            assert torch.equal(a.nan_to_num(7.0), b.nan_to_num(7.0))


def test_c_abi_step_graph_equals_direct_steps():
    """bh_step_graph_create / _replay / _destroy (the step as a CUDA graph for
    C callers): two replays on a non-default stream equal two direct bh_step
    calls bit for bit (faithful variant), and the legacy default stream is
    refused."""
    import ctypes as C
    import bhgpu
    from bhgpu._lib import BhParams, BhPool, lib
    from bhgpu.solver import _p
    vp = C.c_void_p
    lib.bh_step_graph_create.argtypes = [C.POINTER(BhParams), C.POINTER(BhPool), C.c_double, vp, vp, vp, C.c_int32,
                                         vp, C.POINTER(vp)]
    lib.bh_step_graph_replay.argtypes = [vp, vp]
    lib.bh_step_graph_destroy.argtypes = [vp]
    for f in ("bh_step_graph_create", "bh_step_graph_replay", "bh_step_graph_destroy"):
        getattr(lib, f).restype = C.c_int
    q, orc, hp = box_case(2, seed=9, periodic=True, lim=0)
    direct = gpu_tree(q, hp, 0.0, 0.0, 0)
    rk = bhgpu.RK2Integrator(0.4)
    rk.step(direct, check_domain=False)
    rk.step(direct, check_domain=False)
    torch.cuda.synchronize()
    g_tree = gpu_tree(q, hp, 0.0, 0.0, 0)
    P = g_tree.params()
    off = g_tree._wave_off
    s = torch.cuda.Stream()
    h = vp()
    args = (C.byref(P), C.byref(g_tree.pool), 0.4, _p(g_tree.dt), _p(g_tree.waves), off.ctypes.data_as(vp),
            g_tree.nwave)
    assert lib.bh_step_graph_create(*args, None, C.byref(h)) != 0      # legacy default stream refused
    assert lib.bh_step_graph_create(*args, vp(s.cuda_stream), C.byref(h)) == 0 and h.value
    try:
        for _ in range(2):
            assert lib.bh_step_graph_replay(h, vp(s.cuda_stream)) == 0
        s.synchronize()
    finally:
        assert lib.bh_step_graph_destroy(h) == 0
    for name in ("U", "W", "Bf"):
        a, b = getattr(direct, name), getattr(g_tree, name)
        assert torch.equal(a.contiguous().view(torch.int64), b.contiguous().view(torch.int64)), name
    assert torch.equal(direct.dt.view(torch.int64), g_tree.dt.view(torch.int64))
