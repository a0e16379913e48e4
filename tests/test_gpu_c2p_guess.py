"""The learned con2prim guess on the device: the network's gradient
(bh_mlp_train_step) against the CPU restatement (oracle/mlp.py), training on
solver-generated pairs, and what the trained guess does to the reference's
con2prim on held-out cells of the stress batch (Kerr a = 0.9375): fewer
Newton iterations, no more failures, the same primitives where both
succeed (both stop at |f(xi)| < 1e-10 -- a wide band in xi for dilute
cells, so the comparison takes D > 1e-4), except the few cells where the
reference's non-monotonic residual has another root inside the bracket
(measured: 8.59 -> 7.44 iterations, failures 55.84 % -> 55.82 %, 0.12 % of
the dense cells on another root)."""
import numpy as np
import pytest
import torch

from oracle import mlp

pytestmark = pytest.mark.gpu


def batch(n, seed):
    import bhgpu
    from bhgpu import configs
    W, r, th = configs.con2prim_batch(n, seed=seed)
    cn = bhgpu.Conserved(bhgpu.Metric(1.0, 0.9375, 0.0), bhgpu.State(4.0 / 3.0))
    U, _ = cn.ptoc(W, r, th, check_domain=False)
    return cn, U, torch.as_tensor(r, device="cuda"), torch.as_tensor(th, device="cuda")


def test_gradient_matches_the_cpu_restatement():
    import bhgpu
    cn, U, r, th = batch(2048, 11)
    g = bhgpu.C2PGuess(cn, seed=3)
    pre = g.preamble(U, r, th)
    x = g.features(pre, r)
    ok = torch.isfinite(x).all(0) & torch.isfinite(pre).all(0)
    idx = torch.nonzero(ok).flatten()
    pre, rr, x = pre[:, idx].contiguous(), r[idx].contiguous(), x[:, idx]
    g.w[mlp.NPARAM:mlp.NPARAM + 6] = x.mean(1)
    g.w[mlp.NPARAM + 6:] = 1.0 / x.std(1)
    import ctypes as C
    from bhgpu.c2p_guess import lib
    lib.bh_mlp_sync_bf16(C.byref(g.s), None)
    rng = np.random.default_rng(0)
    tgt = torch.as_tensor(rng.normal(size=(2, idx.numel())), dtype=torch.float32, device="cuda")
    L, grad = g.gradient(pre, rr, tgt)
    Lc, gc = mlp.loss_and_grad(g.w.double().cpu().numpy(), mlp.features(pre.cpu().numpy(), rr.cpu().numpy()),
                               tgt.double().cpu().numpy().T)
    assert abs(L - Lc) <= 1e-4 * abs(Lc)
    assert np.abs(grad - gc).max() <= 1e-3 * np.abs(gc).max()


def test_trained_guess_saves_newton_iterations():
    import bhgpu
    cn, U, r, th = batch(1 << 16, 5)
    g = bhgpu.C2PGuess(cn, seed=0)
    hist = g.train(U, r, th, steps=1500, batch=8192)
    assert hist[-1] < 0.05 * hist[0]
    cn2, U2, r2, th2 = batch(1 << 16, 6)             # held out
    W0, Wd0, st0, it0, pa0 = cn.ctop(U2, r2, th2, check_domain=False)
    W1, Wd1, st1, it1, pa1 = g.ctop(U2, r2, th2)
    ok0, ok1 = st0 == 1, st1 == 1
    both = ok0 & ok1
    it_plain = it0[both].double().mean().item()
    it_guess = it1[both].double().mean().item()
    fail0, fail1 = 1 - ok0.double().mean().item(), 1 - ok1.double().mean().item()
    # the reference accepts NaN primitives (its positivity tests are false
    # for NaN); those must agree, the finite ones match to Newton's tolerance
    assert torch.equal(torch.isnan(W1[0][both]), torch.isnan(W0[0][both]))
    fin = both & torch.isfinite(W0[0])
    # Newton stops at |f(xi)| < 1e-10 absolute (A6) and xi scales with the
    # density (1e-8 .. 1 here): for dilute cells that band is wide, and two
    # starting points may stop anywhere inside it.  Where D > 1e-4 the band is
    # narrow, and there only a second root of the residual can separate them.
    dense = g.preamble(U2, r2, th2)[0] > 1e-4
    rel_all = ((W1[0] - W0[0]).abs() / W0[0].abs())
    rel = rel_all[fin & dense]
    other_root = (rel > 1e-6).double().mean().item()
    print(f"dilute cells outside 1e-6: {(rel_all[fin & ~dense] > 1e-6).double().mean().item():.3f}")
    print(f"loss {hist[0]:.3g} -> {hist[-1]:.3g}; Newton iterations {it_plain:.2f} -> {it_guess:.2f}; "
          f"failed {fail0:.4f} -> {fail1:.4f}; rho rel diff median {rel.median().item():.2e}, "
          f"other root {other_root:.2e}")
    assert it_guess < 0.95 * it_plain
    assert fail1 <= fail0 + 2e-3
    # the reference's residual is not monotonic (A3, A4): a few cells have more
    # than one root in the bracket, and another start may settle on another
    assert other_root <= 5e-3                      # measured 1.2e-3
    assert rel.median().item() <= 1e-9


@pytest.mark.parametrize("n", [(1 << 16) + 77, 100])
def test_tensor_core_network_is_the_trained_network(n):
    """bh_ctop_learned evaluates the network on the tensor cores (BF16
    weights, activations as BF16 hi + lo halves, FP32 accumulation in
    tensor memory) in the kernel that also forms con2prim's preamble.  Its
    starting points equal the CUDA-core network's (bh_mlp_guess) up to FP32
    summation order, with the same NaN pattern, on a ragged last tile too;
    the con2prim outcomes then agree with the three-kernel sequence
    bh_ctop_pre, bh_mlp_guess, bh_ctop_guess."""
    import bhgpu
    cn, U, r, th = batch(1 << 16, 5)
    g = bhgpu.C2PGuess(cn, seed=0)
    g.train(U, r, th, steps=500, batch=8192)
    cn2, U2, r2, th2 = batch(n, 6)
    xi_cc = g.guess(g.preamble(U2, r2, th2), r2)
    W1, Wd1, st1, it1, pa1 = g.ctop(U2, r2, th2)
    W2, Wd2, st2, it2, pa2, xi_tc = g.ctop_learned(U2, r2, th2, want_xi0=True)
    torch.cuda.synchronize()
    assert torch.equal(torch.isnan(xi_cc), torch.isnan(xi_tc))
    fin = torch.isfinite(xi_cc)
    assert fin.double().mean().item() > 0.9
    rel = ((xi_tc - xi_cc).abs() / xi_cc.abs())[fin]
    print(f"n={n}: start points, max relative difference {rel.max().item():.2e}, "
          f"median {rel.median().item():.2e}")
    assert rel.max().item() <= 1e-3
    same = (st1 == st2).double().mean().item()
    assert same >= 0.999, same
    ok = (st1 == 1) & (st2 == 1)
    if ok.any():
        d = abs(it1[ok].double().mean().item() - it2[ok].double().mean().item())
        assert d <= 0.01 * it1[ok].double().mean().item() + 0.05


def test_bounded_wait_reports_a_timeout():
    """The tensor-core kernel's bounded mbarrier wait, run on a barrier
    nothing arrives on: it gives up after its limit (about a second) and
    sets BH_ERR_TIMEOUT in the error word; the context stays usable."""
    import bhgpu
    err = bhgpu.wait_selftest()
    assert err == 2
    x = torch.ones(4, device="cuda")
    assert float(x.sum().item()) == 4.0
