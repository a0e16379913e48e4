"""bh_ghosts_prims_static: the ghost fill and reconstruction for callers
that cannot allocate device memory (a host whose memory arena lends
libraries no device memory, for instance).  It keeps its per-cell
scratch in an array inside the library instead of the caller's
pool->status.

Checked through the C ABI against bh_ghosts_prims, the entry point that
takes the scratch from the caller, on two calls in a row with different
states (the second call sees the array the first one left behind).  The
tolerance is the one every GPU test uses for a single launch on identical
input -- here the two paths run the same kernels, so the results must
agree bit for bit.  Runs alone in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import GAMMA, box_case, gpu_tree

pytestmark = pytest.mark.gpu


def _run(tree, fn):
    import bhgpu
    from bhgpu.solver import _stream
    P = tree.params()
    rc = fn(C.byref(P), C.byref(tree.pool), _stream())
    torch.cuda.synchronize()
    assert rc == bhgpu._lib.BH_OK, rc
    return tree.U.cpu().numpy(), tree.W.cpu().numpy()


def test_static_scratch_matches_caller_scratch_two_calls():
    import bhgpu
    lib = bhgpu.lib
    for call, seed in enumerate((11, 12)):          # two calls in a row
        q, orc, hp = box_case(2, seed=seed, periodic=True, lim=0)
        ref_tree = gpu_tree(q, hp, 0.0, 0.0, 0)
        new_tree = gpu_tree(q, hp, 0.0, 0.0, 0)
        for t in (ref_tree, new_tree):               # the oracle's cell geometry
            t.rth.copy_(torch.as_tensor(hp.rth))
        new_tree.status.fill_(0xAB)                  # the caller's scratch must not be used
        U1, W1 = _run(ref_tree, lib.bh_ghosts_prims)
        U2, W2 = _run(new_tree, lib.bh_ghosts_prims_static)
        assert np.array_equal(U1, U2, equal_nan=True), call
        assert np.array_equal(W1, W2, equal_nan=True), call
        assert bool((new_tree.status == 0xAB).all()), "pool->status was written"
        # and it is the reconstruction the oracle computes (1e-12 per variable)
        orc.ghosts(hp); orc.prims(hp)
        for v in range(8):
            a, b = W2[:, v], hp.W[:, v]
            m = np.isfinite(a) & np.isfinite(b)
            assert np.abs(a[m] - b[m]).max() <= 1e-12 * np.abs(b[m]).max(), v


def test_static_scratch_rejects_oversized_pool():
    import bhgpu
    q, orc, hp = box_case(2, seed=11, periodic=True, lim=0)
    tree = gpu_tree(q, hp, 0.0, 0.0, 0)
    pool = bhgpu._lib.BhPool.from_buffer_copy(tree.pool)
    pool.npatch = 1025                               # above BH_STATIC_MAX_PATCHES = 1024
    P = tree.params()
    from bhgpu.solver import _stream
    assert bhgpu.lib.bh_ghosts_prims_static(C.byref(P), C.byref(pool), _stream()) == bhgpu._lib.BH_ERANGE
