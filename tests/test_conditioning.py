"""Documents how far the reference's own result is defined on the
magnetised box, with the C restatement pinned to it: built with one-ulp
noise on its libm results, or with fused multiply-add, the same algorithm
agrees with itself after one step but not after two (its Brent fallback,
conserved.cpp:232-285, and the blow-up of the box amplify last-bit changes
to O(1)).  This is why the GPU parity gate is strict at step 1 and an
envelope afterwards."""
import numpy as np

import oracle
from helpers import box_case, field_linf, mask_disagreement, rel_l1


def test_reference_self_divergence():
    q, orc, hp = box_case(2, seed=4, periodic=True, lim=0)
    noisy = oracle.Oracle(0.0, 0.0, 0.0, 4.0 / 3.0, limiter=0, noise=True, seed=0)
    fma = oracle.Oracle(0.0, 0.0, 0.0, 4.0 / 3.0, limiter=0, fma=True)
    a, b, c = hp.copy(), hp.copy(), hp.copy()
    noisy.geometry(b)
    for s in range(2):
        orc.step(a, 0.4); noisy.step(b, 0.4); fma.step(c, 0.4)
        for other in (b, c):
            if s == 0:
                assert mask_disagreement(other.U, a.U) == 0.0
                assert max(field_linf(other.U, a.U).values()) < 1e-12
            else:
                assert mask_disagreement(other.U, a.U) > 1e-3
                assert max(rel_l1(other.U, a.U)) > 1e-3
