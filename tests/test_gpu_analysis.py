"""The analyser on the device (bh_analysis through bhgpu.Analyser) against
the oracle.  The integrands are the reference's (bit for bit in the host
build, tests/test_hostcheck.py); the device adds them in another order, so
each raw integral must lie within the error bound of serial summation,
2 n u sum|f_i|, of the oracle's.  After a device step, the derived fields
floors records meet the first-step gate and the integrals agree to 1e-10 of
sum|f_i|."""
import numpy as np
import pytest

from bhgpu.mesh import interior_mask
from helpers import box_case, field_linf, gpu_tree, same_nan

pytestmark = pytest.mark.gpu

HRZ, RS = 2.0, 10.0


def case():
    q, orc, hp = box_case(2, seed=4, periodic=False, lim=1, M=1.0, a=0.0, lo=-6.0, hi=6.0)
    return q, orc, hp


def test_integrals_within_the_serial_summation_bound():
    import bhgpu
    q, orc, hp = case()
    orc.step(hp, 0.4)
    tree = gpu_tree(q, hp, M=1.0, a=0.0, lim=1)
    tree.load(Wd=hp.Wd)
    g = bhgpu.Analyser().integrals(tree, HRZ, RS)
    raw, absr = orc.analysis(hp, HRZ, RS)
    n = hp.npatch * 4096
    assert np.all(np.abs(g - raw) <= 2 * n * 2.0 ** -53 * absr), np.abs(g - raw) / np.maximum(absr, 1e-300)
    b = bhgpu.Analyser().batch_(tree, 0.5)
    assert b["Mdot"] != 0.0 and np.isfinite(b["L_BZ"])


def test_derived_fields_and_integrals_after_a_device_step():
    import bhgpu
    q, orc, hp = case()
    tree = gpu_tree(q, hp, M=1.0, a=0.0, lim=1)
    bhgpu.RK2Integrator(0.4).step(tree)
    orc.step(hp, 0.4)
    m = interior_mask()
    Wd = tree.Wd.cpu().numpy()
    assert same_nan(Wd[:, :, m], hp.Wd[:, :, m])
    assert max(field_linf(Wd[:, :, m], hp.Wd[:, :, m], {"lor": [0], "p": [1], "h": [2], "b2": [3]}).values()) <= 1e-12
    g = bhgpu.Analyser().integrals(tree, HRZ, RS)
    raw, absr = orc.analysis(hp, HRZ, RS)
    assert np.all(np.abs(g - raw) <= 1e-10 * absr)
