"""The Fishbone-Moncrief torus initial data (init::fm_init, init::B_pot_init
and the sequence of main(), initconds.cpp / main.cpp:89-160): the kernels'
items built for the host equal the reference's own initialisation bit for
bit on the torus of the Kerr box (a = 0.9375), including the face field from
the curl of A_phi and its ghost-cell densities.  Skipped where the
reference harness is not built."""
import ctypes as C

import numpy as np
import pytest

import oracle
from bhgpu.mesh import Quilt
from hostcheck import HostKernels, _d

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built")

GAMMA = 4.0 / 3.0


def eq(a, b):
    return np.array_equal(a, b, equal_nan=True)


def torus_case(nq=2, a=0.9375):
    q = Quilt([-40.0] * 3, [40.0] * 3, nq)
    ref = oracle.RefSolver(q.dom_l, q.dom_h, nq, 1.0, a, 0.0, GAMMA)
    rc, rho_max = ref.torus_init()
    assert rc == 0
    R = oracle.HostPool(q.tables())
    ref.get(R)
    return q, R, rho_max


@pytest.mark.parametrize("a", [0.9375, 0.0])
def test_torus_initial_data_bitwise(a):
    q, R, rho_max = torus_case(2, a)
    hk = HostKernels(1.0, a, 0.0, GAMMA, 1)
    hp = oracle.HostPool(q.tables())
    pool = hk.pool(hp)
    hk.L.hc_geometry(C.byref(pool))
    out = np.zeros(5)
    hk.L.hc_torus_init.restype = C.c_int
    assert hk.call("hc_torus_init", C.byref(pool), C.c_double(12.0), C.c_double(4.5), _d(out)) == 0
    assert out[4] == rho_max
    if a:
        assert out[0] > 0 and out[2] > 0 and out[3] > 0 and rho_max == 1.0, "the torus exists"
        assert (hp.W[:, 0] > 0.1).sum() > 100
    else:
        # Schwarzschild: ln h < 0 at r_max, so fm_init gives up and keeps the
        # floor state (initconds.cpp:425-429); main() goes on with the field
        assert out[2] <= 0 and out[3] == 0.0 and rho_max < 1e-5
    assert eq(hp.W, R.W) and eq(hp.U, R.U) and eq(hp.Bf, R.Bf)
    assert np.abs(hp.Bf).max() > 0
