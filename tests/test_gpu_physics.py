"""Physics known answers, derived from the equations rather than from
reference data (the reference ships no tests): TGV mass is conserved, its
early kinetic energy decays as exp(-2 nu k^2 t) with k^2 = 3 (2 pi / N)^2,
and the lid-driven cavity settles to a steady state."""
import math

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import api as a

    return a


@pytest.mark.parametrize("storage,arith,mass_tol", [("f64", "exact", 1e-13), ("f64", "fast", 1e-13),
                                                    ("f32", "fast", 1e-6)])
def test_tgv_mass_and_energy_decay(api, storage, arith, mass_tol):
    # Re 10: the viscous decay dominates the transfer to smaller scales
    N, U0, Re, steps = 64, 0.05, 10.0, 100
    nu = U0 * N / (2 * 3.1415926) / Re          # tgv/src/System.cpp:21 (tau = 3 nu)
    with api.LBM("tgv", N, N, N, 3 * nu, 1.0, U0, bc="reference", storage=storage, arith=arith) as lbm:
        m0, k0 = lbm.reduce("mass"), lbm.reduce("kinetic")
        lbm.step(steps)
        m1, k1 = lbm.reduce("mass"), lbm.reduce("kinetic")
    assert abs(m1 - m0) <= mass_tol * abs(m0)
    k2 = 3 * (2 * math.pi / N) ** 2
    want = -2 * nu * k2 * steps                   # log of the energy ratio
    got = math.log(k1 / k0)
    assert abs(got / want - 1) < 0.05, (got, want)


def test_cavity_reaches_steady_state(api):
    N, U, Re = 24, 0.05, 100.0
    with api.LBM("cavity", N, N, N, 3 * U * N / Re, 1.0, U, bc="standard", lid_u=U) as lbm:
        lbm.step(500)
        lbm.reduce("residual")
        res = []
        for _ in range(8):
            lbm.step(500)
            res.append(lbm.reduce("residual"))
    assert all(math.isfinite(r) for r in res)
    assert res[-1] < 0.1 * res[0], res
    assert res[-1] < 1e-3, res
