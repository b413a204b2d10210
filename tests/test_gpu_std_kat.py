"""Known answers of the standard boundaries on the device (the properties
tests/test_std_spec_cpu.py checks on the specification), in FP64 EXACT and
FAST and in the reduced storage formats, plus the lid-driven slab against
its specification bit for bit in EXACT arithmetic."""
import numpy as np
import pytest

from oracle.bindings import OracleStd

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import api as a

    return a


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_moving_lid_cavity_conserves_mass(api, arith):
    with api.LBM("cavity", 24, 22, 26, 0.06, 1.0, 0.1, bc="standard", lid_u=0.1, arith=arith) as lbm:
        for _ in range(3):
            lbm.step(150)
            f = lbm.fields()
            assert abs((3 * f["p"]).sum()) <= 1e-13 * np.abs(3 * f["p"]).sum()


@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f64", "fast"), ("f32", "fast"), ("f16", "fast"),
                                           ("bf16", "fast")])
def test_cavity_at_rest_stays_at_rest(api, storage, arith):
    with api.LBM("cavity", 32, 30, 34, 0.06, 1.0, 0.0, bc="standard", storage=storage, arith=arith) as lbm:
        lbm.step(200)
        f = lbm.fields()
    for k in "uvwp":
        assert np.all(f[k] == 0.0), (storage, k)


@pytest.mark.parametrize("storage,tol", [("f64", 1e-14), ("f32", 1e-7), ("f16", 2e-6), ("bf16", 2e-6)])
def test_channel_without_solid_stays_uniform(api, storage, tol):
    with api.LBM("sphere", 64, 16, 18, 0.05, 1.0, 0.05, bc="standard", storage=storage, arith="fast",
                 inlet_u=0.05, sphere_d=1e-3, sphere_c=(10.5, 6.5, 7.5)) as lbm:
        lbm.step(300)
        f = lbm.fields()
        assert np.all(lbm.mask() == 1)
    assert np.abs(f["u"] - 0.05).max() <= tol, storage
    assert max(np.abs(f["v"]).max(), np.abs(f["w"]).max(), np.abs(f["p"]).max()) <= tol, storage


@pytest.mark.parametrize("storage,arith,tol", [("f64", "exact", 1e-14), ("f64", "fast", 1e-14),
                                               ("f32", "fast", 2e-7)])
def test_slab_reaches_plane_couette_flow(api, storage, arith, tol):
    nz, lid = 8, 0.04
    with api.LBM("cavity", 8, 6, nz, 0.5, 1.0, lid, bc="slab", storage=storage, arith=arith, lid_u=lid) as lbm:
        lbm.step(6000)
        f = lbm.fields()
    want = lid * (np.arange(nz) + 0.5) / nz
    assert np.abs(f["u"] - want[:, None, None]).max() <= tol
    assert max(np.abs(f["v"]).max(), np.abs(f["w"]).max()) <= tol


def test_slab_exact_matches_specification(api):
    nx, ny, nz, tau0, lid = 8, 6, 10, 0.08, 0.05
    o = OracleStd("slab", nx, ny, nz, tau0, 1.0, lid, lid_u=lid)
    o.step(120)
    want = dict(zip("uvwp", o.moments()))
    with api.LBM("cavity", nx, ny, nz, tau0, 1.0, lid, bc="slab", arith="exact", lid_u=lid) as lbm:
        lbm.step(120)
        got = lbm.fields()
    for k in "uvwp":
        assert np.array_equal(got[k], want[k]), (k, np.abs(got[k] - want[k]).max())
