"""Asynchronous field reads (imexlb_get_fields_async): the host buffers get
the fields of the moment of the call, even while later steps run and
rewrite the views, and a restored or re-initialised lattice is not raced by
a pending copy."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import api as a

    return a


def pinned(shape):
    import torch

    return {k: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for k in "uvwp"}


@pytest.mark.parametrize("case,bc,storage,arith,kw", [
    ("cavity", "standard", "f64", "fast", dict(lid_u=0.1)),
    ("cavity", "standard", "f16", "fast", dict(lid_u=0.1)),
    ("tgv", "reference", "f64", "exact", {}),
])
def test_async_read_holds_the_fields_of_its_call(api, case, bc, storage, arith, kw):
    n = (32, 24, 20)
    args = (case, *n, 0.03, 1.0, 0.05)
    with api.LBM(*args, bc=bc, storage=storage, arith=arith, **kw) as ref:
        ref.step(6)
        want6 = ref.fields()
        ref.step(40)
        want46 = ref.fields()
    shape = (n[2], n[1], n[0])
    bufs = [pinned(shape), pinned(shape)]
    with api.LBM(*args, bc=bc, storage=storage, arith=arith, **kw) as lat:
        lat.step(6)
        lat.fields(out=bufs[0], wait=False)
        lat.step(40)  # runs while the copy may still be in flight
        lat.fields(out=bufs[1], wait=False)
        lat.synchronize()
        for k in "uvwp":
            assert np.array_equal(bufs[0][k], want6[k]), f"{k} after 6 steps"
            assert np.array_equal(bufs[1][k], want46[k]), f"{k} after 46 steps"
        # a synchronous read after more steps agrees with the asynchronous one
        lat.step(3)
        a = lat.fields(out=pinned(shape), wait=False)
        lat.synchronize()
        b = lat.fields()
        for k in "uvwp":
            assert np.array_equal(a[k], b[k])
        # re-initialising waits for a pending copy
        lat.fields(out=bufs[0], wait=False)
        lat.Initialize()
        lat.step(6)
        again = lat.fields()
        for k in "uvwp":
            assert np.array_equal(again[k], want6[k])
