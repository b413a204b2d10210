"""Checkpoint / restore: a lattice or engine instance restored from a
checkpoint continues bit for bit, and a checkpoint of other parameters is
refused."""
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


@pytest.mark.parametrize("case,bc,storage,arith,kw", [
    ("cavity", "reference", "f64", "exact", {}),
    ("cavity", "standard", "f16", "fast", dict(lid_u=0.1)),
    ("sphere", "standard", "bf16", "fast", dict(inlet_u=0.05, sphere_d=6.0, sphere_c=(12.0, 8.0, 8.0))),
    ("tgv", "reference", "f32", "fast", {}),
])
def test_lattice_resumes_bit_for_bit(api, case, bc, storage, arith, kw):
    n = (48, 16, 16) if case == "sphere" else (24, 20, 16)
    args = (case, *n, 0.03, 1.0, 0.05)
    with api.LBM(*args, bc=bc, storage=storage, arith=arith, **kw) as a:
        a.step(17)
        ck = a.checkpoint()
        a.step(12)
        want = a.fields()
    with api.LBM(*args, bc=bc, storage=storage, arith=arith, **kw) as b:
        b.restore(ck)
        assert b.steps_taken() == 17
        b.step(12)
        got = b.fields()
    for k in "uvwp":
        assert np.array_equal(got[k], want[k]), k
    with api.LBM(case, *n, 0.04, 1.0, 0.05, bc=bc, storage=storage, arith=arith, **kw) as c:
        with pytest.raises(api.ImexlbError):
            c.restore(ck)  # another tau


def test_engine_instance_preempted_and_resumed(api):
    d = api.instance_desc("cavity", 40, 24, 20, 0.03, 1.0, 0.1, lid_u=0.1)
    other = api.instance_desc("tgv", 32, 32, 32, 0.02, 1.0, 0.05)
    with api.Engine(storage="f16", budget_bytes=1 << 28, max_instances=4) as eng:
        s = eng.add(d)
        eng.add(other)
        eng.step(21)
        ck = eng.checkpoint(s)
        eng.step(13)
        want = eng.fields(s)
        eng.remove(s)
        eng.step(1)  # the engine's step parity differs from the checkpoint's
        r = eng.restore(d, ck)
        eng.step(13)
        got = eng.fields(r)
    for k in "uvwp":
        assert np.array_equal(got[k], want[k]), k
