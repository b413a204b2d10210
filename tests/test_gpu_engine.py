"""GPU checks of the engine (many lattices advanced by one persistent launch).

Each instance's result must be identical to the same lattice run alone
through the single-lattice API: same per-cell code, same arithmetic, so the
fields are compared bit for bit.  That holds while other instances share
the launches, join part-way (at either step parity) and leave; this is the
"same result alone and in the mix" property the serving loop relies on.
"""
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


MIX = [
    ("tgv", (24, 24, 24), 0.02, 0.05, {}),
    ("cavity", (32, 20, 28), 0.03, 0.1, dict(lid_u=0.1)),
    ("sphere", (48, 16, 16), 0.015, 0.05, dict(inlet_u=0.05, sphere_d=6.0, sphere_c=(12.0, 8.0, 8.0))),
    ("cavity", (17, 9, 11), 0.05, 0.1, dict(lid_u=0.08)),
    ("tgv", (40, 16, 20), 0.01, 0.05, {}),
]


def alone(api, case, n, tau, u0, kw, steps, storage, arith):
    bc = "reference" if case == "tgv" else "standard"
    with api.LBM(case, *n, tau, 1.0, u0, bc=bc, storage=storage, arith=arith, **kw) as lbm:
        if steps:
            lbm.step(steps)
        return lbm.fields()


def _same(got, want, storage, case):
    """Bit for bit, except an FP32 cavity: the engine steps it with two
    cells of a column a thread, a single lattice with x-pairs, and the two
    round FP32 differently (within 1e-5 of max |field|)."""
    if storage == "f32" and case == "cavity":
        return np.abs(got - want).max() <= 1e-5 * max(np.abs(want).max(), 1e-30)
    return np.array_equal(got, want)


@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f64", "fast"), ("f16", "fast"), ("f32", "fast")])
def test_instances_match_single_lattices(api, storage, arith):
    steps_a, steps_b = 23, 18
    with api.Engine(storage=storage, arith=arith, budget_bytes=1 << 30, max_instances=16) as eng:
        slots = [eng.add(api.instance_desc(c, *n, tau, 1.0, u0, **kw)) for c, n, tau, u0, kw in MIX[:3]]
        eng.step(steps_a)  # odd: the late instances join at the other parity
        late = [eng.add(api.instance_desc(c, *n, tau, 1.0, u0, **kw)) for c, n, tau, u0, kw in MIX[3:]]
        eng.step(steps_b)
        got = {s: eng.fields(s) for s in slots + late}
        eng.remove(slots[1])  # the cavity leaves; the others carry on
        eng.step(5)
        got_after = {s: eng.fields(s) for s in (slots[0], late[0])}
    for (c, n, tau, u0, kw), s in zip(MIX[:3], slots):
        want = alone(api, c, n, tau, u0, kw, steps_a + steps_b, storage, arith)
        for k in "uvwp":
            assert _same(got[s][k], want[k], storage, c), (c, k, np.abs(got[s][k] - want[k]).max())
    for (c, n, tau, u0, kw), s in zip(MIX[3:], late):
        want = alone(api, c, n, tau, u0, kw, steps_b, storage, arith)
        for k in "uvwp":
            assert _same(got[s][k], want[k], storage, c), (c, k)
    c, n, tau, u0, kw = MIX[0]
    want = alone(api, c, n, tau, u0, kw, steps_a + steps_b + 5, storage, arith)
    assert _same(got_after[slots[0]]["u"], want["u"], storage, c)
    c, n, tau, u0, kw = MIX[3]
    want = alone(api, c, n, tau, u0, kw, steps_b + 5, storage, arith)
    assert _same(got_after[late[0]]["u"], want["u"], storage, c)


def test_tile_widths_do_not_change_results(api):
    outs = []
    for bx in (0, 8, 16, 32, 64, 128):  # 0: rows staged in shared memory
        with api.Engine(storage="f16", budget_bytes=1 << 28, max_instances=2) as eng:
            s = eng.add(api.instance_desc("cavity", 40, 24, 20, 0.03, 1.0, 0.1, lid_u=0.1, tile_bx=bx))
            eng.step(30)
            outs.append(eng.fields(s))
    for o in outs[1:]:
        for k in "uvwp":
            assert np.array_equal(o[k], outs[0][k])


def test_budget_admission_and_residuals(api):
    d = api.instance_desc("cavity", 32, 32, 32, 0.03, 1.0, 0.1, lid_u=0.1)
    need = api.instance_bytes("f16", d)
    with api.Engine(storage="f16", budget_bytes=2 * need + need // 2, max_instances=8) as eng:
        a = eng.add(d)
        b = eng.add(d)
        assert eng.try_add(d) is None  # over budget
        eng.remove(a)
        c = eng.add(d)  # fits again after a removal
        eng.step(50)
        r1 = eng.residuals()
        assert np.isinf(r1[b]) and np.isinf(r1[c])
        eng.step(50)
        r2 = eng.residuals()
        assert 0.0 < r2[b] < 1.0 and 0.0 < r2[c] < 1.0
        assert np.isnan(r2[a]) or a == c
        st = eng.stats()
        assert st["instances"] == 2 and st["used_bytes"] <= st["budget_bytes"]


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("case,n,kw", [
    ("cavity", (272, 20, 12), dict(lid_u=0.1)),  # rows longer than 256: three rows per tile
    ("sphere", (288, 24, 24), dict(inlet_u=0.05, sphere_d=8.0, sphere_c=(60.0, 12.0, 12.0))),
    ("tgv", (64, 24, 16), {}),  # periodic rows wrap inside the staged row
    ("cavity", (40, 24, 20), dict(lid_u=0.1)),  # rows padded to 48 elements
])
def test_staged_rows_match_register_path(api, storage, case, n, kw):
    """A single 2-byte lattice with standard or periodic boundaries runs the
    shared-memory staged kernel; an engine instance given a tile width runs
    the register-staged x-pair kernel.  Both share the per-cell arithmetic,
    so the fields agree bit for bit."""
    tau, u0, steps = 0.03, 0.05, 40
    with api.Engine(storage=storage, arith="fast", budget_bytes=1 << 30, max_instances=2) as eng:
        s = eng.add(api.instance_desc(case, *n, tau, 1.0, u0, tile_bx=32, **kw))
        eng.step(steps)
        got = eng.fields(s)
    want = alone(api, case, n, tau, u0, kw, steps, storage, "fast")
    for k in "uvwp":
        assert np.array_equal(got[k], want[k]), (case, k, np.abs(got[k] - want[k]).max())


def test_first_residual_after_admission_is_infinite(api):
    """An instance admitted into memory another instance used before reads
    +inf (no previous field yet) on its first residual check, not NaN."""
    d = api.instance_desc("tgv", 32, 32, 32, 0.02, 1.0, 0.05)
    with api.Engine(storage="f16", budget_bytes=api.instance_bytes("f16", d) + (8 << 20), max_instances=2) as eng:
        a = eng.add(d)
        eng.step(20)
        eng.residuals()
        eng.step(20)
        r = eng.residuals()
        assert 0.0 < r[a] < 1.0
        eng.remove(a)
        b = eng.add(d)  # same arena bytes, previous field left over
        eng.step(5)
        r = eng.residuals()
        assert np.isinf(r[b])
        eng.step(5)
        r = eng.residuals()
        assert 0.0 < r[b] < 1.0


@pytest.mark.parametrize("storage,arith", [("f64", "exact"), ("f16", "fast"), ("bf16", "fast")])
def test_step_limits_stop_instances_at_their_own_count(api, storage, arith):
    # an instance with a limit stops at exactly that step, with its fields
    # written there, while the others go on; raising the limit resumes it
    with api.Engine(storage=storage, arith=arith, budget_bytes=1 << 30, max_instances=8) as eng:
        slots = [eng.add(api.instance_desc(c, *n, tau, 1.0, u0, **kw)) for c, n, tau, u0, kw in MIX[:3]]
        eng.limit(slots[0], 7)
        eng.limit(slots[1], 0)  # stopped before it starts
        eng.step(12)
        got = {s: eng.fields(s) for s in slots}
        eng.limit(slots[0], None)  # resumes at its own buffer parity
        eng.step(5)
        resumed = eng.fields(slots[0])
    expect = {slots[0]: 7, slots[1]: 0, slots[2]: 12}
    for (c, n, tau, u0, kw), s in zip(MIX[:3], slots):
        want = alone(api, c, n, tau, u0, kw, expect[s], storage, arith)
        for k in "uvwp":
            assert np.array_equal(got[s][k], want[k]), (c, expect[s], k)
    c, n, tau, u0, kw = MIX[0]
    want = alone(api, c, n, tau, u0, kw, 12, storage, arith)
    for k in "uvwp":
        assert np.array_equal(resumed[k], want[k]), k


def test_stopped_instance_reports_negative_residual(api):
    """An instance that took no step since the previous check (stopped at
    its step limit) reports -1, not a residual of 0 that would read as
    convergence; raising its limit brings real residuals back."""
    d = api.instance_desc("cavity", 32, 32, 32, 0.03, 1.0, 0.1, lid_u=0.1)
    with api.Engine(storage="f16", budget_bytes=1 << 30, max_instances=4) as eng:
        a, b = eng.add(d), eng.add(d)
        eng.limit(a, 10)
        eng.step(20)
        r = eng.residuals()
        assert np.isinf(r[a]) and np.isinf(r[b])
        eng.step(20)
        r = eng.residuals()
        assert r[a] == -1.0 and 0.0 < r[b] < 1.0
        eng.limit(a, None)
        eng.step(20)
        r = eng.residuals()
        assert 0.0 < r[a] < 1.0 and 0.0 < r[b] < 1.0
