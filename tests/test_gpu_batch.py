"""GPU checks of the batched FP16 form at the batched configuration's worst
instances (2000 steps, relative velocity L2 against the FP64 run of the
same instances, bound 1e-3 as the configuration states):

* the storage plan of the FP16 form (FP16 where tau - 1/2 >= 0.015, FP32
  below) keeps every instance within 1e-3, including the 24^3 vortices at
  Re 360-440 (tau - 1/2 = 1.3e-3) that miss it by up to 66x in FP16 alone;
* an instance whose FP64 run diverges is retired with the status
  "diverged" in every format;
* instances of two formats in one engine give, bit for bit, what each gives
  in an engine of its own format.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-3  # relative velocity L2 against FP64 after 2000 steps


@pytest.fixture(scope="module")
def batch():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import batch as b

    return b


def _worst(b):
    S = b.Spec
    return [S("tgv", 24, 440.5, 0.05), S("tgv", 24, 395.5, 0.05), S("tgv", 48, 770.9, 0.05),
            S("cavity", 48, 792.7, 0.05), S("cavity", 24, 454.4, 0.05), S("tgv", 24, 52.7, 0.05),
            S("tgv", 32, 184.6, 0.05), S("tgv", 32, 40.0, 0.05), S("cavity", 64, 200.0, 0.05),
            S("tgv", 64, 120.0, 0.05), S("cavity", 48, 400.0, 0.05)]


def test_fp16_form_within_1e3_at_worst_instances(batch):
    specs = _worst(batch)
    plan = batch.storage_plan(specs, "f16")
    assert "f16" in plan and "f32" in plan
    got = batch.run(specs, "f16", 2000)
    ref = batch.run(specs, "f64", 2000)
    for s, st, g, w in zip(specs, plan, got["fields"], ref["fields"]):
        assert g is not None and w is not None, (s, st)
        err = batch.velocity_l2(g, w)
        assert err <= TOL, (s, st, err)


def test_fp16_alone_misses_where_the_plan_uses_fp32(batch):
    """The marginal instance the plan keeps in FP32 misses the bound in FP16
    (the reason for the plan)."""
    specs = [batch.Spec("tgv", 24, 440.5, 0.05)]
    assert batch.storage_plan(specs, "f16") == ["f32"]
    got = batch.run(specs, "f16-all", 2000)
    ref = batch.run(specs, "f64", 2000)
    assert batch.velocity_l2(got["fields"][0], ref["fields"][0]) > TOL


def test_diverged_instance_is_retired(batch):
    specs = [batch.Spec("tgv", 24, 853.7, 0.05), batch.Spec("cavity", 32, 300.0, 0.05)]
    for storage in ("f64", "f16"):
        r = batch.run(specs, storage, 2000)
        assert r["status"] == ["diverged", "ok"], (storage, r["status"])
        assert r["fields"][0] is None and r["fields"][1] is not None


def test_mixed_formats_match_single_format_engines(batch):
    import torch

    from imexlb_b200 import api

    specs = [batch.Spec("tgv", 32, 200.0, 0.05), batch.Spec("cavity", 48, 100.0, 0.05),
             batch.Spec("tgv", 24, 440.5, 0.05), batch.Spec("cavity", 32, 300.0, 0.05)]
    formats = ["f16", "f32", "f32", "f16"]

    def fields(pairs, engine_storage):
        stream = torch.cuda.Stream()
        budget = sum(api.instance_bytes(st, s.desc()) for s, st in pairs) + (64 << 20)
        with api.Engine(storage=engine_storage, budget_bytes=budget, max_instances=len(pairs),
                        stream=stream.cuda_stream) as eng:
            slots = [eng.add(s.desc(), storage=st) for s, st in pairs]
            eng.step(300)
            return [eng.fields(sl) for sl in slots]

    mixed = fields(list(zip(specs, formats)), "f64")
    for st in ("f16", "f32"):
        alone = fields([(s, f) for s, f in zip(specs, formats) if f == st], st)
        want = iter(alone)
        for got, f in zip(mixed, formats):
            if f != st:
                continue
            w = next(want)
            for k in "uvwp":
                assert np.isfinite(got[k]).all(), (st, k)
                assert np.array_equal(got[k], w[k]), (st, k)
