"""Host logic of the batched configuration and the autotuner cache (no GPU)."""
import json
import math

from imexlb_b200 import batch, tune


def test_batch_is_seeded_and_spans_the_mix():
    a, b = batch.batch_specs(), batch.batch_specs()
    assert a == b and len(a) == 256
    assert {s.case for s in a} == {"tgv", "cavity"}
    assert {s.edge for s in a} == set(batch.EDGES)
    assert all(50.0 <= s.Re <= 1000.0 for s in a)
    tgv = sum(s.case == "tgv" for s in a)
    assert 100 < tgv < 156  # 50/50 draw
    assert batch.batch_specs(seed=1) != a


def test_tau_follows_the_reference_system():
    # tgv/src/System.cpp:21: tau = u0*sx/Re/cs2/2/pi with pi = 3.1415926;
    # lid_driven_cavity/src/System.cpp:19: tau = u0*R/Re/cs2
    s = batch.Spec("tgv", 64, 100.0, 0.05)
    assert math.isclose(s.tau0, 0.05 * 64 / 100.0 / (1.0 / 3.0) / 2 / 3.1415926, rel_tol=1e-15)
    c = batch.Spec("cavity", 128, 1000.0, 0.1)
    assert math.isclose(c.tau0 + 0.5, 0.5384, rel_tol=1e-12)


def test_velocity_l2():
    import numpy as np

    want = {k: np.ones((2, 2, 2)) for k in "uvw"}
    got = {k: v.copy() for k, v in want.items()}
    assert batch.velocity_l2(got, want) == 0.0
    got["u"] = got["u"] * 1.1
    assert math.isclose(batch.velocity_l2(got, want), math.sqrt(0.01 * 8 / 24))


def test_tiles_come_from_the_cache(tmp_path):
    specs = [batch.Spec("cavity", 48, 100.0, 0.05), batch.Spec("tgv", 24, 80.0, 0.05)]
    cache = tmp_path / "t.json"
    entries = {tune.key_of("f16", "cavity", (48,) * 3): {"tile_bx": 32, "ns_per_cell": 0.1},
               tune.key_of("f16", "tgv", (24,) * 3): {"tile_bx": 0, "ns_per_cell": 0.2}}
    cache.write_text(json.dumps({"device": "x", "entries": entries}))
    tiles = tune.tiles_for(specs, "f16", cache=str(cache), tune_missing=False)
    assert tiles["f16/cavity/48x48x48"] == 32 and tiles["f16/tgv/24x24x24"] == 0


def test_fp16_storage_plan():
    """The FP16 form stores marginally stable instances (tau - 1/2 below
    FP16_MIN_TAU0) in FP32; "f16-all" and the other formats store every
    instance in one format."""
    from imexlb_b200 import batch, serve

    specs = batch.batch_specs(256)
    plan = batch.storage_plan(specs, "f16")
    assert all((st == "f16") == (s.tau0 >= batch.FP16_MIN_TAU0) for s, st in zip(specs, plan))
    assert 0 < plan.count("f32") < plan.count("f16")
    assert batch.storage_plan(specs, "f16-all") == ["f16"] * 256
    assert batch.storage_plan(specs, "f32") == ["f32"] * 256
    assert batch.engine_storage("f16-all") == "f16"
    reqs = serve.request_stream(200, 10.0)
    for r in reqs:
        if r.case == "tgv":
            want = "f32" if r.tau0 >= serve.TGV_FP32_MIN_TAU0 else "f64"
        else:
            want = "f16" if r.tau0 >= batch.FP16_MIN_TAU0 else "f32"
        assert serve.storage_for(r, "f16") == want
        assert serve.storage_for(r, "f64") == "f64"
