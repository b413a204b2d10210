"""The accuracy study's lattices use the served mix's tau - 1/2 (no GPU)."""
from imexlb_b200 import accuracy, serve


def test_tau0_matches_the_served_requests():
    for r in serve.request_stream(300, 10.0):
        assert accuracy.tau0_of(r.case, r.n[0], r.Re) == r.tau0


def test_default_cases_cover_the_storage_plan_thresholds():
    taus = {(c, st): [] for c in ("cavity", "sphere", "tgv") for st in ("f16", "f32")}
    for case, n, Re, storages in accuracy.DEFAULT_CASES:
        for st in storages.split(","):
            if (case, st) in taus:
                taus[(case, st)].append(accuracy.tau0_of(case, n, Re))
    # vortices in FP32 on both sides of the served plan's FP32 / FP64 threshold
    assert min(taus[("tgv", "f32")]) < serve.TGV_FP32_MIN_TAU0 < max(taus[("tgv", "f32")])
    assert taus[("cavity", "f16")] and taus[("sphere", "f16")]
