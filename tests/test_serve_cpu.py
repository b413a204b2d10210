"""Host logic of the serving loop (no GPU): the request stream and the
one-at-a-time FP64 queue model."""
import math

from imexlb_b200 import serve


def test_stream_is_seeded_and_follows_the_mix():
    a = serve.request_stream(2000, 50.0)
    assert a == serve.request_stream(2000, 50.0)
    frac = {c: sum(r.case == c for r in a) / len(a) for c in ("cavity", "tgv", "sphere")}
    assert abs(frac["cavity"] - 0.4) < 0.05 and abs(frac["tgv"] - 0.4) < 0.05 and abs(frac["sphere"] - 0.2) < 0.03
    assert all(5000 <= r.max_steps <= 20000 for r in a)
    for r in a:
        if r.case == "sphere":
            L = r.n[0]
            assert L in serve.SPHERE_L and r.n == (L, L // 4, L // 4) and 20 <= r.Re <= 200
        else:
            assert r.n[0] in serve.EDGES and r.n[0] == r.n[1] == r.n[2]
            assert (100 <= r.Re <= 1000) if r.case == "cavity" else (50 <= r.Re <= 800)
    # Poisson arrivals: mean gap 1 / rate, first request at t = 0
    gaps = [b.arrival - a_.arrival for a_, b in zip(a, a[1:])]
    assert a[0].arrival == 0.0 and all(g >= 0 for g in gaps)
    assert abs(sum(gaps) / len(gaps) - 1 / 50.0) < 0.1 / 50.0
    # the same requests at another rate, only the times differ
    b = serve.request_stream(2000, 5.0)
    assert [(r.case, r.n, r.Re, r.max_steps) for r in a] == [(r.case, r.n, r.Re, r.max_steps) for r in b]


def test_fifo_one_at_a_time():
    reqs = [serve.Request(i, t, "tgv", (32, 32, 32), 100.0, 10) for i, t in enumerate([0.0, 0.5, 0.6, 5.0])]
    service = {i: dict(service=1.0, steps=10) for i in range(4)}
    q = serve.fifo_one_at_a_time(reqs, service)
    # finishes at 1, 2, 3, 6 -> latencies 1, 1.5, 2.4, 1
    assert math.isclose(q["p50"], 1.25) and math.isclose(q["span"], 6.0)
    assert math.isclose(q["solves_per_s"], 4 / 6.0)
