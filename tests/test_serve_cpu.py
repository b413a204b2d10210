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


class FakeEngine:
    """The engine's step-limit semantics on the host: an instance with a
    limit stops there; fields report the steps each instance took."""

    def __init__(self, **kw):
        self.taken, self.left, self.calls, self.res = {}, {}, [], {}
        self.next = 0

    def try_add(self, desc, storage=None):
        s = self.next
        self.next += 1
        self.taken[s], self.left[s], self.res[s] = 0, None, float("inf")
        return s

    def limit(self, slot, steps):
        self.left[slot] = steps

    def step(self, n):
        self.calls.append(n)
        for s in self.taken:
            k = n if self.left[s] is None else min(n, self.left[s])
            self.taken[s] += k
            if self.left[s] is not None:
                self.left[s] -= k
            self.res[s] = 1.0 / (1 + self.taken[s])  # falls as the solve settles

    def residuals(self):
        return [self.res.get(s, float("inf")) for s in range(max(self.next, 1))]

    def fields(self, slot):
        return {"steps": self.taken[slot], "answer": "fields"}

    def plane(self, slot, k):
        return {"steps": self.taken[slot], "answer": "plane", "k": k}

    def remove(self, slot):
        del self.taken[slot], self.left[slot], self.res[slot]

    def close(self):
        pass


def test_server_retires_each_request_at_its_own_step_count(monkeypatch):
    monkeypatch.setattr(serve.api, "Engine", FakeEngine)
    srv = serve.Server(chunk=100)
    reqs = [serve.Request(i, 0.0, "tgv", (32, 32, 32), 100.0, m, tol=1e-9) for i, m in enumerate((30, 250, 100, 7))]
    for r in reqs:
        assert srv.try_admit(r)
    retired = {}
    while srv.active:
        for req, f, steps, res in srv.advance():
            retired[req.rid] = (f["steps"], steps)
    # every answer is taken at exactly its request's step count
    assert retired == {r.rid: (r.max_steps, r.max_steps) for r in reqs}
    # fixed-length calls (the engine stops each instance at its own count),
    # the last one only as long as the longest remaining request needs
    assert srv.eng.calls == [100, 100, 50]


def test_server_retires_on_the_residual_tolerance(monkeypatch):
    monkeypatch.setattr(serve.api, "Engine", FakeEngine)
    srv = serve.Server(chunk=100)
    req = serve.Request(0, 0.0, "cavity", (32, 32, 32), 100.0, 10_000, tol=1.0 / 150)
    assert srv.try_admit(req)
    out = []
    while srv.active:
        out += srv.advance()
    # residual 1 / (1 + steps) drops under the tolerance after 200 steps
    assert [(r.rid, steps) for r, f, steps, res in out] == [(0, 200)]


def test_server_answers_with_a_plane_or_the_whole_fields(monkeypatch):
    """The default answer is the middle z plane; the requests named in
    full_ids (the accuracy sample) are answered with their whole fields."""
    monkeypatch.setattr(serve.api, "Engine", FakeEngine)
    srv = serve.Server(chunk=100, full_ids={1})
    reqs = [serve.Request(i, 0.0, "cavity", (32, 32, 40), 100.0, 50, tol=1e-9) for i in range(2)]
    for r in reqs:
        assert srv.try_admit(r)
    got = {}
    while srv.active:
        for req, f, steps, res in srv.advance():
            got[req.rid] = f
    assert got[0]["answer"] == "plane" and got[0]["k"] == 20
    assert got[1]["answer"] == "fields"
