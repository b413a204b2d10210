"""Served solve stream: requests arrive over time and share the GPU.

The reference solves one lattice per process run; this is the serving loop
of this project over the engine (imexlb_engine_*).  Requests arrive as a
Poisson process of rate lambda; each asks for a TGV, lid-driven cavity or
sphere-channel solve of its own size and Re, to a step count or until the
steady residual (relative change of the velocity field between two checks)
falls below a tolerance.  The loop does continuous batching:

* admission: waiting requests are admitted in arrival order as instances
  of one engine while they fit its HBM budget (cells x bytes per cell, the
  engine's arena refuses what does not fit) and the active cells stay under
  a cap that already fills the GPU; the lattices stay resident in HBM;
* stepping: all admitted instances advance together, `chunk` steps per call,
  as persistent launches replayed from CUDA graphs; each instance carries
  its request's step count as an engine step limit (imexlb_engine_limit),
  so it stops at exactly that step, with its fields written there, while
  the others go on;
* retirement: after each call the residuals are read; an instance that
  reached its step count or the tolerance is retired, its u, v, w, p are
  read back to the host (the request's answer) and its memory is freed for
  the next admission.

Latency = answer read back - arrival, on the host clock.  The baseline is
one-at-a-time plain FP64: each request alone on the GPU, its service time
measured once, queued in arrival order (a single server).

The request mix: 40% cavity (edge 32..128 in steps of 16, Re 100..1000),
40% TGV (edge 32..128, Re 50..800), 20% sphere channel (L x L/4 x L/4,
L in {256, 384, 512}, diameter L/24, Re 20..200), 5000..20000 steps or a
1e-6 residual; Re log-uniform, U0 = u_w = inlet speed = 0.05.

    python -m imexlb_b200.serve --rates 1,20,200 --count 40
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import time

import numpy as np

from . import api

SERVE_SEED = 7051
EDGES = (32, 48, 64, 80, 96, 112, 128)
SPHERE_L = (256, 384, 512)
U = 0.05


@dataclasses.dataclass(frozen=True)
class Request:
    rid: int
    arrival: float   # seconds after the stream starts
    case: str
    n: tuple
    Re: float
    max_steps: int
    tol: float = 1e-6

    @property
    def cells(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    @property
    def tau0(self) -> float:
        if self.case == "tgv":
            return 3.0 * U * (self.n[0] / 2.0 / 3.1415926) / self.Re
        if self.case == "sphere":
            return 3.0 * U * (self.n[0] / 24.0) / self.Re
        return 3.0 * U * self.n[0] / self.Re

    def desc(self, tile_bx: int = 0) -> api.InstanceDesc:
        kw = {}
        if self.case == "cavity":
            kw = dict(lid_u=U)
        elif self.case == "sphere":
            kw = dict(inlet_u=U, sphere_d=self.n[0] / 24.0)
        return api.instance_desc(self.case, *self.n, self.tau0, 1.0, U, tile_bx=tile_bx, **kw)


def request_stream(count: int, rate: float, seed: int = SERVE_SEED, steps=(5000, 20000), tol: float = 1e-6,
                   scale_steps: float = 1.0) -> list[Request]:
    """`count` requests with Poisson arrivals of `rate` per second.  The mix
    does not depend on the rate (same seed: same requests, other times)."""
    rng = np.random.default_rng(seed)
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, count)
    t = np.cumsum(gaps) - gaps[0]
    out = []
    for i in range(count):
        r = rng.random()
        if r < 0.4:
            case, e = "cavity", int(rng.choice(EDGES))
            n, Re = (e, e, e), math.exp(rng.uniform(math.log(100.0), math.log(1000.0)))
        elif r < 0.8:
            case, e = "tgv", int(rng.choice(EDGES))
            n, Re = (e, e, e), math.exp(rng.uniform(math.log(50.0), math.log(800.0)))
        else:
            case, L = "sphere", int(rng.choice(SPHERE_L))
            n, Re = (L, L // 4, L // 4), math.exp(rng.uniform(math.log(20.0), math.log(200.0)))
        ms = int(rng.integers(steps[0], steps[1] + 1) * scale_steps)
        out.append(Request(i, float(t[i]), case, n, float(Re), max(1, ms), tol))
    return out


class Server:
    """Continuous batching of requests into one engine."""

    def __init__(self, storage: str = "f16", budget_bytes: int = 150 << 30, max_active_cells: int = 48 << 20,
                 max_instances: int = 512, chunk: int = 200, tiles: dict | None = None, stream=None):
        self.storage = storage
        self.eng = api.Engine(storage=storage, arith="fast", budget_bytes=budget_bytes, max_instances=max_instances,
                              stream=stream)
        self.max_active_cells = max_active_cells
        self.chunk = chunk
        self.tiles = tiles or {}
        self.active: dict[int, tuple] = {}   # slot -> (request, steps done)
        self.steps_run = 0

    def close(self):
        self.eng.close()

    def _tile(self, req: Request) -> int:
        from . import tune

        return self.tiles.get(tune.key_of(self.storage, req.case, req.n), 0)

    def try_admit(self, req: Request) -> bool:
        cells = sum(r.cells for r, _ in self.active.values())
        if self.active and cells + req.cells > self.max_active_cells:
            return False
        slot = self.eng.try_add(req.desc(self._tile(req)))
        if slot is None:
            return False
        self.eng.limit(slot, req.max_steps)
        self.active[slot] = (req, 0)
        return True

    def launch(self) -> int:
        """Queue one stepping call for the admitted instances and return at
        once; the steps run while the host admits more requests."""
        if not self.active:
            return 0
        n = min(self.chunk, max(r.max_steps - done for r, done in self.active.values()))
        self.eng.step(n)
        self.steps_run += n
        self._stepped = (n, set(self.active))
        return n

    def collect(self) -> list[tuple]:
        """Wait for the queued steps, read the residuals and retire; returns
        [(request, fields, steps, residual)] of the retired requests.
        Requests admitted after launch() did not take part in its steps."""
        n, stepped = getattr(self, "_stepped", (0, set()))
        self._stepped = (0, set())
        if not n:
            return []
        res = self.eng.residuals()
        done_now = []
        for slot in list(self.active):
            if slot not in stepped:
                continue
            req, done = self.active[slot]
            done += min(n, req.max_steps - done)  # the engine stops it at its step count
            self.active[slot] = (req, done)
            r = float(res[slot])
            # retire at the step count, at the tolerance, or when the lattice
            # diverged (NaN); the first check after admission reads +inf
            if done >= req.max_steps or r < req.tol or math.isnan(r):
                f = self.eng.fields(slot)
                self.eng.remove(slot)
                del self.active[slot]
                done_now.append((req, f, done, r))
        return done_now

    def advance(self) -> list[tuple]:
        """One stepping call and its retirements."""
        self.launch()
        return self.collect()


def serve(requests: list[Request], storage: str = "f16", keep_fields: bool = False, **kw) -> dict:
    """Run the stream in real time; latencies and throughput on the host clock."""
    import torch

    stream = torch.cuda.Stream()
    srv = Server(storage=storage, stream=stream.cuda_stream, **kw)
    waiting = list(requests)
    results = {}
    t0 = time.perf_counter()
    def admit_arrived():
        now = time.perf_counter() - t0
        while waiting and waiting[0].arrival <= now and srv.try_admit(waiting[0]):
            waiting.pop(0)
        return now

    try:
        while waiting or srv.active:
            now = admit_arrived()
            if not srv.active:
                if waiting[0].arrival <= now:
                    raise RuntimeError(f"request {waiting[0].rid} does not fit the engine's memory budget")
                # idle until the next arrival
                time.sleep(max(0.0, waiting[0].arrival - (time.perf_counter() - t0)))
                continue
            srv.launch()
            admit_arrived()  # host set-up of new arrivals overlaps the queued steps
            for req, f, steps, r in srv.collect():
                t = time.perf_counter() - t0
                results[req.rid] = dict(latency=t - req.arrival, steps=steps, residual=r,
                                        fields=f if keep_fields else None)
    finally:
        srv.close()
    span = time.perf_counter() - t0
    lat = np.array([results[r.rid]["latency"] for r in requests])
    work = sum(results[r.rid]["steps"] * r.cells for r in requests)
    return dict(results=results, span=span, p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)),
                solves_per_s=len(requests) / span, mlups=work / span / 1e6)


def service_times_alone(requests: list[Request], storage: str = "f64", chunk: int = 200) -> dict:
    """Each request alone on the GPU (its own engine, one instance): host
    time from admission to its answer read back."""
    import torch

    stream = torch.cuda.Stream()
    out = {}
    for req in requests:
        d = req.desc()
        budget = api.instance_bytes(storage, d) + (64 << 20)
        torch.cuda.synchronize()
        t = time.perf_counter()
        srv = Server(storage=storage, budget_bytes=budget, max_instances=1, chunk=chunk, stream=stream.cuda_stream)
        try:
            assert srv.try_admit(req)
            done = []
            while not done:
                done = srv.advance()
            _, f, steps, r = done[0]
        finally:
            srv.close()
        out[req.rid] = dict(service=time.perf_counter() - t, steps=steps, residual=r)
    return out


def fifo_one_at_a_time(requests: list[Request], service: dict) -> dict:
    """Single-server queue in arrival order with the measured service times."""
    free = 0.0
    lat = []
    for r in requests:
        start = max(free, r.arrival)
        free = start + service[r.rid]["service"]
        lat.append(free - r.arrival)
    span = free - requests[0].arrival
    work = sum(service[r.rid]["steps"] * r.cells for r in requests)
    return dict(p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)),
                solves_per_s=len(requests) / span, mlups=work / span / 1e6, span=span)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--rates", default="1,20,200")
    ap.add_argument("--count", type=int, default=40)
    ap.add_argument("--storage", default="f16")
    ap.add_argument("--scale-steps", type=float, default=1.0, help="multiply the 5000..20000 step counts")
    ap.add_argument("--max-active-cells", type=int, default=48 << 20)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--no-baseline", action="store_true")
    args = ap.parse_args(argv)
    from . import tune

    rates = [float(x) for x in args.rates.split(",")]
    base_reqs = request_stream(args.count, rates[0], scale_steps=args.scale_steps)
    tiles = tune.load(None)
    tiles = {k: v["tile_bx"] for k, v in tiles.items()}
    alone = None if args.no_baseline else service_times_alone(base_reqs, "f64")
    for rate in rates:
        reqs = request_stream(args.count, rate, scale_steps=args.scale_steps)
        res = serve(reqs, args.storage, budget_bytes=int(args.budget_gb * (1 << 30)),
                    max_active_cells=args.max_active_cells, tiles=tiles)
        line = dict(rate=rate, count=args.count, storage=args.storage, p50_s=res["p50"], p99_s=res["p99"],
                    solves_per_s=res["solves_per_s"], mlups=res["mlups"], span_s=res["span"],
                    steps_scale=args.scale_steps)
        if alone:
            b = fifo_one_at_a_time(reqs, alone)
            line["fp64_one_at_a_time"] = dict(p50_s=b["p50"], p99_s=b["p99"], solves_per_s=b["solves_per_s"],
                                              mlups=b["mlups"])
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
