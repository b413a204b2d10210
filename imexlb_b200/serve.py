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
  reached its step count or the tolerance is retired, its answer is read
  back to the host and its memory is freed for the next admission.  The
  answer is the u, v, w, p of the lattice's middle z plane (answer="plane",
  the default: a cut through the flow, at most 2 MB) or of the whole lattice
  (answer="fields": up to 268 MB for the largest sphere channel, 77 GB for
  the configuration's 2000 requests, which would make the stream a test of
  the host link rather than of the solver).

Storage: with storage "f16" (storage_for; one engine holds every format)
a cavity or sphere request is stored in FP16 when its tau - 1/2 is at least
imexlb_b200.batch.FP16_MIN_TAU0 and in FP32 otherwise; its FP16 stores round
stochastically, so that their error stays at a few 1e-4 over the 5000-20000
steps instead of growing with the step count.  A Taylor-Green vortex, a
decaying flow whose FP16 error against FP64 grows past 1e-3 within a few
thousand steps, is stored in FP32 when tau - 1/2 is at least
TGV_FP32_MIN_TAU0 and in FP64 below it, where the collision's FP32 rounding
grows past 1e-3 by 10000-20000 steps (measured on 32^3-128^3 vortices at
Re 100-800).  A request whose lattice goes non-finite is retired with the
status "diverged" and no fields.

Latency = answer read back - arrival, on the host clock.  The baseline is
one-at-a-time plain FP64 queued in arrival order (a single server): each
request alone on the GPU in its own engine, with its service time either
measured whole (small streams) or, for long streams, composed from
measurements per lattice shape: the fixed cost (admission, set-up, answer
read-back) and the time per step of that shape alone, times the request's
own step count.  A sample of the served answers is checked against FP64
runs of the same requests to the same step counts (relative velocity L2).

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
from .batch import FP16_MIN_TAU0

# below this tau - 1/2 the served FP16 form stores a vortex in FP64
TGV_FP32_MIN_TAU0 = 0.005

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


def storage_for(req: Request, storage: str) -> str:
    """A request's storage format in the served FP16 form (module docstring):
    cavity and sphere in FP16 (FP32 when tau - 1/2 < FP16_MIN_TAU0), the
    vortex in FP32 (FP64 when tau - 1/2 < TGV_FP32_MIN_TAU0); other formats
    store every request in themselves."""
    if storage != "f16":
        return storage
    if req.case == "tgv":
        return "f32" if req.tau0 >= TGV_FP32_MIN_TAU0 else "f64"
    return "f16" if req.tau0 >= FP16_MIN_TAU0 else "f32"


class Server:
    """Continuous batching of requests into one engine."""

    def __init__(self, storage: str = "f16", budget_bytes: int = 150 << 30, max_active_cells: int = 48 << 20,
                 max_instances: int = 512, chunk: int = 200, tiles: dict | None = None, stream=None,
                 answer: str = "plane", full_ids=()):
        self.storage = storage
        self.answer = answer
        self.full_ids = set(full_ids)  # requests answered with their whole fields
        self.eng = api.Engine(storage=storage, arith="fast", budget_bytes=budget_bytes, max_instances=max_instances,
                              stream=stream)
        self.max_active_cells = max_active_cells
        self.chunk = chunk
        self.tiles = tiles or {}
        self.active: dict[int, tuple] = {}   # slot -> (request, steps done)
        self.steps_run = 0

    def close(self):
        self.eng.close()

    def _tile(self, req: Request, storage: str) -> int:
        from . import tune

        return self.tiles.get(tune.key_of(storage, req.case, req.n), 0)

    def try_admit(self, req: Request) -> bool:
        cells = sum(r.cells for r, _ in self.active.values())
        if self.active and cells + req.cells > self.max_active_cells:
            return False
        st = storage_for(req, self.storage)
        slot = self.eng.try_add(req.desc(self._tile(req, st)), storage=st)
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
        [(request, answer, steps, residual)] of the retired requests (the
        middle z plane or the whole fields, see the module docstring; None
        for a diverged one).  Requests admitted after launch() did not take
        part in its steps."""
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
            if done >= req.max_steps or 0 <= r < req.tol or math.isnan(r):
                if math.isnan(r):
                    f = None
                elif self.answer == "fields" or req.rid in self.full_ids:
                    f = self.eng.fields(slot)
                else:
                    f = self.eng.plane(slot, req.n[2] // 2)
                self.eng.remove(slot)
                del self.active[slot]
                done_now.append((req, f, done, r))
        return done_now

    def advance(self) -> list[tuple]:
        """One stepping call and its retirements."""
        self.launch()
        return self.collect()


def status_of(req: Request, steps: int, residual: float) -> str:
    if math.isnan(residual):
        return "diverged"
    # a negative residual: the instance took no step since the last check
    return "converged" if 0 <= residual < req.tol and steps < req.max_steps else "steps"


def serve(requests: list[Request], storage: str = "f16", keep_fields=False, **kw) -> dict:
    """Run the stream in real time; latencies and throughput on the host
    clock.  keep_fields: True, or a set of request ids whose answers to keep."""
    import torch

    stream = torch.cuda.Stream()
    full = keep_fields if isinstance(keep_fields, (set, frozenset, list, tuple)) else ()
    if keep_fields is True:
        kw["answer"] = "fields"
    srv = Server(storage=storage, stream=stream.cuda_stream, full_ids=full, **kw)
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
                keep = keep_fields is True or (keep_fields and req.rid in keep_fields)
                results[req.rid] = dict(latency=t - req.arrival, steps=steps, residual=r,
                                        status=status_of(req, steps, r), storage=storage_for(req, storage),
                                        fields=f if keep else None)
    finally:
        srv.close()
    span = time.perf_counter() - t0
    lat = np.array([results[r.rid]["latency"] for r in requests])
    work = sum(results[r.rid]["steps"] * r.cells for r in requests)
    status = [results[r.rid]["status"] for r in requests]
    return dict(results=results, span=span, p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)),
                solves_per_s=len(requests) / span, mlups=work / span / 1e6,
                status={k: status.count(k) for k in sorted(set(status))},
                storage={k: sum(1 for r in requests if results[r.rid]["storage"] == k)
                         for k in sorted({results[r.rid]["storage"] for r in requests})})


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


def run_alone(req: Request, storage: str, steps: int, chunk: int = 200, stream=None, answer: str = "fields"):
    """One request alone in its own engine for exactly `steps` steps: host
    seconds from admission to its answer (the whole fields, or the middle z
    plane) read back, and the answer."""
    import torch

    d = req.desc()
    budget = api.instance_bytes(storage, d) + (64 << 20)
    torch.cuda.synchronize()
    t = time.perf_counter()
    with api.Engine(storage=storage, arith="fast", budget_bytes=budget, max_instances=1, stream=stream) as eng:
        slot = eng.add(d)
        left = steps
        while left > 0:
            n = min(chunk, left)
            eng.step(n)
            eng.residuals()  # the per-call check the serving loop makes
            left -= n
        f = eng.fields(slot) if answer == "fields" else eng.plane(slot, req.n[2] // 2)
    return time.perf_counter() - t, f


def service_model_by_shape(requests: list[Request], storage: str = "f64", probes=(200, 1000)) -> dict:
    """Per (case, shape): the fixed cost and the time per step of one request
    alone on the GPU, from two runs of probes[0] and probes[1] steps (the
    second minus the first gives the per-step time)."""
    import torch

    stream = torch.cuda.Stream()
    shapes = sorted({(r.case, r.n) for r in requests})
    out = {}
    for case, n in shapes:
        req = next(r for r in requests if (r.case, r.n) == (case, n))
        run_alone(req, storage, 20, stream=stream.cuda_stream, answer="plane")  # warm the kernels of this shape
        t1, _ = run_alone(req, storage, probes[0], stream=stream.cuda_stream, answer="plane")
        t2, _ = run_alone(req, storage, probes[1], stream=stream.cuda_stream, answer="plane")
        per_step = max(0.0, (t2 - t1) / (probes[1] - probes[0]))
        out[(case, n)] = dict(fixed=max(0.0, t1 - per_step * probes[0]), per_step=per_step)
    return out


def modelled_service(requests: list[Request], model: dict, steps: dict) -> dict:
    """Service time of each request alone: fixed + steps x per-step of its shape."""
    out = {}
    for r in requests:
        m = model[(r.case, r.n)]
        out[r.rid] = dict(service=m["fixed"] + steps[r.rid] * m["per_step"], steps=steps[r.rid])
    return out


def accuracy_sample(requests: list[Request], results: dict, rids) -> dict:
    """Relative velocity L2 of served answers against FP64 runs of the same
    requests alone to the same step counts."""
    import torch

    from .batch import velocity_l2

    stream = torch.cuda.Stream()
    errs = []
    by_id = {r.rid: r for r in requests}
    for rid in rids:
        res = results[rid]
        if res["fields"] is None:
            continue
        _, want = run_alone(by_id[rid], "f64", res["steps"], stream=stream.cuda_stream)
        errs.append(dict(rid=rid, case=by_id[rid].case, n=by_id[rid].n, Re=round(by_id[rid].Re, 1),
                         storage=res["storage"], steps=res["steps"], err=velocity_l2(res["fields"], want)))
    vals = np.array([e["err"] for e in errs]) if errs else np.array([np.nan])
    return dict(checked=len(errs), max=float(vals.max()), p95=float(np.percentile(vals, 95)),
                median=float(np.median(vals)), over_1e3=int((vals > 1e-3).sum()),
                worst=sorted(errs, key=lambda e: -e["err"])[:5])


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
    ap.add_argument("--baseline", choices=["measured", "by-shape"], default="measured",
                    help="one-at-a-time FP64: every request measured whole, or fixed + per-step time per shape")
    ap.add_argument("--check-error", type=int, default=0,
                    help="check this many served answers (seeded sample) against FP64 runs alone")
    ap.add_argument("--out", default=None, help="append each rate's JSON line to this file")
    ap.add_argument("--answer", choices=["plane", "fields"], default="plane",
                    help="what a retired request reads back: its middle z plane or its whole fields")
    args = ap.parse_args(argv)
    from . import tune

    rates = [float(x) for x in args.rates.split(",")]
    base_reqs = request_stream(args.count, rates[0], scale_steps=args.scale_steps)
    tiles = tune.load(None)
    tiles = {k: v["tile_bx"] for k, v in tiles.items()}
    alone = None
    if not args.no_baseline and args.baseline == "measured":
        alone = service_times_alone(base_reqs, "f64")
    model = None
    if not args.no_baseline and args.baseline == "by-shape":
        model = service_model_by_shape(base_reqs, "f64")
    for rate in rates:
        reqs = request_stream(args.count, rate, scale_steps=args.scale_steps)
        sample = set()
        if args.check_error:
            rng = np.random.default_rng(SERVE_SEED + 2)
            sample = set(int(x) for x in rng.choice(len(reqs), min(args.check_error, len(reqs)), replace=False))
        t0 = time.perf_counter()
        res = serve(reqs, args.storage, budget_bytes=int(args.budget_gb * (1 << 30)),
                    max_active_cells=args.max_active_cells, tiles=tiles, keep_fields=sample, answer=args.answer)
        line = dict(rate=rate, count=args.count, storage=args.storage, p50_s=res["p50"], p99_s=res["p99"],
                    solves_per_s=res["solves_per_s"], mlups=res["mlups"], span_s=res["span"],
                    steps_scale=args.scale_steps, status=res["status"], storage_requests=res["storage"],
                    answer=args.answer,
                    wall_s=time.perf_counter() - t0)
        steps = {r.rid: res["results"][r.rid]["steps"] for r in reqs}
        base = None
        if alone:
            base, how = fifo_one_at_a_time(reqs, alone), "each request measured alone"
        elif model:
            base = fifo_one_at_a_time(reqs, modelled_service(reqs, model, steps))
            how = "fixed + per-step time per shape measured alone, times each request's served step count"
        if base:
            line["fp64_one_at_a_time"] = dict(p50_s=base["p50"], p99_s=base["p99"],
                                              solves_per_s=base["solves_per_s"], mlups=base["mlups"], how=how)
        if sample:
            line["accuracy_vs_fp64"] = accuracy_sample(reqs, res["results"], sorted(sample))
        print(json.dumps(line), flush=True)
        if args.out:
            with open(args.out, "a") as fh:
                fh.write(json.dumps(line) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
