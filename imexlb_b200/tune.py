"""Autotuner of the engine's tile shape and thread-to-cell mapping.

For every lattice shape, case rule and storage format the engine can run a
tile in several ways: FP64 and FP32 tiles of 2^b threads along x (one cell
per thread for FP64, a y-pair per thread for FP32); 2-byte tiles either of
whole rows staged in shared memory (tile_bx = 0, x-pairs read from the
stage) or of 2^b x-pairs read straight from global memory.  Which is
fastest depends on the row length (padding waste, coalescing) and on the
rule, so it is measured: each candidate runs an engine holding copies of the
shape (enough cells to fill the GPU), timed with CUDA events on the engine's
stream, and the fastest per key is kept in a JSON cache

    {"device": "...", "entries": {"f16/cavity/48x48x48": {"tile_bx": 0, "ns_per_cell": ...}}}

which the batch and the serving loop read (tiles_for).  The reference has no
tuner (one lattice per process).

    python -m imexlb_b200.tune --storage f16 --cache tuned.json
"""
from __future__ import annotations

import argparse
import json
import os

from . import api

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CACHE = os.path.join(HERE, "tuned_b200.json")
CANDIDATES_2B = (0, 16, 32, 64, 128)
CANDIDATES = (16, 32, 64, 128)
FILL_CELLS = 4 << 20   # copies of a shape up to about this many cells
MAX_COPIES = 64


def key_of(storage: str, case: str, n) -> str:
    rule = "tgv" if case == "tgv" else case
    return f"{storage}/{rule}/{n[0]}x{n[1]}x{n[2]}"


def candidates(storage: str):
    return CANDIDATES_2B if storage in ("f16", "bf16") else CANDIDATES


def _desc(case: str, n, tile_bx: int) -> api.InstanceDesc:
    tau = 3.0 * 0.05 * n[0] / 500.0
    kw = dict(lid_u=0.05) if case == "cavity" else {}
    if case == "sphere":
        kw = dict(inlet_u=0.05, sphere_d=n[0] / 24.0)
    return api.instance_desc(case, *n, tau, 1.0, 0.05, tile_bx=tile_bx, **kw)


def measure(storage: str, case: str, n, tile_bx: int, steps: int = 12, arith: str = "fast") -> float:
    """Nanoseconds per cell update of `copies` instances of the shape."""
    import torch

    cells = n[0] * n[1] * n[2]
    copies = max(1, min(MAX_COPIES, FILL_CELLS // cells))
    d = _desc(case, n, tile_bx)
    budget = copies * api.instance_bytes(storage, d) + (64 << 20)
    stream = torch.cuda.Stream()
    with api.Engine(storage=storage, arith=arith, budget_bytes=budget, max_instances=copies,
                    stream=stream.cuda_stream) as eng:
        for _ in range(copies):
            eng.add(d)
        eng.step(4)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step(steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    return ms * 1e6 / (copies * cells * steps)


def tune_shapes(shapes, storage: str, arith: str = "fast") -> dict:
    """shapes: iterable of (case, (nx, ny, nz)); returns key -> entry."""
    out = {}
    for case, n in sorted(set((c, tuple(n)) for c, n in shapes)):
        best = None
        times = {}
        for bx in candidates(storage):
            t = measure(storage, case, n, bx, arith=arith)
            times[str(bx)] = t
            if best is None or t < best[1]:
                best = (bx, t)
        out[key_of(storage, case, n)] = dict(tile_bx=best[0], ns_per_cell=best[1], candidates=times)
    return out


def load(cache: str | None) -> dict:
    path = cache or DEFAULT_CACHE
    if not os.path.exists(path):
        return {}
    with open(path) as fh:
        return json.load(fh).get("entries", {})


def save(entries: dict, cache: str) -> None:
    import torch

    old = {}
    if os.path.exists(cache):
        with open(cache) as fh:
            old = json.load(fh).get("entries", {})
    old.update(entries)
    with open(cache, "w") as fh:
        json.dump({"device": torch.cuda.get_device_name(), "entries": old}, fh, indent=1, sort_keys=True)


def tiles_for(specs, storage: str, cache: str | None = None, tune_missing: bool = True) -> dict:
    """key -> tile_bx for every shape in `specs` (objects with .case and
    .edge), from the cache, tuning the shapes it lacks."""
    entries = load(cache)
    shapes = {(s.case, (s.edge,) * 3) for s in specs}
    missing = [(c, n) for c, n in shapes if key_of(storage, c, n) not in entries]
    if missing and tune_missing:
        new = tune_shapes(missing, storage)
        entries.update(new)
        if cache:
            save(new, cache)
    return {k: v["tile_bx"] for k, v in entries.items()}


def main(argv=None) -> int:
    from .batch import EDGES

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--storage", default="f16", choices=sorted(api.STORAGES))
    ap.add_argument("--cache", default=DEFAULT_CACHE)
    args = ap.parse_args(argv)
    shapes = [(c, (e, e, e)) for c in ("tgv", "cavity") for e in EDGES]
    entries = tune_shapes(shapes, args.storage)
    save(entries, args.cache)
    for k, v in sorted(entries.items()):
        print(k, v["tile_bx"], f"{v['ns_per_cell']:.4f} ns/cell", v["candidates"])
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
