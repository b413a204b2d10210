#!/usr/bin/env python
"""Benchmark of the fused D3Q27 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload: the lid-driven cavity, plain FP64, 128^3 lattice, halfway
bounce-back on five walls and a lid moving at u_w = (0.1, 0, 0) with the
-2 w_i rho (c_i . u_w)/cs^2 correction, Re = 1000 (nu = 0.1*128/1000,
tau = 0.5 + 3 nu).  A "step" is one lattice time step over the whole box.
Metric: MLUPS (million lattice-cell updates per second), whole job.

* value     device-resident throughput: K steps on the lattice's stream timed
            with CUDA events (barrier + synchronize on both sides, max over
            ranks); the two 470 MB distribution buffers exceed the 126 MB L2,
            so no flush is needed between steps.
* e2e       the same solve through the public C ABI, host wall clock: create
            (the cavity's initial state is built on the device; the vortex
            uploads its initial fields), K steps in ten calls, each followed
            by the velocity residual read into pinned host memory
            (imexlb_reduce_async, the convergence check of a steady solve),
            the u, v, w, p fields read into pinned host memory at the end,
            destroy.
* roofline  the fused step kernel: 432 algorithmic bytes per cell update
            (27 FP64 loads + 27 FP64 stores) x cells / its mean launch
            duration over the timed region (CUDA events on the launching
            stream around the K launches, times the step kernel's share of
            a step from a second pass with events around each launch, whose
            per-launch durations are reported as isolated_launch_ms),
            against the measured HBM copy bandwidth of MEASURED_PEAKS.json.
* cpu_baseline  the reference's own solver (oracle/_ref) on the host cores,
            rank 0, a bounded sample of full-size steps (subprocess).
* secondary the batched configuration (256 seeded instances, imexlb_b200.batch)
            in FP16 storage and in plain FP64, each timed the same way over
            K steps, with its own roofline and end-to-end figures, and the
            ratio of the two aggregate MLUPS (one GPU only; --no-secondary
            skips it).
--impl reference runs only that CPU measurement (rank 0) and prints its line.
With --gpus N (torchrun, one rank per GPU) every rank advances its own
replica of the workload: the path has no exchange step ("replicas only").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    # BASELINE configuration: lid-driven cavity, plain FP64, 128^3, Re 1000
    "cavity128-f64": dict(case="cavity", bc="standard", storage="f64", arith="fast", n=(128, 128, 128), Re=1000,
                          u0=0.1, R=128.0, lid_u=0.1),
    "cavity128-f64-exact": dict(case="cavity", bc="standard", storage="f64", arith="exact", n=(128, 128, 128),
                                Re=1000, u0=0.1, R=128.0, lid_u=0.1),
    # the reference's own boundary passes (bit-exact drop-in) at Re 100: at Re
    # 1000 they overflow after about 70 steps (the wall sits on the fluid node
    # and the lid speed is forced on the top plane), and a bench would time
    # NaN arithmetic; at Re 100 the flow stays bounded
    "cavity128-f64-refbc": dict(case="cavity", bc="reference", storage="f64", arith="exact", n=(128, 128, 128),
                                Re=100, u0=0.1, R=128.0, lid_u=0.1),
    "tgv64-f64": dict(case="tgv", bc="reference", storage="f64", arith="exact", n=(64, 64, 64), Re=100, u0=0.05,
                      R=0.1, lid_u=0.0),
    "tgv256-f64": dict(case="tgv", bc="reference", storage="f64", arith="fast", n=(256, 256, 256), Re=1600,
                       u0=0.05, R=0.1, lid_u=0.0),
    "cavity128-f16": dict(case="cavity", bc="standard", storage="f16", arith="fast", n=(128, 128, 128), Re=1000,
                          u0=0.1, R=128.0, lid_u=0.1),
    "cavity128-f64-refbc-fast": dict(case="cavity", bc="reference", storage="f64", arith="fast", n=(128, 128, 128),
                                     Re=100, u0=0.1, R=128.0, lid_u=0.1),
    # the same passes resolved per link inside the step kernel (no gather)
    "cavity128-f64-refbc-links": dict(case="cavity", bc="reference-links", storage="f64", arith="exact",
                                      n=(128, 128, 128), Re=100, u0=0.1, R=128.0, lid_u=0.1),
    "cavity128-bf16": dict(case="cavity", bc="standard", storage="bf16", arith="fast", n=(128, 128, 128), Re=1000,
                           u0=0.1, R=128.0, lid_u=0.1),
    "cavity256-f64": dict(case="cavity", bc="standard", storage="f64", arith="fast", n=(256, 256, 256), Re=1000,
                          u0=0.1, R=256.0, lid_u=0.1),
    "cavity256-f16": dict(case="cavity", bc="standard", storage="f16", arith="fast", n=(256, 256, 256), Re=1000,
                          u0=0.1, R=256.0, lid_u=0.1),
    "cavity128-f32": dict(case="cavity", bc="standard", storage="f32", arith="fast", n=(128, 128, 128), Re=1000,
                          u0=0.1, R=128.0, lid_u=0.1),
    "tgv128-f32": dict(case="tgv", bc="standard", storage="f32", arith="fast", n=(128, 128, 128), Re=1600,
                       u0=0.05, R=0.1, lid_u=0.0),
    "tgv128-f16": dict(case="tgv", bc="standard", storage="f16", arith="fast", n=(128, 128, 128), Re=1600,
                       u0=0.05, R=0.1, lid_u=0.0),
    "tgv256-f16": dict(case="tgv", bc="standard", storage="f16", arith="fast", n=(256, 256, 256), Re=1600,
                       u0=0.05, R=0.1, lid_u=0.0),
    # flow past a sphere: 768 x 192 x 192 channel, D = 32 at (192, 96, 96), Re 100
    "sphere768-f16": dict(case="sphere", bc="standard", storage="f16", arith="fast", n=(768, 192, 192), Re=100,
                          u0=0.05, R=32.0, lid_u=0.0, inlet_u=0.05, sphere_d=32.0, sphere_c=(192.0, 96.0, 96.0)),
    "sphere768-bf16": dict(case="sphere", bc="standard", storage="bf16", arith="fast", n=(768, 192, 192), Re=100,
                           u0=0.05, R=32.0, lid_u=0.0, inlet_u=0.05, sphere_d=32.0, sphere_c=(192.0, 96.0, 96.0)),
    "sphere768-f64": dict(case="sphere", bc="standard", storage="f64", arith="fast", n=(768, 192, 192), Re=100,
                          u0=0.05, R=32.0, lid_u=0.0, inlet_u=0.05, sphere_d=32.0, sphere_c=(192.0, 96.0, 96.0)),
    # the served stream's middle sphere channel (L = 384, D = L / 24)
    "sphere384-f16": dict(case="sphere", bc="standard", storage="f16", arith="fast", n=(384, 96, 96), Re=100,
                          u0=0.05, R=16.0, lid_u=0.0, inlet_u=0.05, sphere_d=16.0, sphere_c=(96.0, 48.0, 48.0)),
    # batched solves: 256 seeded TGV / cavity instances (imexlb_b200.batch) in
    # one engine; case/n/R/Re/u0 name the instance the CPU baseline times
    # FP16 storage, FP32 for the instances with tau - 1/2 < 0.015 (imexlb_b200.batch)
    "batched256-f16": dict(kind="batch", storage="f16", arith="fast", count=256, case="cavity", bc="standard",
                           n=(64, 64, 64), Re=400, u0=0.05, R=64.0, lid_u=0.05),
    "batched256-f16-all": dict(kind="batch", storage="f16-all", arith="fast", count=256, case="cavity",
                               bc="standard", n=(64, 64, 64), Re=400, u0=0.05, R=64.0, lid_u=0.05),
    "batched256-bf16": dict(kind="batch", storage="bf16", arith="fast", count=256, case="cavity", bc="standard",
                            n=(64, 64, 64), Re=400, u0=0.05, R=64.0, lid_u=0.05),
    "batched256-f32": dict(kind="batch", storage="f32", arith="fast", count=256, case="cavity", bc="standard",
                           n=(64, 64, 64), Re=400, u0=0.05, R=64.0, lid_u=0.05),
    "batched256-f64": dict(kind="batch", storage="f64", arith="fast", count=256, case="cavity", bc="standard",
                           n=(64, 64, 64), Re=400, u0=0.05, R=64.0, lid_u=0.05),
}
# The 128^3 lid-driven cavity in FP64 with EXACT arithmetic: bit-identical
# to the oracle's specification of the standard boundaries, and as fast as
# FAST arithmetic (0.90 of the copy bandwidth either way over 1000 steps)
DEFAULT_WORKLOAD = "cavity128-f64-exact"

# DRAM bytes (read + write) of one step launch from one ncu capture of the
# workload (the summaries in profiles/ give the commands)
TRAFFIC = {"cavity128-f64": 857.3e6, "cavity128-f64-exact": 855.4e6, "cavity128-f16": 178.5e6}


def tau_of(w) -> float:
    """tau0 = 3 nu: System::tau of the reference (tgv/src/System.cpp:21,
    lid_driven_cavity/src/System.cpp:19)."""
    cs2 = 1.0 / 3.0
    if w["case"] == "tgv":
        return w["u0"] * w["n"][0] / w["Re"] / cs2 / 2 / 3.1415926
    return w["u0"] * w["R"] / w["Re"] / cs2


def dtype_of(w) -> str:
    return {"f64": "f64", "f32": "f32 (fp32 collide)", "f16": "f16 storage / fp32 collide",
            "f16-all": "f16 storage / fp32 collide", "bf16": "bf16 storage / fp32 collide"}[w["storage"]]


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    return dict(hbm_gbs=6650.0, source="fallback")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.25)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"], samples=0)
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(smax) if smax else None,
                    reasons=sorted(reasons), samples=len(sm))


def run_cpu_baseline(w, seconds: float, max_steps: int | None = None) -> dict:
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
    env["OMP_PROC_BIND"] = "false"
    cmd = [sys.executable, "-m", "oracle.cpu_baseline", "--case", w["case"], "--n", *map(str, w["n"]),
           "--R", repr(w["R"]), "--Re", str(w["Re"]), "--u0", repr(w["u0"]), "--seconds", str(seconds)]
    if max_steps:
        cmd += ["--max-steps", str(max_steps)]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    if out.returncode != 0:
        return dict(value=None, unit="MLUPS", cores=None, kind=None, sample="failed: " + out.stderr[-300:])
    res = json.loads(out.stdout.strip().splitlines()[-1])
    return dict(value=res["mlups"], unit="MLUPS", cores=res["cores"], kind=res["kind"], sample=res["sample"],
                seconds=res["seconds"])


def create_upload_bytes(w) -> int:
    """Host-to-device bytes imexlb_create copies for the workload's lattice:
    the vortex's initial u, v, w, p (computed on the host with the
    reference's expressions); the standard sphere's fluid mask and solid-link
    table; the reference sphere's padded fields; nothing for the cavity, whose
    initial state the device builds."""
    nx, ny, nz = w["n"]
    cells = nx * ny * nz
    if w["case"] == "tgv":
        return 4 * 8 * cells
    if w["case"] == "sphere":
        if w["bc"] == "standard":
            return cells * (1 + 4)
        return 4 * 8 * (nx + 6) * (ny + 6) * (nz + 6) + 4 * 8 * cells + cells
    return 0


def config_of(w, name, n_gpus) -> dict:
    nx, ny, nz = w["n"]
    return {"workload": name, "case": w["case"], "boundary": w["bc"], "storage": w["storage"],
            "arith": w["arith"], "lattice": f"{nx}x{ny}x{nz}", "Re": w["Re"], "tau": 0.5 + tau_of(w),
            "lid_u": w["lid_u"], "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU",
            "l2": "inputs larger than L2 (two distribution buffers of "
                  f"{27 * nx * ny * nz * (8 if w['storage'] == 'f64' else 4 if w['storage'] == 'f32' else 2) / 1e6:.0f} MB)"}


def reference_arm(args, w, name, rank, world):
    if rank != 0:
        return 0
    # each reference "step" is one full-size lattice step; the sample is
    # bounded so that the whole run ends within minutes
    cb = run_cpu_baseline(w, seconds=min(60.0, 5.0 + 0.5 * args.steps), max_steps=args.steps)
    line = {"impl": "reference", "metric": "D3Q27 MLUPS", "value": cb["value"], "unit": "MLUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (1e3 * cb["seconds"] / max(1, int(cb["sample"].split()[0]))) if cb["value"] else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic initial and boundary conditions of the case)",
            "config": config_of(w, name, 1),
            "cpu_baseline": {"value": cb["value"], "unit": "MLUPS", "cores": cb["cores"], "kind": cb["kind"],
                             "sample": cb["sample"]},
            "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def replica_throughput(elapsed_ms: float, seconds_e2e: float | None, cells: int, steps: int, dist=None,
                       device: str = "cuda") -> tuple[float, float, float | None, float | None]:
    """Whole-job MLUPS of N independent replicas (one per rank): every rank
    advanced `cells` cells `steps` steps; the job took as long as its slowest
    rank (the max over ranks of the device time, and of the end-to-end host
    time when given).  Returns (value, max_ms, e2e, max_e2e_s)."""
    import torch

    world = dist.get_world_size() if dist is not None else 1
    t = torch.tensor([elapsed_ms, seconds_e2e if seconds_e2e is not None else 0.0], dtype=torch.float64,
                     device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms, max_e2e = float(t[0].item()), float(t[1].item())
    value = world * cells * steps / (max_ms * 1e-3) / 1e6
    e2e = world * cells * steps / max_e2e / 1e6 if seconds_e2e is not None else None
    return value, max_ms, e2e, (max_e2e if seconds_e2e is not None else None)


def measure_batch(storage: str, arith: str, steps: int, warmup: int, tune_cache=None, check_error=False,
                  count: int = 256) -> dict:
    """The batched configuration (imexlb_b200.batch): every instance advances
    together in one engine (persistent launches per kernel group, two steps
    per graph replay).  Device-timed aggregate MLUPS over `steps` steps after
    `warmup`, and end to end from admission to every instance's u, v, w, p
    in pinned host memory."""
    import torch

    from imexlb_b200 import api, batch, tune

    specs = batch.batch_specs(count)
    cells = batch.total_cells(specs)
    plan = batch.storage_plan(specs, storage)
    tiles = batch.tiles_for(specs, storage, cache=tune_cache)
    stream = torch.cuda.Stream()
    budget = batch.budget_for(specs, storage)
    est = batch.engine_storage(storage)
    with torch.cuda.stream(stream):
        eng = api.Engine(storage=est, arith=arith, budget_bytes=budget, max_instances=len(specs),
                         stream=stream.cuda_stream)
        slots = batch.add_all(eng, specs, tiles, storage)
        eng.step(warmup)
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device())
        sampler.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        eng.step(steps)
        ev1.record(stream)
        ev1.synchronize()
        clocks = sampler.stop()
        ms = ev0.elapsed_time(ev1)
        stats = eng.stats()
        fields = [eng.fields(s) for s in slots] if check_error else None
        eng.close()
    value = cells * steps / (ms * 1e-3) / 1e6

    # end to end: admission from the host (the vortices' initial fields
    # uploaded, the cavities' built on the device), the steps, every
    # instance's u, v, w, p read back into pinned host memory (one pinned set
    # per lattice shape, allocated beforehand as a caller would)
    pinned = {}
    for sp in specs:
        shp = (sp.edge,) * 3
        if shp not in pinned:
            pinned[shp] = {k: torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy() for k in "uvwp"}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        eng = api.Engine(storage=est, arith=arith, budget_bytes=budget, max_instances=len(specs),
                         stream=stream.cuda_stream)
        slots = batch.add_all(eng, specs, tiles, storage)
        eng.step(steps)
        for sl, sp in zip(slots, specs):
            eng.fields(sl, out=pinned[(sp.edge,) * 3])
        eng.close()
    e2e_s = time.perf_counter() - t0
    e2e = cells * steps / e2e_s / 1e6
    tgv_cells = sum(sp.cells for sp in specs if sp.case == "tgv")

    errs = None
    if check_error:
        # the timed run took warm-up + timed steps: the FP64 run takes as many
        ref = batch.run(specs, "f64", warmup + steps, fields=True)
        errs = batch.error_report(specs, fields, ref["fields"])

    peaks = load_peaks()
    # algorithmic bytes of one step: 27 loads + 27 stores per cell in each
    # instance's own format
    step_bytes = sum(2 * 27 * api.BYTES_PER_VALUE[st] * sp.cells for sp, st in zip(specs, plan))
    step_ms = ms / steps
    achieved = step_bytes / (step_ms * 1e-3) / 1e9
    groups = len({(st, sp.case, tiles.get(tune.key_of(st, sp.case, (sp.edge,) * 3), 0) == 0)
                  for sp, st in zip(specs, plan)})
    storage_cells = {st: sum(sp.cells for sp, x in zip(specs, plan) if x == st) for st in sorted(set(plan))}
    return {
        "value": value, "unit": "MLUPS", "ms_per_step": step_ms, "steps": steps, "warmup": warmup,
        "instances": len(specs), "cells": cells, "storage": storage, "seed": batch.BATCH_SEED,
        "storage_instances": {st: plan.count(st) for st in sorted(set(plan))}, "storage_cells": storage_cells,
        "roofline": {"bound": "hbm", "kernel": "engine step launches (all kernel groups of one step)",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"],
                     "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)", "traffic": None,
                     "bytes_per_cell_update": step_bytes / cells},
        "e2e": {"value": e2e, "unit": "MLUPS", "h2d_bytes_per_step": 4 * 8 * tgv_cells / steps,
                "d2h_bytes_per_step": 4 * 8 * cells / steps, "seconds": e2e_s},
        "gpu_launches": steps * groups, "clocks": clocks, "engine_tiles": stats["tiles"],
        "per_instance_velocity_l2_vs_fp64": errs,
    }


def bench_batch(args, w, name, cpu) -> int:
    """The batched workload's own bench line."""
    from imexlb_b200 import batch

    r = measure_batch(w["storage"], w["arith"], args.steps, args.warmup, args.tune_cache, args.check_error,
                      w["count"])
    cells, bpv = r["cells"], r["roofline"]["bytes_per_cell_update"] / 54
    line = {
        "metric": "D3Q27 MLUPS (aggregate over the batch)", "value": r["value"], "unit": "MLUPS", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(w),
        "data": "synthetic: 256 seeded instances (analytic initial and boundary conditions)",
        "config": {"workload": name, "instances": r["instances"], "cells": cells, "storage": w["storage"],
                   "storage_instances": r["storage_instances"],
                   "storage_policy": ("FP16 where tau - 1/2 >= 0.015, FP32 below (imexlb_b200.batch)"
                                      if w["storage"] == "f16" else "every instance in the one format"),
                   "mix": "TGV / lid-driven cavity 50/50, edge in {24..128}, Re log-uniform [50, 1000], U0 = 0.05",
                   "seed": batch.BATCH_SEED, "tiles": "autotuned per (edge, case, storage)",
                   "parallelism": "single GPU, one engine",
                   "l2": f"inputs larger than L2 (distribution buffers {2 * 27 * bpv * cells / 1e9:.1f} GB)"},
        "roofline": r["roofline"],
        "e2e": r["e2e"],
        "gpu_launches": r["gpu_launches"],
        "clocks": r["clocks"],
        "cpu_baseline": ({"value": cpu["value"], "unit": "MLUPS", "cores": cpu["cores"], "kind": cpu["kind"],
                          "sample": cpu["sample"] + " (the batch's median-size cavity instance, 64^3)"}
                         if cpu else None),
        "check": {"engine_tiles": r["engine_tiles"],
                  "per_instance_velocity_l2_vs_fp64": r["per_instance_velocity_l2_vs_fp64"]},
    }
    print(json.dumps(line), flush=True)
    return 0


def secondary_batches(args) -> dict:
    """The batched configuration in FP16 storage and in plain FP64 at the
    run's step counts, for the bench line of the default workload: the FP16
    form's aggregate MLUPS against the FP64 form's on the same GPU."""
    out = {}
    for storage in ("f16", "f64"):
        r = measure_batch(storage, "fast", args.steps, max(3, args.warmup), args.tune_cache)
        r.pop("per_instance_velocity_l2_vs_fp64", None)
        out[f"batched256_{storage}"] = r
    out["f16_over_f64"] = out["batched256_f16"]["value"] / out["batched256_f64"]["value"]
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--check-error", action="store_true", help="batched workloads: per-instance error vs FP64")
    ap.add_argument("--tune-cache", default=None, help="batched workloads: autotuner cache (JSON)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="single-lattice workloads: skip the batched FP16 / FP64 measurements (secondary)")
    args = ap.parse_args(argv)
    w = WORKLOADS[args.workload]
    name = args.workload

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, w, name, rank, world)

    # CPU baseline first, in a subprocess, before this process touches CUDA
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(w, args.cpu_seconds)

    if w.get("kind") == "batch":
        # one GPU: ranks other than 0 have no work in this workload
        import torch

        torch.cuda.set_device(local)
        return bench_batch(args, w, name, cpu) if rank == 0 else 0

    import numpy as np
    import torch

    from imexlb_b200 import api

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    nx, ny, nz = w["n"]
    cells = nx * ny * nz
    tau = tau_of(w)
    kw = dict(bc=w["bc"], storage=w["storage"], arith=w["arith"], lid_u=w["lid_u"])
    for key in ("inlet_u", "sphere_d", "sphere_c"):
        if key in w:
            kw[key] = w[key]

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        lbm = api.LBM(w["case"], nx, ny, nz, tau, 1.0, w["u0"], stream=stream.cuda_stream, **kw)
        lbm.step(args.warmup)
        barrier()
        sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
        if sampler:
            sampler.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        ev0.record(stream)
        lbm.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        barrier()
        clocks = sampler.stop() if sampler else None
        elapsed_ms = ev0.elapsed_time(ev1)
        # per-launch kernel times for the roofline, in a pass of their own:
        # events between the launches keep consecutive steps from
        # overlapping their launch with the previous step's end
        prof_steps = min(args.steps, 200)
        lbm.profile(True)
        lbm.step(prof_steps)
        torch.cuda.synchronize()
        kt = lbm.profile_read()
        lbm.profile(False)
        resid = lbm.reduce("umax")
        lbm.close()

    value, max_ms, _, _ = replica_throughput(elapsed_ms, None, cells, args.steps, dist)

    # ---- end to end through the public API, host memory in and out: create
    # the lattice, run the steps in ten calls with the velocity residual of
    # each call read back (the convergence check of a steady solve), read
    # the u, v, w, p fields once at the end, destroy
    checks = 10
    chunk = max(1, args.steps // checks)
    pinned = {k: torch.empty((nz, ny, nx), dtype=torch.float64, pin_memory=True).numpy() for k in "uvwp"}
    res_host = torch.empty(checks + 1, dtype=torch.float64, pin_memory=True).numpy()
    barrier()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        lbm2 = api.LBM(w["case"], nx, ny, nz, tau, 1.0, w["u0"], stream=stream.cuda_stream, **kw)
        done = 0
        nres = 0
        while done < args.steps:
            s = min(chunk, args.steps - done)
            lbm2.step(s)
            done += s
            lbm2.reduce_async("residual", res_host, min(nres, checks))
            nres += 1
        lbm2.fields(out=pinned, wait=False)
        lbm2.synchronize()  # every residual and the fields are in host memory
        lbm2.close()
    e2e_s = time.perf_counter() - t0
    _, _, e2e, e2e_s = replica_throughput(elapsed_ms, e2e_s, cells, args.steps, dist)
    h2d = create_upload_bytes(w) / args.steps
    d2h = (nres * 8 + 4 * 8 * cells) / args.steps

    # the batched configuration in FP16 storage and FP64 beside the headline
    # (one GPU; measured after the headline's timed regions)
    secondary = None
    if rank == 0 and world == 1 and not args.no_secondary:
        secondary = secondary_batches(args)

    if rank == 0:
        peaks = load_peaks()
        bpv = api.BYTES_PER_VALUE[w["storage"]]
        alg_bytes = 2 * 27 * bpv * cells
        # the step kernel's mean launch duration over the timed region: the
        # timed time per step times the step kernel's share of a step (from
        # the profiled pass, where events between the launches also give
        # each launch's duration on its own)
        iso_ms = kt["step_ms"] / max(1, kt["step_launches"])
        share = kt["step_ms"] / max(1e-12, kt["step_ms"] + kt["ghost_ms"])
        step_ms = max_ms / args.steps * share
        achieved = alg_bytes / (step_ms * 1e-3) / 1e9
        dominant = "step_kernel (fused pull/moments/collide)"
        # kernels of ours launched in the timed region: those of a profiled
        # step, times the timed steps
        launches = round((kt["step_launches"] + kt["ghost_launches"]) * args.steps / prof_steps)
        if w["case"] == "sphere" and w["storage"] in ("f16", "bf16"):
            launches += 1  # the drag kernel after the last step (drag_links_kernel)
        line = {
            "metric": "D3Q27 MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(w),
            "data": "synthetic (analytic initial and boundary conditions of the case)",
            "config": config_of(w, name, world),
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)",
                         "traffic": TRAFFIC.get(name), "bytes_per_cell_update": 2 * 27 * bpv,
                         "mean_launch_ms": step_ms, "isolated_launch_ms": iso_ms,
                         "ghost_gather_ms_per_step": kt["ghost_ms"] / max(1, kt["ghost_launches"])
                         if kt["ghost_launches"] else 0.0},
            "e2e": {"value": e2e, "unit": "MLUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "seconds": e2e_s, "residual_reads": nres, "field_reads": 1,
                    "inputs": ("the case parameters: the cavity starts at rest (f = 0) and its initial state "
                               "is built on the device, as the reference's Initialize builds it"
                               if h2d == 0 else "initial fields and masks uploaded at create"),
                    "final_residual": float(res_host[min(nres, checks) - 1]) if nres else None},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": ({"value": cpu["value"], "unit": "MLUPS", "cores": cpu["cores"], "kind": cpu["kind"],
                              "sample": cpu["sample"]} if cpu else None),
            "check": {"max_speed_after_run": resid},
        }
        if secondary is not None:
            line["secondary"] = secondary
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
