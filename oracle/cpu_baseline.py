"""CPU baseline timing -- TEST/MEASUREMENT INFRASTRUCTURE ONLY.

Times the reference's own solver (oracle/_ref, the reference sources compiled
here against the single-rank Kokkos/MPI stand-in, OpenMP on all host cores)
or, if that build is absent, the C restatement (oracle/liboracle.so), on a
bounded number of full-size time steps.  Run as a subprocess so its OpenMP
runtime and thread count are independent of the calling process:

    OMP_NUM_THREADS=N python -m oracle.cpu_baseline --case cavity --n 128 128 128 \
        --Re 1000 --u0 0.1 --R 128 --seconds 20

Prints one JSON object: {"mlups", "steps", "seconds", "cores", "kind", "sample"}.
The initialisation cost is removed by timing two runs of different step
counts and taking the difference.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.bindings import (HERE, Oracle, Reference, oracle_lib, oracle_system,  # noqa: E402
                             reference_available)


def _time_reference(case, rho0, R, Re, u0, n, steps):
    ref = Reference(case, fast=True)
    d = tempfile.mkdtemp(prefix="imexlb_cpu_")
    Reference.write_input(d, rho0, R, Re, u0, steps, 10 ** 9, *n)
    t0 = time.perf_counter()
    ref.run(d, steps, 0, 0, want_f=False)
    return time.perf_counter() - t0


def _time_port(case, rho0, R, Re, u0, n, steps):
    tau = oracle_system(case, rho0, R, Re, u0, steps, 1, n[0])["tau"]
    t0 = time.perf_counter()
    o = Oracle(case, *n, tau, rho0, u0)
    o.initialize()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    return dt


def measure(case, rho0, R, Re, u0, n, seconds, max_steps=None, kind=None):
    kind = kind or ("reference" if reference_available(case) else "port")
    timer = _time_reference if kind == "reference" else _time_port
    base = timer(case, rho0, R, Re, u0, n, 1)  # init + 1 step
    two = timer(case, rho0, R, Re, u0, n, 3)   # init + 3 steps
    per_step = max((two - base) / 2.0, 1e-9)
    steps = max(2, int(seconds / per_step))
    if max_steps:
        steps = min(steps, max_steps)
    t_hi = timer(case, rho0, R, Re, u0, n, steps + 1)
    dt = max(t_hi - base, 1e-9)
    cells = n[0] * n[1] * n[2]
    if kind == "reference":
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    else:
        cores = oracle_lib().oracle_threads()
    return dict(mlups=cells * steps / dt / 1e6, steps=steps, seconds=dt, cores=cores, kind=kind,
                sample=f"{steps} full {n[0]}x{n[1]}x{n[2]} {case} steps of the "
                       f"{'reference solver (oracle/_ref)' if kind == 'reference' else 'C restatement'} "
                       f"on {cores} OpenMP threads, initialisation subtracted")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="cavity")
    ap.add_argument("--n", type=int, nargs=3, default=[128, 128, 128])
    ap.add_argument("--rho0", type=float, default=1.0)
    ap.add_argument("--R", type=float, default=128.0)
    ap.add_argument("--Re", type=int, default=1000)
    ap.add_argument("--u0", type=float, default=0.1)
    ap.add_argument("--seconds", type=float, default=20.0)
    ap.add_argument("--max-steps", type=int, default=None)
    ap.add_argument("--kind", choices=["reference", "port"], default=None)
    a = ap.parse_args(argv)
    res = measure(a.case, a.rho0, a.R, a.Re, a.u0, tuple(a.n), a.seconds, a.max_steps, a.kind)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
