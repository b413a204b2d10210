"""Error of the reduced storage formats against FP64, as the step count grows.

Each case (a lid-driven cavity, sphere channel or Taylor-Green vortex of the
batched and served mixes, U0 = u_w = inlet speed = 0.05, standard
boundaries, FAST arithmetic) runs alone once in FP64 and once in every
listed storage format, and the relative velocity L2 error against the FP64
run, sqrt(sum |u - u64|^2 / sum |u64|^2) over the lattice, is taken at each
checkpoint.  This is the evidence behind the storage plans of the batched
and served FP16 forms (imexlb_b200.batch.storage_plan,
imexlb_b200.serve.storage_for).

    python -m imexlb_b200.accuracy --out accuracy.jsonl
    python -m imexlb_b200.accuracy --cases cavity:80:186.4,tgv:64:300 --storages f16,f32
"""
from __future__ import annotations

import argparse
import json
import time

from . import api
from .batch import velocity_l2

U = 0.05
PI_REF = 3.1415926

# (case, edge, Re, storages): cavities and spheres in the 2-byte formats
# (stochastic rounding), vortices in FP32 across tau - 1/2
DEFAULT_CASES = [
    ("cavity", 80, 186.4, "f16,bf16,f32"), ("cavity", 128, 150.3, "f16,bf16"), ("cavity", 64, 117.2, "f16"),
    ("cavity", 48, 600.0, "f16,f32"), ("cavity", 32, 300.0, "f16"), ("cavity", 128, 1000.0, "f16,f32"),
    ("cavity", 96, 400.0, "f16"), ("sphere", 256, 100.0, "f16,bf16"), ("sphere", 384, 200.0, "f16"),
    ("sphere", 512, 20.0, "f16"), ("tgv", 32, 100.0, "f32,f16"), ("tgv", 32, 400.0, "f32"),
    ("tgv", 64, 300.0, "f32"), ("tgv", 64, 800.0, "f32"), ("tgv", 96, 800.0, "f32"), ("tgv", 128, 800.0, "f32"),
    ("tgv", 128, 50.0, "f32,f16"), ("tgv", 48, 779.2, "f32"),
]


def tau0_of(case: str, n: int, Re: float) -> float:
    """tau - 1/2 = 3 nu, with the length scale of the served mix: n / 2 pi
    (vortex), the edge (cavity), the sphere's diameter n / 24 (channel)."""
    if case == "tgv":
        return 3.0 * U * (n / 2.0 / PI_REF) / Re
    if case == "sphere":
        return 3.0 * U * (n / 24.0) / Re
    return 3.0 * U * n / Re


def lattice(case: str, n: int, Re: float, storage: str) -> api.LBM:
    t = tau0_of(case, n, Re)
    if case == "cavity":
        return api.LBM("cavity", n, n, n, t, 1.0, U, bc="standard", storage=storage, arith="fast", lid_u=U)
    if case == "tgv":
        return api.LBM("tgv", n, n, n, t, 1.0, U, bc="standard", storage=storage, arith="fast")
    return api.LBM("sphere", n, n // 4, n // 4, t, 1.0, U, bc="standard", storage=storage, arith="fast",
                   inlet_u=U, sphere_d=n / 24.0, sphere_c=(n / 4.0, n / 8.0, n / 8.0))


def velocities(case: str, n: int, Re: float, storage: str, checkpoints, rounding: str | None = None) -> list[dict]:
    out = []
    with lattice(case, n, Re, storage) as lbm:
        if rounding is not None:
            lbm.set_rounding(rounding)
        done = 0
        for c in checkpoints:
            lbm.step(c - done)
            done = c
            f = lbm.fields()
            out.append({k: f[k] for k in "uvw"})
    return out


def study(cases, checkpoints, nearest_too: bool = False) -> list[dict]:
    """`nearest_too`: also run the cavity's and sphere's 2-byte formats with
    round-to-nearest stores (imexlb_set_rounding), beside their default
    stochastic rounding."""
    lines = []
    for case, n, Re, storages in cases:
        t0 = time.perf_counter()
        ref = velocities(case, n, Re, "f64", checkpoints)
        runs = []
        for st in storages.split(","):
            two_byte_sr = st in ("f16", "bf16") and case != "tgv"
            runs.append((st, "stochastic" if two_byte_sr else "nearest", None))
            if two_byte_sr and nearest_too:
                runs.append((st, "nearest", "nearest"))
        for st, label, rounding in runs:
            got = velocities(case, n, Re, st, checkpoints, rounding)
            line = dict(case=case, n=n, Re=Re, tau0=tau0_of(case, n, Re), storage=st, rounding=label,
                        steps=list(checkpoints), velocity_l2_vs_f64=[velocity_l2(a, b) for a, b in zip(got, ref)])
            lines.append(line)
            print(json.dumps(line), flush=True)
        print(json.dumps({"case_seconds": round(time.perf_counter() - t0, 1)}), flush=True)
    return lines


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--cases", default=None,
                    help="case:edge:Re[,...] (default: the built-in list); storages from --storages")
    ap.add_argument("--storages", default="f16,f32")
    ap.add_argument("--checkpoints", default="2000,5000,10000,20000")
    ap.add_argument("--nearest-too", action="store_true",
                    help="also run the cavity's and sphere's 2-byte formats with round-to-nearest stores")
    ap.add_argument("--out", default=None, help="also write the JSON lines to this file")
    args = ap.parse_args(argv)
    if args.cases:
        cases = []
        for item in args.cases.split(","):
            c, n, Re = item.split(":")
            cases.append((c, int(n), float(Re), args.storages))
    else:
        cases = DEFAULT_CASES
    checkpoints = [int(x) for x in args.checkpoints.split(",")]
    lines = study(cases, checkpoints, args.nearest_too)
    if args.out:
        with open(args.out, "w") as fh:
            for line in lines:
                fh.write(json.dumps(line) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
