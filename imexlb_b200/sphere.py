"""Flow past a sphere: drag coefficient and the error of reduced storage.

The mixed-precision configuration: a channel of 768 x 192 x 192 cells with a
voxelised sphere of diameter 32 centred at (192, 96, 96), an equilibrium
velocity inlet u = (0.05, 0, 0), a zero-gradient outlet, periodic lateral
sides, Re = 100 (nu = 0.05 * 32 / 100).  The momentum-exchange force is summed
in FP64 every `--every` steps; the drag coefficient is

    Cd = F_x / (1/2 rho U^2 pi D^2 / 4).

Each storage format runs the same steps; the report gives the last Cd, its
mean over the last tenth of the samples, and the relative velocity L2 error
of the reduced formats against the FP64 run at the end.

    python -m imexlb_b200.sphere --steps 30000 --storages f64,f16,bf16
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import api
from .batch import velocity_l2


def run(storage: str, n=(768, 192, 192), D: float = 32.0, centre=(192.0, 96.0, 96.0), U: float = 0.05,
        Re: float = 100.0, steps: int = 30000, every: int = 100) -> dict:
    tau0 = 3.0 * U * D / Re
    area = math.pi * D * D / 4.0
    t0 = time.perf_counter()
    cds = []
    with api.LBM("sphere", *n, tau0, 1.0, U, bc="standard", storage=storage, arith="fast", inlet_u=U,
                 sphere_d=D, sphere_c=centre) as lbm:
        done = 0
        while done < steps:
            k = min(every, steps - done)
            lbm.step(k)
            done += k
            fx = lbm.reduce("drag")[0]
            cds.append(fx / (0.5 * 1.0 * U * U * area))
        fields = lbm.fields()
    tail = cds[-max(1, len(cds) // 10):]
    return dict(storage=storage, steps=steps, cd_last=cds[-1], cd_tail_mean=float(np.mean(tail)),
                cd_tail_std=float(np.std(tail)), seconds=time.perf_counter() - t0, fields=fields,
                cd_every=every, cd_series=[round(c, 6) for c in cds])


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--steps", type=int, default=30000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--storages", default="f64,f16,bf16")
    ap.add_argument("--out", default=None, help="also write the JSON lines (with the Cd series) to this file")
    args = ap.parse_args(argv)
    results = {}
    for st in args.storages.split(","):
        results[st] = run(st, steps=args.steps, every=args.every)
    ref = results.get("f64")
    lines = []
    for st, r in results.items():
        line = {k: v for k, v in r.items() if k != "fields"}
        line.update(lattice=[768, 192, 192], sphere_d=32.0, sphere_c=[192.0, 96.0, 96.0], inlet_u=0.05, Re=100.0)
        if ref is not None and st != "f64":
            line["velocity_l2_vs_f64"] = velocity_l2(r["fields"], ref["fields"])
            line["cd_rel_err_vs_f64"] = abs(r["cd_tail_mean"] - ref["cd_tail_mean"]) / abs(ref["cd_tail_mean"])
        print(json.dumps({k: v for k, v in line.items() if k != "cd_series"}), flush=True)
        lines.append(line)
    if args.out:
        with open(args.out, "w") as fh:
            for line in lines:
                fh.write(json.dumps(line) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
