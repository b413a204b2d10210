"""High-resolution FP64 oracle of the Taylor-Green vortex's kinetic energy -- TEST INFRASTRUCTURE.

    python tests/golden/tgv_spectral.py [--n 64] [--re 100] [--steps 1000] [--lattice 64]

Solves the incompressible Navier-Stokes equations on the periodic box
[0, 2 pi)^3 by the Fourier pseudo-spectral method (rotational form u x omega,
2/3-rule dealiasing, classical RK4 with the viscous term integrated exactly
through the factor exp(-nu k^2 t)), from the vortex the benchmark starts
from:

    u = sin x cos y cos z,  v = -cos x sin y cos z,  w = 0,  nu = 1 / Re

(velocity scale U0 = 1, length scale 1).  A lattice of N cells per side run
at lattice velocity U0_lat maps lattice step s to the time t = s U0_lat 2 pi / N.
Writes the kinetic-energy ratio E(t)/E(0) at every 100 lattice steps of the
64^3, U0 = 0.05 lattice to tests/golden/tgv_spectral_re100.json, with the
viscous-only decay exp(-6 t / Re) beside it for comparison.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))


def solve(n: int, re: float, t_out: list[float], dt: float) -> list[float]:
    nu = 1.0 / re
    x = np.arange(n) * (2.0 * np.pi / n)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = np.stack([np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z), np.zeros_like(X)])
    k1 = np.fft.fftfreq(n, 1.0 / n)
    kz1 = np.fft.rfftfreq(n, 1.0 / n)
    KX, KY, KZ = np.meshgrid(k1, k1, kz1, indexing="ij")
    K = np.stack([KX, KY, KZ])
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    K2inv = np.where(K2 == 0, 0.0, 1.0 / np.where(K2 == 0, 1.0, K2))
    kmax = n // 2
    dealias = ((np.abs(KX) < 2.0 / 3.0 * kmax) & (np.abs(KY) < 2.0 / 3.0 * kmax) &
               (np.abs(KZ) < 2.0 / 3.0 * kmax)).astype(np.float64)

    def fwd(a):
        return np.fft.rfftn(a, axes=(1, 2, 3))

    def inv(a):
        return np.fft.irfftn(a, s=(n, n, n), axes=(1, 2, 3))

    def rhs(uh):
        # -(u . grad) u = u x omega - grad(|u|^2 / 2); the gradient is removed by the projection
        w = inv(1j * np.stack([K[1] * uh[2] - K[2] * uh[1], K[2] * uh[0] - K[0] * uh[2],
                               K[0] * uh[1] - K[1] * uh[0]]))
        uu = inv(uh)
        nl = np.stack([uu[1] * w[2] - uu[2] * w[1], uu[2] * w[0] - uu[0] * w[2], uu[0] * w[1] - uu[1] * w[0]])
        nh = fwd(nl) * dealias
        kdotn = (K * nh).sum(axis=0)
        return nh - K * (kdotn * K2inv)

    def energy(uh):
        uu = inv(uh)
        return 0.5 * float((uu ** 2).sum(axis=0).mean())

    uh = fwd(u)
    e0 = energy(uh)
    out = []
    t = 0.0
    for target in t_out:
        while t < target - 1e-12:
            h = min(dt, target - t)
            ef = np.exp(-nu * K2 * h)
            eh = np.exp(-nu * K2 * h / 2)
            a1 = rhs(uh)
            a2 = rhs(eh * (uh + 0.5 * h * a1))
            a3 = rhs(eh * uh + 0.5 * h * a2)
            a4 = rhs(ef * uh + h * eh * a3)
            uh = ef * uh + (h / 6.0) * (ef * a1 + 2.0 * eh * (a2 + a3) + a4)
            t += h
        out.append(energy(uh) / e0)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64, help="spectral grid points per side")
    ap.add_argument("--re", type=float, default=100.0)
    ap.add_argument("--steps", type=int, default=1000, help="lattice steps covered")
    ap.add_argument("--every", type=int, default=100, help="lattice steps between samples")
    ap.add_argument("--lattice", type=int, default=64, help="lattice cells per side")
    ap.add_argument("--u0", type=float, default=0.05, help="lattice velocity")
    ap.add_argument("--dt", type=float, default=0.005)
    args = ap.parse_args()
    steps = list(range(0, args.steps + 1, args.every))
    t_out = [s * args.u0 * 2.0 * np.pi / args.lattice for s in steps]
    ratio = solve(args.n, args.re, t_out, args.dt)
    rec = dict(method="Fourier pseudo-spectral, 2/3 dealiasing, RK4 with exact viscous factor",
               grid=args.n, Re=args.re, dt=args.dt, lattice=args.lattice, u0_lattice=args.u0,
               lattice_steps=steps, t=t_out, kinetic_ratio=ratio,
               viscous_only=[float(np.exp(-6.0 * t / args.re)) for t in t_out])
    path = os.path.join(OUT, f"tgv_spectral_re{int(args.re)}.json")
    with open(path, "w") as fh:
        json.dump(rec, fh, indent=1)
    print(path)
    for s, t, r, v in zip(steps, t_out, ratio, rec["viscous_only"]):
        print(f"{s:6d} t={t:.4f} E/E0={r:.6f} viscous-only={v:.6f}")


if __name__ == "__main__":
    main()
