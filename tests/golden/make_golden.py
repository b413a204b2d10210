"""Generate the golden fixtures in tests/golden from the reference's own solver.

Run from the repository root after ``make -C oracle ref`` (which compiles the
reference's lbm.cpp / System.cpp / mpi_view_transfer.cpp from the reference
tree against oracle/refshim):

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py
    python tests/golden/make_golden.py --configs [name ...]   # the configuration-size runs

Each fixture records the inputs (the nine input.in numbers, the step count,
the sphere's `ran` field) and the reference's outputs after that many steps:
interior u, v, w, p (x fastest), a SHA-256 of the padded distribution array
f (population fastest, exactly as the reference stores it) and of the solid
mask.  The three input.in files the reference ships are recorded with the
parameters System derives from them, and one Tecplot file written by the
reference's MPIoutput is recorded by digest and header bytes.

``--configs`` adds (under the manifest's "configs" key, leaving the rest as
it is) the reference's results at the benchmark configurations' sizes and
step counts: the 64^3 Taylor-Green vortex at Re 100 after 1000 steps and the
128^3 lid-driven cavity at Re 1000 (the reference's own boundary passes)
after 200 steps.  Those fields are too large to commit, so each is recorded
by the SHA-256 of its FP64 bytes ((nz, ny, nx), x fastest) with a few
summary values; a bit-exact run must reproduce the digests.

The reference tree comes from oracle.refpath.reference_root() (the
IMEXLB_REFERENCE environment variable, else BASELINE.json's reference_path).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.bindings import Reference, run_reference_case  # noqa: E402
from oracle.refpath import reference_root  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, case, rho0, R, Re, u0, nx, ny, nz, steps)
CASES = [
    ("tgv_8x8x8_s10", "tgv", 1.0, 0.1, 100, 0.05, 8, 8, 8, 10),
    ("tgv_10x12x9_s7", "tgv", 1.0, 0.1, 1600, 0.05, 10, 12, 9, 7),
    ("cavity_8x8x8_s20", "cavity", 1.0, 8.0, 100, 0.1, 8, 8, 8, 20),
    ("cavity_9x11x10_s12", "cavity", 1.0, 10.0, 50, 0.1, 9, 11, 10, 12),
    ("sphere_72x12x12_s4", "sphere", 1.0, 2.0, 100, 0.1, 72, 12, 12, 4),
]

# the three input.in files of the reference tree, as (case, nine numbers)
SHIPPED = {
    "tgv": "tgv/input.in",
    "cavity": "lid_driven_cavity/input.in",
    "sphere": "sphere/input.in",
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# configuration-size runs: (name, case, rho0, R, Re, u0, n, steps)
# (the reference's own cavity boundary passes make the 128^3 cavity at Re
# 1000 overflow after about 70 steps: the 50-step entry is before that, the
# 200-step one records the overflowed state)
CONFIGS = [
    ("tgv_64_re100_s1000", "tgv", 1.0, 0.1, 100, 0.05, 64, 1000),
    ("cavity_128_re1000_s50", "cavity", 1.0, 128.0, 1000, 0.1, 128, 50),
    ("cavity_128_re1000_s200", "cavity", 1.0, 128.0, 1000, 0.1, 128, 200),
]


def canonical_nan(a: np.ndarray) -> np.ndarray:
    """FP64 copy with every NaN replaced by one bit pattern (NaN payloads
    differ between processors; which values are NaN does not)."""
    a = np.array(a, dtype=np.float64, copy=True)
    a[np.isnan(a)] = np.float64("nan")
    return np.ascontiguousarray(a)


def field_summary(fields: dict) -> dict:
    """Digests (NaNs canonical) and summary values of the u, v, w, p fields
    ((nz, ny, nx))."""
    out = {f"{k}_sha256": sha(canonical_nan(fields[k])) for k in "uvwp"}
    u, v, w, p = (np.asarray(fields[k], dtype=np.float64) for k in "uvwp")
    finite = bool(all(np.isfinite(a).all() for a in (u, v, w, p)))
    out["finite"] = finite
    out["nonfinite_values"] = {k: int((~np.isfinite(np.asarray(fields[k]))).sum()) for k in "uvwp"}
    if finite:
        out["kinetic"] = float(0.5 * (u * u + v * v + w * w).sum())
        out["mass"] = float((3.0 * p).sum())
        out["umax"] = float(np.sqrt(u * u + v * v + w * w).max())
        out["max_abs"] = {k: float(np.abs(fields[k]).max()) for k in "uvwp"}
    return out


def configs(names=None):
    path = os.path.join(OUT, "manifest.json")
    with open(path) as fh:
        manifest = json.load(fh)
    entries = dict(manifest.get("configs", {}))
    for name, case, rho0, R, Re, u0, n, steps in CONFIGS:
        if names and name not in names:
            continue
        r = run_reference_case(case, rho0, R, Re, u0, n, n, n, steps, warmup=0, want_f=False, fast=True)
        s = r["system"]
        entries[name] = dict(case=case, rho0=rho0, R=R, Re=Re, u0=u0, nx=n, ny=n, nz=n, steps=steps,
                             tau=s["tau"], **field_summary(r))
        print(name, "ok", entries[name].get("kinetic"), entries[name]["nonfinite_values"])
    manifest["configs"] = entries
    if not names or "sphere_mask_shipped" in names:
        manifest["sphere_mask_shipped"] = shipped_sphere_mask()
    with open(path, "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print("wrote", path)


def shipped_sphere_mask() -> dict:
    """The reference's solid mask usr (sphere/src/lbm.cpp:238) for the
    shipped sphere input.in (512 x 128 x 128): SHA-256 of the interior as
    int32 (nz, ny, nx), the solid cell count and the solid box."""
    r = run_reference_case("sphere", 1.0, 8.0, 100, 0.1, 512, 128, 128, 0, want_f=False, fast=True)
    usr = np.ascontiguousarray(r["usr"][3:-3, 3:-3, 3:-3], dtype=np.int32)
    solid = np.argwhere(usr == 0)
    return dict(nx=512, ny=128, nz=128, input=["1.0", "8.0", "100", "0.1", "100", "10", "512", "128", "128"],
                usr_sha256=sha(usr), solid_cells=int((usr == 0).sum()),
                solid_box_zyx=[solid.min(axis=0).tolist(), solid.max(axis=0).tolist()])


def main(refroot: str | None = None):
    refroot = refroot or reference_root()
    if not refroot:
        raise SystemExit("reference tree not found: set IMEXLB_REFERENCE")
    manifest = {}
    for name, case, rho0, R, Re, u0, nx, ny, nz, steps in CASES:
        r = run_reference_case(case, rho0, R, Re, u0, nx, ny, nz, steps, warmup=20)
        s = r["system"]
        arrays = dict(u=r["u"], v=r["v"], w=r["w"], p=r["p"])
        if case == "sphere":
            arrays["ran"] = r["ran"].astype(np.uint8)
        np.savez_compressed(os.path.join(OUT, f"ref_{name}.npz"), **arrays)
        manifest[name] = dict(case=case, rho0=rho0, R=R, Re=Re, u0=u0, nx=nx, ny=ny, nz=nz, steps=steps,
                              tau=s["tau"], f_sha256=sha(r["f"]), usr_sha256=sha(r["usr"]),
                              solid_cells=int((r["usr"][3:-3, 3:-3, 3:-3] == 0).sum()) if case == "sphere" else 0)
        print(name, "ok")

    systems = {}
    for case, rel in SHIPPED.items():
        src = os.path.join(refroot, rel)
        with open(src) as fh:
            nums = fh.read().split()[:9]
        d = tempfile.mkdtemp(prefix="imexlb_sys_")
        with open(os.path.join(d, "input.in"), "w") as fh:
            fh.write(f"{nums[0]} {nums[1]} {nums[2]}\n{nums[3]} {nums[4]} {nums[5]}\n{nums[6]} {nums[7]} {nums[8]}\n")
        systems[case] = dict(input=nums, derived=Reference(case).system(d))
    manifest["shipped_input_in"] = systems

    # Tecplot output of the cavity driver: MPIoutput(0) and every 5 steps
    d = tempfile.mkdtemp(prefix="imexlb_plt_")
    run_reference_case("cavity", 1.0, 8.0, 100, 0.1, 8, 8, 8, 10, out_every=5, want_f=False, workdir=d)
    plt = {}
    for n in (0, 1, 2):
        with open(os.path.join(d, f"output{n}.plt"), "rb") as fh:
            data = fh.read()
        plt[f"output{n}.plt"] = dict(size=len(data), sha256=hashlib.sha256(data).hexdigest(),
                                     header_hex=data[:332].hex())
    manifest["tecplot_cavity_8x8x8"] = dict(rho0=1.0, R=8.0, Re=100, u0=0.1, nx=8, ny=8, nz=8, steps=10,
                                            out_every=5, files=plt)

    with open(os.path.join(OUT, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print("wrote", os.path.join(OUT, "manifest.json"))


if __name__ == "__main__":
    if "--configs" in sys.argv[1:]:
        configs([a for a in sys.argv[1:] if not a.startswith("--")] or None)
    else:
        main(*sys.argv[1:])
