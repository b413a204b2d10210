"""Pin the CPU restatement (oracle/imexlb_oracle.c) to the reference.

Two anchors:
* the golden fixtures in tests/golden, written by tests/golden/make_golden.py
  from the reference's own solver sources (lbm.cpp, System.cpp,
  mpi_view_transfer.cpp of each case) compiled against oracle/refshim;
* when oracle/_ref is present (built here from the reference tree), a live
  comparison on further sizes and step counts.
The bar is bit-exact: the restatement keeps the reference's expression order.
"""
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

from oracle.bindings import Oracle, Reference, oracle_system, reference_available, run_reference_case


def _manifest(golden_dir):
    with open(os.path.join(golden_dir, "manifest.json")) as fh:
        return json.load(fh)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


FIXTURES = ["tgv_8x8x8_s10", "tgv_10x12x9_s7", "cavity_8x8x8_s20", "cavity_9x11x10_s12", "sphere_72x12x12_s4"]


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_reference_fixture(golden_dir, name):
    m = _manifest(golden_dir)[name]
    data = np.load(os.path.join(golden_dir, f"ref_{name}.npz"))
    ran = data["ran"].astype(np.int32) if "ran" in data else None
    o = Oracle(m["case"], m["nx"], m["ny"], m["nz"], m["tau"], m["rho0"], m["u0"], ran)
    o.initialize()
    o.step(m["steps"])
    for name_, got in zip("uvwp", o.moments()):
        want = data[name_]
        assert np.array_equal(got, want), f"{name_}: max |diff| {np.abs(got - want).max()}"
    assert _sha(o.f_padded()) == m["f_sha256"]
    assert _sha(o.usr_padded()) == m["usr_sha256"]


@pytest.mark.parametrize("case", ["tgv", "cavity", "sphere"])
def test_system_derivation_matches_reference(golden_dir, case):
    entry = _manifest(golden_dir)["shipped_input_in"][case]
    nums = entry["input"]
    want = entry["derived"]
    got = oracle_system(case, float(nums[0]), float(nums[1]), int(nums[2]), float(nums[3]), int(nums[4]),
                        int(nums[5]), int(nums[6]))
    assert got["tau"] == want["tau"]
    assert got["miu"] == want["miu"]
    assert got["Ma"] == want["Ma"]
    assert got["Time"] == want["Time"]
    assert got["inter"] == want["inter"]


def test_tecplot_writer_matches_reference(golden_dir, tmp_path):
    t = _manifest(golden_dir)["tecplot_cavity_8x8x8"]
    tau = oracle_system("cavity", t["rho0"], t["R"], t["Re"], t["u0"], t["steps"], t["out_every"], t["nx"])["tau"]
    o = Oracle("cavity", t["nx"], t["ny"], t["nz"], tau, t["rho0"], t["u0"])
    o.initialize()
    for n in range(3):
        if n:
            o.step(t["out_every"])
        path = str(tmp_path / f"output{n}.plt")
        o.write_tecplot(path, n)
        data = open(path, "rb").read()
        want = t["files"][f"output{n}.plt"]
        assert data[:332].hex() == want["header_hex"]
        assert len(data) == want["size"]
        assert hashlib.sha256(data).hexdigest() == want["sha256"]


LIVE = [
    ("tgv", 1.0, 0.1, 400, 0.05, 6, 7, 8, 15),
    ("tgv", 1.0, 0.1, 100, 0.08, 12, 6, 6, 9),
    ("cavity", 1.0, 6.0, 30, 0.1, 7, 6, 9, 25),
    ("cavity", 1.0, 12.0, 1000, 0.1, 12, 12, 12, 6),
    ("sphere", 1.0, 3.0, 60, 0.1, 80, 12, 14, 3),
]


@pytest.mark.skipif(not all(reference_available(c) for c in ("tgv", "cavity", "sphere")),
                    reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("case,rho0,R,Re,u0,nx,ny,nz,steps", LIVE)
def test_oracle_matches_reference_live(case, rho0, R, Re, u0, nx, ny, nz, steps):
    r = run_reference_case(case, rho0, R, Re, u0, nx, ny, nz, steps, warmup=3)
    s = r["system"]
    o = Oracle(case, nx, ny, nz, s["tau"], s["rho0"], s["u0"], r["ran"])
    o.initialize()
    o.step(steps)
    for name_, got in zip("uvwp", o.moments()):
        assert np.array_equal(got, r[name_]), name_
    assert np.array_equal(o.f_padded(), r["f"])
    assert np.array_equal(o.usr_padded(), r["usr"])


def _sha_nan(a):
    """SHA-256 of FP64 bytes with every NaN in one bit pattern (as
    tests/golden/make_golden.py --configs records them)."""
    a = np.array(a, dtype=np.float64, copy=True)
    a[np.isnan(a)] = np.float64("nan")
    return _sha(a)


@pytest.mark.parametrize("name", ["tgv_64_re100_s1000", "cavity_128_re1000_s50", "cavity_128_re1000_s200"])
def test_oracle_reproduces_reference_at_config_size(golden_dir, name):
    """The restatement at the benchmark configurations' sizes and step counts
    reproduces the reference's digests (including the reference cavity's
    overflow after about 70 steps at Re 1000)."""
    m = _manifest(golden_dir)["configs"][name]
    o = Oracle(m["case"], m["nx"], m["ny"], m["nz"], m["tau"], m["rho0"], m["u0"])
    o.initialize()
    o.step(m["steps"])
    for k, got in zip("uvwp", o.moments()):
        assert _sha_nan(got) == m[f"{k}_sha256"], f"{name}: field {k}"
