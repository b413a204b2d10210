"""GPU parity at the benchmark configurations' own sizes and step counts.

* 64^3 Taylor-Green vortex, Re 100, 1000 steps, and the 128^3 lid-driven
  cavity with the reference's own boundary passes, Re 1000, 50 steps: FP64
  EXACT reproduces the digests of the reference's own solver
  (tests/golden/manifest.json "configs", written by
  tests/golden/make_golden.py --configs) bit for bit; FP64 FAST stays
  within 1e-12 of it (max |diff| / max |field| per field).
* The same cavity after 200 steps: the reference's boundary passes make it
  overflow after about 70 steps (BGK at tau = 0.5384 with the lid forced on
  the top fluid plane); EXACT reproduces that state too, every finite value
  bit for bit and NaN exactly where the reference has NaN (NaN payloads
  differ between processors, so both sides are compared with one NaN
  pattern).  The same two digests hold with the boundary passes resolved
  per link inside the step kernel (bc "reference-links").
* The 128^3 standard cavity (the default benchmark workload, FAST
  arithmetic) after 20000 steps, the configuration's step count, stays within
  1e-12 of the EXACT run of the same lattice.
* Kinetic energy of the 64^3 vortex at Re 100 against the FP64
  pseudo-spectral Navier-Stokes solution (tests/golden/tgv_spectral.py) at
  every 100 steps up to 1000: E(t)/E(0) within 1 % of it, and the decay after
  the first 100 steps, E(t)/E(100), within 0.2 %.  (The lattice starts from
  f = feq with no non-equilibrium part and loses about 0.5 % of its energy to
  that initial layer in the first steps; afterwards its decay follows the
  spectral solution, whose energy falls to 0.60 of the initial by step 1000
  against 0.74 for viscous decay alone.)
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FAST = 1e-12  # FP64 FAST against EXACT: max |diff| / max |field|
TOL_KE = 1e-2     # E(t)/E(0) against the spectral solution, relative
TOL_KE_DECAY = 2e-3  # E(t)/E(100) against the spectral solution, relative


@pytest.fixture(scope="module")
def api():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import api as a

    return a


@pytest.fixture(scope="module")
def configs(golden_dir):
    with open(os.path.join(golden_dir, "manifest.json")) as fh:
        return json.load(fh)["configs"]


def _sha(a):
    """SHA-256 of the FP64 bytes with every NaN in one bit pattern (as
    tests/golden/make_golden.py records them)."""
    a = np.array(a, dtype=np.float64, copy=True)
    a[np.isnan(a)] = np.float64("nan")
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _rel(got, want):
    return float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-300))


_EXACT = {}


def _run(api, m, arith):
    key = (m["case"], m["nx"], m["steps"], arith)
    if key not in _EXACT:
        with api.LBM(m["case"], m["nx"], m["ny"], m["nz"], m["tau"], m["rho0"], m["u0"], arith=arith) as lbm:
            lbm.step(m["steps"])
            _EXACT[key] = lbm.fields()
    return _EXACT[key]


@pytest.mark.parametrize("name", ["tgv_64_re100_s1000", "cavity_128_re1000_s50", "cavity_128_re1000_s200"])
def test_exact_reproduces_reference_at_config(api, configs, name):
    m = configs[name]
    got = _run(api, m, "exact")
    for k in "uvwp":
        assert _sha(got[k]) == m[f"{k}_sha256"], f"{name}: field {k} differs from the reference's"


@pytest.mark.parametrize("name", ["cavity_128_re1000_s50", "cavity_128_re1000_s200"])
def test_per_link_boundaries_reproduce_reference_at_config(api, configs, name):
    """The reference's boundary passes resolved per link inside the step
    (bc "reference-links") give the same digests as the reference."""
    m = configs[name]
    with api.LBM(m["case"], m["nx"], m["ny"], m["nz"], m["tau"], m["rho0"], m["u0"], bc="reference-links") as lbm:
        lbm.step(m["steps"])
        got = lbm.fields()
    for k in "uvwp":
        assert _sha(got[k]) == m[f"{k}_sha256"], f"{name}: field {k} differs from the reference's"


@pytest.mark.parametrize("name", ["tgv_64_re100_s1000", "cavity_128_re1000_s50"])
def test_fast_within_1e12_at_config(api, configs, name):
    m = configs[name]
    exact = _run(api, m, "exact")
    fast = _run(api, m, "fast")
    for k in "uvwp":
        assert _rel(fast[k], exact[k]) <= TOL_FAST, f"{name} {k}: {_rel(fast[k], exact[k])}"


def test_standard_cavity_fast_within_1e12_after_20000_steps(api):
    n, steps = 128, 20000
    tau = 0.1 * 128.0 / 1000 * 3.0  # 3 nu, nu = u_w R / Re
    out = {}
    for arith in ("exact", "fast"):
        with api.LBM("cavity", n, n, n, tau, 1.0, 0.1, bc="standard", lid_u=0.1, arith=arith) as lbm:
            lbm.step(steps)
            out[arith] = lbm.fields()
    for k in "uvwp":
        assert _rel(out["fast"][k], out["exact"][k]) <= TOL_FAST, f"{k}: {_rel(out['fast'][k], out['exact'][k])}"


def test_tgv_kinetic_energy_follows_spectral_solution(api, configs, golden_dir):
    with open(os.path.join(golden_dir, "tgv_spectral_re100.json")) as fh:
        spec = json.load(fh)
    m = configs["tgv_64_re100_s1000"]
    ratios = []
    with api.LBM("tgv", 64, 64, 64, m["tau"], m["rho0"], m["u0"], arith="fast") as lbm:
        e0 = lbm.reduce("kinetic")
        done = 0
        for s in spec["lattice_steps"]:
            lbm.step(s - done)
            done = s
            ratios.append(lbm.reduce("kinetic") / e0)
    want_all = spec["kinetic_ratio"]
    i100 = spec["lattice_steps"].index(100)
    for s, got, want in zip(spec["lattice_steps"], ratios, want_all):
        assert abs(got - want) <= TOL_KE * want, (s, got, want)
        if s >= 100:
            decay, want_decay = got / ratios[i100], want / want_all[i100]
            assert abs(decay - want_decay) <= TOL_KE_DECAY * want_decay, (s, decay, want_decay)
