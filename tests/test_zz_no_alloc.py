"""imexlb_reduce_fields_noalloc: the reduction for callers that may not
allocate device memory (its partial sums live in a fixed array inside the
library).  Its results must agree with imexlb_reduce, which uses memory the
lattice allocated, on two calls in a row, and sizes beyond its fixed capacity
must be refused.  The test allocates the caller's inputs and outputs itself;
the entry point allocates nothing.  Collected last (file name) so that a run
stopping at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# 1e-12 relative, as the FP64 parity tests, taken against the sum of the
# terms' magnitudes: the two reductions add the same terms in different orders,
# and a sum that cancels (the cavity's total mass is ~1e-14) has no meaningful
# relative error of its own.
TOL = 1e-12
KINDS = {"mass": 0, "kinetic": 1, "umax": 4}
MAX_CELLS = 268435456


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import api

    return torch, api


def _noalloc(api, torch, kind, fields, n, out, stream):
    lib = api.load_library()
    rc = lib.imexlb_reduce_fields_noalloc(KINDS[kind], *[ctypes.c_void_p(t.data_ptr()) for t in fields],
                                          ctypes.c_int64(n), ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(stream))
    return rc


@pytest.mark.parametrize("case,n,kw", [("cavity", (40, 36, 44), dict(bc="standard", lid_u=0.1)),
                                       ("tgv", (48, 48, 48), {})])
def test_noalloc_matches_allocating_reduction(env, case, n, kw):
    torch, api = env
    nx, ny, nz = n
    with api.LBM(case, nx, ny, nz, 0.03, 1.0, 0.1 if case == "cavity" else 0.05, **kw) as lbm:
        lbm.step(60)
        host = lbm.fields()
        want = {k: lbm.reduce(k) for k in KINDS}
    speed = np.sqrt(host["u"] ** 2 + host["v"] ** 2 + host["w"] ** 2)
    scale = {"mass": float(np.abs(3.0 * host["p"]).sum()), "kinetic": float((0.5 * speed ** 2).sum()),
             "umax": float(speed.max())}
    fields = [torch.from_numpy(np.ascontiguousarray(host[k]).ravel()).cuda() for k in "uvwp"]
    stream = torch.cuda.current_stream().cuda_stream
    for kind in KINDS:
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):  # two calls in a row share the fixed scratch
            out.fill_(float("nan"))
            rc = _noalloc(api, torch, kind, fields, nx * ny * nz, out, stream)
            assert rc == 0, api.load_library().imexlb_last_error().decode()
            torch.cuda.synchronize()
            got = out.item()
            assert abs(got - want[kind]) <= TOL * scale[kind], (kind, call, got, want[kind], scale[kind])


def test_noalloc_refuses_sizes_beyond_capacity(env):
    torch, api = env
    fields = [torch.zeros(8, dtype=torch.float64, device="cuda") for _ in range(4)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _noalloc(api, torch, "mass", fields, MAX_CELLS + 1, out, torch.cuda.current_stream().cuda_stream)
    assert rc == 1  # IMEXLB_E_ARG, before any work is queued
    assert b"capacity" in api.load_library().imexlb_last_error()


@pytest.mark.parametrize("n", [20_000_003, MAX_CELLS])
def test_noalloc_mass_many_partials(env, n):
    """More partial sums than the final pass has threads (n / 65536 > 256),
    a last chunk shorter than the others, and the capacity itself (accepted):
    the sum of 3p matches torch's FP64 sum under the same relative bound."""
    torch, api = env
    g = torch.Generator(device="cuda").manual_seed(5)
    p = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.25
    want = float((3.0 * p).sum().item())
    scale = float((3.0 * p).abs().sum().item())
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out.fill_(float("nan"))
        rc = _noalloc(api, torch, "mass", [p, p, p, p], n, out, stream)
        assert rc == 0, api.load_library().imexlb_last_error().decode()
        torch.cuda.synchronize()
        assert abs(out.item() - want) <= TOL * scale, (n, call, out.item(), want)
    del p
    torch.cuda.empty_cache()


def test_noalloc_umax_reports_nan(env):
    """A NaN in a field shows as a NaN maximum (the asynchronous call cannot
    return an error code for it, as imexlb_reduce does)."""
    torch, api = env
    n = 100_000
    u = torch.linspace(0.0, 0.1, n, dtype=torch.float64, device="cuda")
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _noalloc(api, torch, "umax", [u, z, z, z], n, out, stream) == 0
    torch.cuda.synchronize()
    assert out.item() == pytest.approx(0.1, rel=1e-15)
    u[77_777] = float("nan")
    assert _noalloc(api, torch, "umax", [u, z, z, z], n, out, stream) == 0
    torch.cuda.synchronize()
    assert np.isnan(out.item())
