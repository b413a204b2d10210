"""GPU checks of the serving loop: every request's answer is the same when
it is served in the mix (arriving while others run, admitted and retired
around them) as when it runs alone, and its error against the plain FP64
solve is within the FP16-storage bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STREAM = [  # (arrival s, case, n, Re, steps)
    (0.00, "cavity", (32, 32, 32), 400.0, 180),
    (0.00, "tgv", (48, 48, 48), 200.0, 120),
    (0.01, "sphere", (96, 24, 24), 60.0, 150),
    (0.02, "cavity", (48, 48, 48), 150.0, 90),
    (0.03, "tgv", (32, 32, 32), 80.0, 200),
    (0.05, "cavity", (40, 40, 40), 700.0, 60),
]


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from imexlb_b200 import batch, serve

    return serve, batch


def _requests(serve):
    return [serve.Request(i, t, c, n, Re, steps) for i, (t, c, n, Re, steps) in enumerate(STREAM)]


def _alone(serve, req, storage):
    srv = serve.Server(storage=storage, budget_bytes=1 << 30, max_instances=1, chunk=25, answer="fields")
    try:
        assert srv.try_admit(req)
        done = []
        while not done:
            done = srv.advance()
        return done[0][1]
    finally:
        srv.close()


def test_answers_are_the_same_alone_and_in_the_mix(env):
    serve, batch = env
    reqs = _requests(serve)
    # a small active-cell cap makes later requests wait for earlier ones
    res = serve.serve(reqs, "f16", keep_fields=True, budget_bytes=1 << 30, max_active_cells=200_000, chunk=25)
    for r in reqs:
        got = res["results"][r.rid]
        assert got["steps"] == r.max_steps
        alone = _alone(serve, r, "f16")
        for k in "uvwp":
            assert np.array_equal(got["fields"][k], alone[k]), (r.case, r.n, k)
        ref = _alone(serve, r, "f64")
        err = batch.velocity_l2(got["fields"], ref)
        assert err <= 1e-3, (r.case, r.n, err)
    assert res["p99"] >= res["p50"] > 0.0
