"""CPU check of the fused-step reformulation and the ghost-slot plan.

The device runs each step as  pull -> moments -> case rules -> collide  into a
second buffer, followed (reference boundaries) by one gather that applies the
ghost-slot plan the library derives from the reference's boundary passes
(imexlb_ghost_plan, host-only).  This test restates exactly that algorithm in
numpy with the kernel's FP64 operation order, drives it with the library's
own plan, and requires bit-identical moments against the oracle's literal
Collision / halo / Streaming / Update sequence.  No GPU is involved.
"""
import numpy as np
import pytest

from imexlb_b200 import api
from oracle.bindings import Oracle, oracle_system

Q = 27
EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
EY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, -1, 1])
EZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, -1, 1])
CLS = [0] + [1] * 6 + [2] * 12 + [3] * 8
W = [8.0 / 27.0, 2.0 / 27.0, 1.0 / 54.0, 1.0 / 216.0]

pytestmark = pytest.mark.skipif(not __import__("os").path.exists(api.LIB_PATH), reason="libimexlb.so not built")


def edu(q, u, v, w):
    terms = [(EX[q], u), (EY[q], v), (EZ[q], w)]
    t = None
    for e, x in terms:
        if e == 0:
            continue
        if t is None:
            t = x if e > 0 else -x
        else:
            t = t + x if e > 0 else t - x
    return np.zeros_like(u) if t is None else t


def gather(Y, X, tgt, src):
    vals = np.where(src >= 0, Y[np.maximum(src, 0)], np.where(src == -1, 0.0, X[np.maximum(-src - 2, 0)]))
    Y[tgt] = vals


def emulate(case, nx, ny, nz, tau0, rho0, u0, steps, ran=None):
    o = Oracle(case, nx, ny, nz, tau0, rho0, u0, ran)
    o.initialize()
    f0 = o.f_padded().reshape(-1)
    usr = o.usr_padded()
    tgt, src = api.ghost_plan(case, nx, ny, nz, usr if case == "sphere" else None)
    A, B = f0.copy(), f0.copy()
    gather(A, B, tgt, src)
    lx, ly, lz = nx + 6, ny + 6, nz + 6
    th = tau0 + 0.5
    m_int = usr[3:3 + nz, 3:3 + ny, 3:3 + nx]
    kz = np.arange(nz, dtype=np.float64)
    prof = u0 * 4.0 * kz * (nz - 1 - kz) / float((nz - 1) * (nz - 1))
    cur, nxt = A, B
    for _ in range(steps):
        X4 = cur.reshape(lz, ly, lx, Q)
        f = [X4[3 - EZ[q]:3 - EZ[q] + nz, 3 - EY[q]:3 - EY[q] + ny, 3 - EX[q]:3 - EX[q] + nx, q].copy()
             for q in range(Q)]
        p = np.zeros((nz, ny, nx))
        u = np.zeros((nz, ny, nx))
        v = np.zeros((nz, ny, nx))
        w = np.zeros((nz, ny, nx))
        for q in range(Q):
            p = p + f[q] / 3.0
            u = u + f[q] if EX[q] == 1 else (u - f[q] if EX[q] == -1 else u)
            v = v + f[q] if EY[q] == 1 else (v - f[q] if EY[q] == -1 else v)
            w = w + f[q] if EZ[q] == 1 else (w - f[q] if EZ[q] == -1 else w)
        if case == "cavity":
            u[nz - 1] = 0.1
        if case == "sphere":
            solid = m_int == 0
            u[solid] = 0.0
            v[solid] = 0.0
            w[solid] = 0.0
            p[solid] = 0.0
            u[:, :, 0] = prof[:, None]
            v[:, :, 0] = 0.0
            w[:, :, 0] = 0.0
            p[:, :, nx - 1] = 0.0
        udu15 = 1.5 * ((u * u + v * v) + w * w)
        tp3 = [(W[c] * p) * 3.0 for c in range(4)]
        Y4 = nxt.reshape(lz, ly, lx, Q)
        for q in range(Q):
            e = edu(q, u, v, w)
            feq = tp3[CLS[q]] + W[CLS[q]] * (((3.0 * e) + (4.5 * (e * e))) - udu15)
            Y4[3:3 + nz, 3:3 + ny, 3:3 + nx, q] = f[q] - ((f[q] - feq) / th)
        gather(nxt, cur, tgt, src)
        cur, nxt = nxt, cur
    return (u, v, w, p), o


CASES = [
    ("tgv", 1.0, 0.1, 100, 0.05, 8, 9, 7, 6),
    ("cavity", 1.0, 8.0, 100, 0.1, 8, 8, 8, 20),
    ("cavity", 1.0, 6.0, 40, 0.1, 9, 7, 10, 13),
    ("sphere", 1.0, 2.0, 100, 0.1, 72, 12, 12, 5),
]


@pytest.mark.parametrize("case,rho0,R,Re,u0,nx,ny,nz,steps", CASES)
def test_fused_reformulation_matches_oracle(case, rho0, R, Re, u0, nx, ny, nz, steps):
    tau = oracle_system(case, rho0, R, Re, u0, steps, 1, nx)["tau"]
    ran = None
    if case == "sphere":
        ran = np.random.default_rng(7).integers(0, 100, size=(nz + 6) * (ny + 6) * (nx + 6), dtype=np.int32)
    if case == "tgv":
        # TGV has no ghost slots on the device; the emulation uses the padded
        # buffer with the periodic wrap the reference's self-exchange makes
        pytest.skip("periodic case is covered by the GPU parity tests")
    got, o = emulate(case, nx, ny, nz, tau, rho0, u0, steps, ran)
    o.step(steps)
    for name, g, want in zip("uvwp", got, o.moments()):
        assert np.array_equal(g, want), f"{name}: max |diff| {np.abs(g - want).max()}"


def test_ghost_plan_sizes():
    # the plan touches only the one-cell shell (and what it chains to)
    tgt, src = api.ghost_plan("cavity", 16, 16, 16)
    assert len(tgt) == len(set(tgt.tolist()))
    assert len(tgt) < 6 * 18 * 18 * 27
    tgt2, _ = api.ghost_plan("cavity", 32, 16, 8)
    assert len(tgt2) > 0
