"""The shared-memory staged kernels' copy plan, checked on the CPU.

The library lists the bulk copies of every tile with the same tile_runs
code the kernels run (imexlb_debug_stage_plan, host build of
stage_core.cuh).  For every lattice shape the tests, the benches, the
batched configuration and the served stream use, each copy must start on a
16-byte boundary, move a multiple of 16 bytes, stay inside its source plane
and its stage slot, and the slot rows must hold exactly the rows the pull
reads: the periodic image on a wrapping axis, the cell's own opposite
population beyond a cavity wall (halfway bounce-back).  A cavity tile also
copies the wall records of its rows (64 bytes a row) into a 1 KB area.
The sphere channel's flat tiles (a run of C elements of a plane across row
ends) must stage, in every slot element, the plane element its pull reads:
the run shifted by -e_y rows, 8 guard elements a side, wrapped around the
periodic y and z.
"""
import ctypes

import numpy as np
import pytest

from imexlb_b200 import api

# D3Q27 in the reference's ordering (tgv/src/lbm.cpp:27-190)
EX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1]
EY = [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, -1, 1]
EZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, -1, 1]
BB = [0] + [q + 1 if q % 2 else q - 1 for q in range(1, 27)]
ELEM = 2  # bytes per stored value (FP16 / BF16)
MAX_TX = (1 << 20) - 1  # an mbarrier's transaction count
REC_BYTES, REC_AREA = 64, 1024  # wall record of a row; record area of a stage


MODES = {"cavity": 0, "tgv": 1, "sphere": 2}
GUARD = 8  # guard elements a side of a flat tile's slot


def plan(nx, ny, nz, mode):
    lib = api.load_library()
    fn = lib.imexlb_debug_stage_plan
    fn.restype = ctypes.c_int64
    fn.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    geo = np.zeros(10, np.int32)
    n = fn(nx, ny, nz, mode, geo.ctypes.data, None, 0)
    if n < 0:
        return None, None
    runs = np.zeros((n, 6), np.int32)
    assert fn(nx, ny, nz, mode, geo.ctypes.data, runs.ctypes.data, n) == n
    keys = ("P", "R", "cap", "nty", "sq", "sz", "pitch", "base", "flat", "C")
    return dict(zip(keys, geo.tolist())), runs


def check_flat(g, runs, nx, ny, nz):
    """A flat tile's slots hold, element by element, the plane elements the
    tile's pulls read (with guards), wrapped around the periodic y and z."""
    P, cap, C = g["P"], g["cap"], g["C"]
    NP = ny * P
    assert g["sz"] == NP and C + 2 * GUARD <= cap and C % 16 == 0
    t, q, pop, src, dst, nbytes = (runs[:, i].astype(np.int64) for i in range(6))
    assert np.all(nbytes > 0) and np.all(nbytes % 16 == 0)
    assert np.all((src * ELEM) % 16 == 0) and np.all((dst * ELEM) % 16 == 0)
    assert np.all(pop == q)
    rel = src - g["base"]
    plane, off = rel // g["sz"], rel % g["sz"]
    nel = nbytes // ELEM
    assert np.all(rel >= 0) and np.all(plane < nz) and np.all(off + nel <= NP), "copy leaves its plane"
    slot0 = dst - q * cap
    assert np.all(slot0 >= 0) and np.all(slot0 + nel <= cap)
    per_tile = np.bincount(t, weights=nbytes, minlength=g["nty"] * nz)
    assert per_tile.max() <= MAX_TX
    # every slot element once, with the plane element its pull reads: on the
    # planes where z wraps and one inside plane (the others repeat it)
    nty = g["nty"]
    for k in sorted({0, 1, nz // 2, nz - 1}):
        sel = (t // nty) == k
        width = C + 2 * GUARD
        have = np.full((nty, 27, width), -1, np.int64)  # (plane, element) as plane * NP + element
        count = np.zeros((nty, 27, width), np.int64)
        for i in np.nonzero(sel)[0]:
            tt, qq, s0, n = int(t[i]) % nty, int(q[i]), int(slot0[i]), int(nel[i])
            have[tt, qq, s0:s0 + n] = plane[i] * NP + off[i] + np.arange(n)
            count[tt, qq, s0:s0 + n] += 1
        e0 = np.arange(nty) * C
        n_tile = np.minimum(C, NP - e0)
        o = np.arange(width)
        for qq in range(27):
            want = ((k - EZ[qq]) % nz) * NP + (e0[:, None] - EY[qq] * P - GUARD + o[None, :]) % NP
            used = o[None, :] < (n_tile[:, None] + 2 * GUARD)
            assert np.all(count[:, qq][used] == 1), (k, qq, "slot element not written exactly once")
            assert np.all(have[:, qq][used] == want[used]), (k, qq)
            assert np.all(count[:, qq][~used] == 0), (k, qq, "elements copied beyond the tile")


def shapes():
    out = set()
    # single-lattice benches and tests
    for e in (12, 16, 32, 64, 128, 256):
        out.add(("tgv", (e, e, e)))
    for e in (12, 16, 32, 64, 128, 256):
        out.add(("cavity", (e, e, e)))
    out |= {("cavity", (96, 32, 32)), ("tgv", (96, 32, 32)), ("cavity", (32, 16, 8)), ("tgv", (34, 18, 10)),
            ("cavity", (34, 18, 10)), ("cavity", (1000, 3, 3)), ("tgv", (2, 2, 2)), ("cavity", (4, 5, 3))}
    # batched configuration and served stream
    for e in (24, 32, 48, 64, 80, 96, 112, 128):
        out.add(("tgv", (e, e, e)))
        out.add(("cavity", (e, e, e)))
    for L in (256, 384, 512, 768):
        out.add(("sphere", (L, L // 4, L // 4)))
    # sphere channels of the GPU tests
    for n in ((64, 16, 16), (64, 16, 18), (96, 24, 24), (96, 32, 32), (288, 24, 24), (48, 16, 16),
              (40, 12, 14), (96, 20, 20), (72, 12, 12), (144, 36, 36), (192, 48, 48)):
        out.add(("sphere", n))
    return sorted(out)


@pytest.mark.parametrize("case,n", shapes())
def test_stage_copy_plan(case, n):
    nx, ny, nz = n
    wrap = case != "cavity"
    g, runs = plan(nx, ny, nz, MODES[case])
    if g is None:
        assert nx % 2 or nx > 1024 or (not wrap and nx < 4), f"{case} {n} should be staged"
        return
    if g["flat"]:
        assert case == "sphere"
        check_flat(g, runs, nx, ny, nz)
        return
    assert case != "sphere" or ny * g["P"] < 1008 + 2 * g["P"] + 16, f"{case} {n} should take flat tiles"
    P, R, cap = g["P"], g["R"], g["cap"]
    assert g["pitch"] == P and P % 8 == 0 and P >= nx
    assert 1 <= R <= ny and R * P <= cap and g["nty"] * R >= ny
    assert (g["sq"] * ELEM) % 16 == 0 and (g["base"] * ELEM) % 16 == 0

    # the cavity's wall records: one copy a tile, its rows in order
    rec = runs[:, 1] == 27
    if wrap:
        assert not rec.any()
    else:
        rr = runs[rec].astype(np.int64)
        assert len(rr) == g["nty"] * nz and np.array_equal(rr[:, 0], np.arange(len(rr)))
        j0 = (rr[:, 0] % g["nty"]) * R
        k = rr[:, 0] // g["nty"]
        rv = np.minimum(R, ny - j0)
        assert np.array_equal(rr[:, 3], (k * ny + j0) * (REC_BYTES // ELEM))
        assert np.array_equal(rr[:, 5], rv * REC_BYTES) and rr[:, 5].max() <= REC_AREA
        assert np.all((rr[:, 3] * ELEM) % 16 == 0) and np.all(rr[:, 5] % 16 == 0)
    rec_per_tile = np.bincount(runs[rec, 0], weights=runs[rec, 5].astype(np.int64), minlength=g["nty"] * nz)
    runs = runs[~rec]

    t, q, pop, src, dst, nbytes = (runs[:, i].astype(np.int64) for i in range(6))
    # alignment and size of every bulk copy
    assert np.all(nbytes > 0) and np.all(nbytes % 16 == 0)
    assert np.all((src * ELEM) % 16 == 0) and np.all((dst * ELEM) % 16 == 0)
    # whole rows
    row_bytes = P * ELEM
    assert np.all(nbytes % row_bytes == 0)
    rel = src - g["base"]
    assert np.all(rel >= 0) and np.all(rel % P == 0)
    nrows = nbytes // row_bytes
    plane, row0 = rel // g["sz"], (rel % g["sz"]) // P
    assert np.all(plane < nz) and np.all(row0 + nrows <= ny), "copy leaves its source plane"
    slot0 = dst - q * cap
    assert np.all(slot0 >= 0) and np.all(slot0 % P == 0) and np.all(slot0 + nbytes // ELEM <= cap)
    # bytes per tile (one mbarrier transaction count)
    per_tile = np.bincount(t, weights=nbytes, minlength=g["nty"] * nz) + rec_per_tile
    assert per_tile.max() <= MAX_TX

    # every slot row holds exactly the row its cells pull
    got = {}
    for i in range(len(runs)):
        for r in range(int(nrows[i])):
            key = (int(t[i]), int(q[i]), int(slot0[i]) // P + r)
            assert key not in got, f"slot row written twice: {key}"
            got[key] = (int(pop[i]), int(plane[i]), int(row0[i]) + r)
    for tile in range(g["nty"] * nz):
        j0, k = (tile % g["nty"]) * R, tile // g["nty"]
        rv = min(R, ny - j0)
        for qq in range(27):
            for r in range(rv):
                kk, jj = k - EZ[qq], j0 + r - EY[qq]
                if wrap:
                    want = (qq, kk % nz, jj % ny)
                elif 0 <= kk < nz and 0 <= jj < ny:
                    want = (qq, kk, jj)
                else:
                    want = (BB[qq], k, j0 + r)
                assert got.pop((tile, qq, r), None) == want, (tile, qq, r)
    assert not got, f"rows copied beyond the tiles: {sorted(got)[:4]}"


def test_bounce_table_matches():
    assert all(BB[BB[q]] == q and (EX[BB[q]], EY[BB[q]], EZ[BB[q]]) == (-EX[q], -EY[q], -EZ[q]) for q in range(27))
