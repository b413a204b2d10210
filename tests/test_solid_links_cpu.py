"""The standard sphere's solid-link table, checked on the CPU.

For every fluid cell, bit q is set when its pull along -e_q starts in a
solid cell: x is not periodic (the inlet and outlet rules own the x ends),
y and z are.  The library builds the table from the solid's neighbourhood
only, one plane per host thread (imexlb_debug_solid_links); here it is
compared with a direct restatement over every cell and population, for
voxelised spheres and for random masks whose solid touches and wraps the
periodic sides.
"""
import ctypes

import numpy as np
import pytest

from imexlb_b200 import api

EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1])
EY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, -1, 1])
EZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, -1, 1])


def library_links(fluid):
    nz, ny, nx = fluid.shape
    lib = api.load_library()
    fn = lib.imexlb_debug_solid_links
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 3
    f = np.ascontiguousarray(fluid, dtype=np.uint8)
    links = np.zeros(f.shape, np.uint32)
    box = np.zeros(6, np.int32)
    assert fn(nx, ny, nz, f.ctypes.data, links.ctypes.data, box.ctypes.data) == 0
    return links, box


def reference_links(fluid):
    nz, ny, nx = fluid.shape
    solid = fluid == 0
    links = np.zeros(fluid.shape, np.uint32)
    for q in range(27):
        # source of the pull along -e_q: (x - ex, y - ey, z - ez), y and z wrapped
        src = np.roll(solid, shift=(EZ[q], EY[q]), axis=(0, 1))
        shifted = np.zeros_like(src)
        if EX[q] > 0:
            shifted[:, :, 1:] = src[:, :, :-1]
        elif EX[q] < 0:
            shifted[:, :, :-1] = src[:, :, 1:]
        else:
            shifted = src
        links |= (shifted & ~solid).astype(np.uint32) << np.uint32(q)
    box = np.array([nx, ny, nz, -1, -1, -1], np.int32)
    k, j, i = np.nonzero(links)
    if len(i):
        box = np.array([i.min(), j.min(), k.min(), i.max(), j.max(), k.max()], np.int32)
    return links, box


def sphere(nx, ny, nz, c, d):
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return ((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 > 0.25 * d * d).astype(np.uint8)


CASES = [
    ("sphere", sphere(48, 16, 16, (12.0, 8.0, 8.0), 6.0)),
    ("sphere", sphere(96, 24, 24, (24.0, 12.0, 12.0), 4.0)),
    ("touching y and z", sphere(40, 20, 18, (20.0, 0.0, 17.0), 9.0)),
    ("at the x ends", sphere(30, 16, 16, (0.0, 8.0, 8.0), 7.0) & sphere(30, 16, 16, (29.0, 8.0, 8.0), 7.0)),
    ("no solid", np.ones((8, 9, 10), np.uint8)),
    ("all solid", np.zeros((4, 5, 6), np.uint8)),
    ("thin y", sphere(20, 2, 12, (10.0, 1.0, 6.0), 5.0)),
]


@pytest.mark.parametrize("name,fluid", CASES, ids=[c[0] for c in CASES])
def test_solid_links_match_direct_restatement(name, fluid):
    got, gbox = library_links(fluid)
    want, wbox = reference_links(fluid)
    assert np.array_equal(got, want), name
    assert np.array_equal(gbox, wbox), (name, gbox, wbox)


def test_solid_links_random_masks():
    rng = np.random.default_rng(11)
    for _ in range(6):
        nz, ny, nx = rng.integers(3, 14, size=3)
        fluid = (rng.random((nz, ny, nx)) > 0.08).astype(np.uint8)
        got, gbox = library_links(fluid)
        want, wbox = reference_links(fluid)
        assert np.array_equal(got, want)
        assert np.array_equal(gbox, wbox)
