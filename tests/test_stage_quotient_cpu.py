"""The staged kernels map a thread's pair to its tile row without an integer
division (small_quotient, imexlb_b200/csrc/stage_core.cuh): n / d as the
truncation of (n + 1/2) * RN(1/d) in FP32.  The claim is exactness for every
0 <= n < 2048 and 4 <= d <= 1024 (whole-row tiles: n < SLOT_CAP / 2 pairs,
d = half a row; flat tiles: n < P + C elements, d = the row pitch).  IEEE
FP32 arithmetic in numpy rounds the same way as the device's, so this checks
the bound on the CPU for every case."""
import numpy as np


def test_fp32_quotient_is_exact_for_every_tile_shape():
    n = np.arange(2048, dtype=np.int64)
    nf = n.astype(np.float32) + np.float32(0.5)
    for d in range(4, 1025):
        inv = np.float32(1.0) / np.float32(d)  # correctly rounded, like __frcp_rn
        q = np.trunc((nf * inv).astype(np.float32)).astype(np.int64)
        assert np.array_equal(q, n // d), d
