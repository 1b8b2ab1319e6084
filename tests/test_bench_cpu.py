"""The bench's accounting on the CPU: the force-error norms and the
algorithmic / issued transform work that the roofline object is built from."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_force_error_norms():
    # two cases, three steps; case 0 has a large first-step force (impulsive start)
    fx0 = np.array([[100.0, 1.0, 1.0], [2.0, 2.0, 2.0]])
    fy0 = np.zeros_like(fx0)
    fx1 = fx0 + np.array([[0.0, 1e-9, 0.0], [0.0, 0.0, 4e-9]])
    fy1 = fy0 + np.array([[1e-8, 0.0, 0.0], [0.0, 0.0, 0.0]])
    hmax, hmed, smax, smed = bench.force_err(fx1, fy1, fx0, fy0)
    # history norm: max error over max |force| of the case
    h = [1e-8 / 100.0, 4e-9 / 2.0]
    # per step: the error over the same step's |force|
    s = [max(1e-8 / 100.0, 1e-9 / 1.0), 4e-9 / 2.0]
    assert np.isclose(hmax, max(h)) and np.isclose(hmed, np.median(h))
    assert np.isclose(smax, max(s)) and np.isclose(smed, np.median(s))


def test_algorithmic_transform_flops():
    # 7L+2 two-dimensional DSTs per case-step, each 2 (m-1)(n-1)[(m-1)+(n-1)]
    cases = [dict(m=129, n=129), dict(m=65, n=33)]
    got = bench.algorithmic_transform_flops(cases, [3, 2])
    want = 23 * 2.0 * 128 * 128 * 256 + 16 * 2.0 * 64 * 32 * 96
    assert got == want


def test_issued_tensor_flops():
    # one level: 2 Poisson solves of 6 + 6 products and 2 others of 6 + 3, four
    # GEMMs each, on 128-padded tiles with K padded to 64
    got = bench.issued_tensor_flops([dict(m=129, n=129)], [1])
    assert got == 4 * 2.0 * 128 ** 2 * 128 * (2 * 12 + 2 * 9)
    # m - 1 = 191 pads to 256 rows and columns and 192 in K
    got = bench.issued_tensor_flops([dict(m=192, n=192)], [1])
    assert got == 4 * 2.0 * 256 ** 2 * 192 * 42
    # the issued work always exceeds the algorithmic work (slices, corrections, padding)
    cases = [dict(m=m, n=m) for m in (128, 192, 256, 384, 512)]
    for L in (2, 3, 4, 5):
        nl = [L] * len(cases)
        assert bench.issued_tensor_flops(cases, nl) > 8 * bench.algorithmic_transform_flops(cases, nl)
