"""The oracle's NCC search pinned against the reference's own OpenCL kernel.

tests/golden/optkmatch_cases.npz holds outputs of optKmatch
(src/mirorr/kernels/optKmatchMask.cl) compiled for the CPU
(tests/golden/make_golden.py).  The oracle restates the CPU matcher
(itkBlockMatcher.txx); both must pick the same match wherever the kernel's
best/second gap exceeds 1e-4, and report the same best score to 1e-6.
"""
import numpy as np
import pytest

from oracle import oracle as O

CASES = ["plain_bw4_w7_g3", "masked_bw4_w7_g3", "plain_bw4_w5_g2", "plain_bw2_w5_g2",
         "plain_bw4_w9_g3", "flat_bw4_w5_g2"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_kernel(golden, name):
    c = golden[name]
    bw, nw, bgap, ngap = [int(v) for v in c["params"]]
    r = O.match_blocks(c["base"], c["search"], c["bmask"], c["smask"],
                       O.BMParams(bw, bgap, ngap, nw, 1.0), threads=4)
    d, h, w = c["base"].shape
    lin = r.match[:, 2] * w * h + r.match[:, 1] * w + r.match[:, 0]
    gap = c["ref_best"].astype(np.float64) - c["ref_second"].astype(np.float64)
    clear = gap > 1e-4
    assert clear.sum() > 0.5 * gap.size
    np.testing.assert_array_equal(lin[clear], c["ref_match"][clear])
    np.testing.assert_allclose(r.best, c["ref_best"], atol=1e-6, rtol=0)
    np.testing.assert_allclose(r.second, c["ref_second"], atol=1e-6, rtol=0)


def test_flat_region_scores_minus_two(golden):
    c = golden["flat_bw4_w5_g2"]
    bw, nw, bgap, ngap = [int(v) for v in c["params"]]
    r = O.match_blocks(c["base"], c["search"], c["bmask"], c["smask"],
                       O.BMParams(bw, bgap, ngap, nw, 1.0), threads=2)
    # blocks lying wholly in the constant slab have zero base variance
    assert np.any(c["ref_best"] == -2.0)
    np.testing.assert_array_equal(r.best == -2.0, c["ref_best"] == -2.0)
