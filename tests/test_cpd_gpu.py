"""CPD-ALS on the device vs the oracle (pinned to the reference's splatt_cpd):
same glibc-rand initial factors, TWOMODE CSF, closed-form ALS.

Tolerances (FP64): per-run fit |delta| <= 1e-10; lambda and factors relative
max error <= 1e-8.  ALS amplifies last-ulp differences of reordered sums
over iterations, so factors get a looser bar than the single MTTKRP."""
import numpy as np
import pytest

import datasets as D

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,R,its", [("small3", 8, 20), ("med3", 16, 20),
                                        ("small4", 6, 15), ("zipf3", 10, 10)])
def test_cpd_matches_oracle(lib64, port, name, R, its):
    inds, vals, dims = D.ALL[name]()
    csf = lib64.csf_convert(inds, vals, 1)
    got = lib64.cpd(csf, R, niters=its, tol=0.0, seed=42)
    ref = port.cpd(inds, vals, dims, R, its, 0.0, 42)
    assert abs(got["fit"] - ref["fit"]) <= 1e-10
    assert np.abs(got["lam"] - ref["lam"]).max() <= 1e-8 * np.abs(ref["lam"]).max()
    for a, b in zip(got["factors"], ref["factors"]):
        assert np.abs(a - b).max() <= 1e-8 * max(np.abs(b).max(), 1.0)


@pytest.mark.parametrize("name,R,its", [("med3", 16, 10), ("small4", 6, 10)])
def test_cpd_fp32_fit_within_1e4(lib32, port, name, R, its):
    """The 32-bit build (uint32 / float, Grams on the tensor cores with split
    TF32 products): fit within 1e-4 of the FP64 oracle from the same initial
    factors."""
    inds, vals, dims = D.ALL[name]()
    csf = lib32.csf_convert([x.astype(np.uint32) for x in inds], vals.astype(np.float32), 1)
    got = lib32.cpd(csf, R, niters=its, tol=0.0, seed=42)
    ref = port.cpd(inds, vals, dims, R, its, 0.0, 42)
    assert abs(got["fit"] - ref["fit"]) <= 1e-4, (got["fit"], ref["fit"])
