"""CSF MTTKRP on the device vs the oracle for every mode, every allocation
scheme (root / internal / leaf traversals), FP64 and FP32 builds.

Tolerances: FP64 relative max-abs error <= 1e-12 (the plain FP64 bar);
FP32 build vs the FP64 oracle <= 2e-5 relative (the reference's own FP32
test uses an absolute 9e-3, tests/mttkrp_test.c:26)."""
import numpy as np
import pytest

import datasets as D

pytestmark = pytest.mark.gpu


def _mats(dims, R, seed):
    rng = np.random.default_rng(seed)
    return [rng.random((int(d), R)) * 2 - 1 for d in dims]


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", list(D.ALL))
@pytest.mark.parametrize("alloc", [0, 1, 2])
@pytest.mark.parametrize("R", [3, 16])
def test_mttkrp_fp64(lib64, port, name, alloc, R):
    inds, vals, dims = D.ALL[name]()
    csf = lib64.csf_convert(inds, vals, alloc)
    mats = _mats(dims, R, 5)
    for m in range(len(inds)):
        got = lib64.mttkrp(csf, m, mats)
        ref = port.mttkrp_coo(inds, vals, dims, m, mats)
        assert _relerr(got, ref) <= 1e-12, (name, alloc, m)


@pytest.mark.parametrize("R", [1, 5, 32, 64, 100])
def test_mttkrp_ranks(lib64, port, R):
    inds, vals, dims = D.zipf4()
    csf = lib64.csf_convert(inds, vals, 1)
    mats = _mats(dims, R, 7)
    for m in range(4):
        got = lib64.mttkrp(csf, m, mats)
        ref = port.mttkrp_coo(inds, vals, dims, m, mats)
        assert _relerr(got, ref) <= 1e-12, (R, m)


@pytest.mark.parametrize("alloc", [0, 2])
def test_mttkrp_fp32(lib32, port, alloc):
    inds, vals, dims = D.zipf4()
    csf = lib32.csf_convert(inds, vals, alloc)
    mats = _mats(dims, 64, 9)
    for m in range(4):
        got = lib32.mttkrp(csf, m, [x.astype(np.float32) for x in mats])
        ref = port.mttkrp_coo(inds, vals, dims, m,
                              [x.astype(np.float32).astype(np.float64) for x in mats])
        assert _relerr(got.astype(np.float64), ref) <= 2e-5, m
