"""Root-output FP32 MTTKRP of 3- and 4-level ALLMODE trees (k_csf_root, the
static-MTTKRP kernel) vs the oracle on the shapes that stress its chunk /
fiber / node bookkeeping: one nonzero, a fiber split over many worker
chunks, fibers of one nonzero, roots and nodes split between chunks, ragged
nonzero counts, more than one column window (R = 128).

Tolerance: FP32 vs the FP64 oracle <= 2e-5 relative max-abs error (the bar
of the other FP32 MTTKRP tests; the reference's own FP32 test uses an
absolute 9e-3, tests/mttkrp_test.c:26)."""
import numpy as np
import pytest

import datasets as D
import splatt_b200 as sb

pytestmark = pytest.mark.gpu


def _mats(dims, R, seed):
    rng = np.random.default_rng(seed)
    return [(rng.random((int(d), R)) * 2 - 1).astype(np.float32) for d in dims]


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _dedup(inds, vals):
    key = np.stack(inds, axis=1)
    _, first = np.unique(key, axis=0, return_index=True)
    first = np.sort(first)
    return [x[first] for x in inds], vals[first]


def _check(lib, port, inds, vals, R, seed=3):
    dims = [int(x.max()) + 1 for x in inds]          # splatt_csf_convert's dims
    csf = lib.csf_convert(inds, vals, sb.CSF_ALLMODE)
    mats = _mats(dims, R, seed)
    m64 = [x.astype(np.float64) for x in mats]
    for m in range(len(inds)):
        got = lib.mttkrp(csf, m, mats)
        ref = port.mttkrp_coo(inds, vals, dims, m, m64)
        assert _relerr(got.astype(np.float64), ref) <= 2e-5, m


@pytest.mark.parametrize("name", ["small3", "med3", "small4", "zipf3", "zipf4"])
@pytest.mark.parametrize("R", [64, 128])
def test_root_root_datasets(lib32, port, name, R):
    inds, vals, _ = D.ALL[name]()
    _check(lib32, port, inds, vals, R)


@pytest.mark.parametrize("nmodes", [3, 4])
def test_root_single_nonzero(lib32, port, nmodes):
    inds = [np.array([i + 1], np.uint64) for i in range(nmodes)]
    vals = np.array([0.75])
    _check(lib32, port, inds, vals, 64)


@pytest.mark.parametrize("nmodes", [3, 4])
def test_root_long_fiber(lib32, port, nmodes):
    """One fiber of 20,000 nonzeros (every root / node / fiber above it shared)
    beside a scatter of short ones: the long fiber spans many chunks."""
    rng = np.random.default_rng(21)
    K = 20000
    dims = [40] * (nmodes - 1) + [K]
    long_ = [np.zeros(K, np.uint64) for _ in range(nmodes - 1)] + [np.arange(K, dtype=np.uint64)]
    n = 3000
    rest = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    inds = [np.concatenate([a, b]) for a, b in zip(long_, rest)]
    vals = rng.random(K + n) + 0.01
    inds, vals = _dedup(inds, vals)
    _check(lib32, port, inds, vals, 64)


@pytest.mark.parametrize("nmodes", [3, 4])
def test_root_singleton_fibers(lib32, port, nmodes):
    """Hypersparse: almost every fiber and node holds one nonzero."""
    rng = np.random.default_rng(22)
    dims = [3000] * nmodes
    n = 25000
    inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    vals = rng.random(n) + 0.01
    inds, vals = _dedup(inds, vals)
    _check(lib32, port, inds, vals, 64)


@pytest.mark.parametrize("nnz", [5, 17, 33, 257, 1000])
def test_root_ragged_sizes(lib32, port, nnz):
    """Nonzero counts that leave partial stages, windows and chunks."""
    rng = np.random.default_rng(nnz)
    dims = [17, 13, 11, 7]
    inds = [rng.integers(0, d, 4 * nnz).astype(np.uint64) for d in dims]
    vals = rng.random(4 * nnz) + 0.01
    inds, vals = _dedup(inds, vals)
    inds, vals = [x[:nnz] for x in inds], vals[:nnz]
    _check(lib32, port, inds, vals, 64)
