"""The root MTTKRP (k_csf_root) on trees of millions of nonzeros, beyond the
small parity tensors: 3- and 4-mode Zipf(1.2) tensors, FP32 values and
factors, uint32 indices, rank 64, one CSF per mode (every MTTKRP writes the
root of its own tree).  Every mode's MTTKRP matches the oracle's FP64 COO
MTTKRP within 2e-5 relative (max-abs error / max-abs value): hot root rows
sum over hundreds of thousands of nonzeros here, through many workers'
atomics."""
import numpy as np
import pytest

import splatt_b200 as sb
import splatt_synth as S

pytestmark = pytest.mark.gpu


def _zipf(dims, nnz, seed):
    import torch
    dinds, dvals, nd = S.zipf_tensor_torch(torch, list(dims), nnz, 1.2, seed)
    inds = [x.cpu().numpy().astype(np.uint32) for x in dinds]
    return inds, dvals.cpu().numpy(), nd


def _check_all_modes(lib32, port, inds, vals, dims, R):
    rng = np.random.default_rng(7)
    mats = [rng.random((d, R), dtype=np.float32) for d in dims]
    csf = lib32.csf_convert(inds, vals, sb.CSF_ALLMODE)
    i64 = [x.astype(np.uint64) for x in inds]
    v64 = vals.astype(np.float64)
    m64 = [m.astype(np.float64) for m in mats]
    try:
        for m in range(len(dims)):
            exp = port.mttkrp_coo(i64, v64, np.array(dims, np.uint64), m, m64)
            got = lib32.mttkrp(csf, m, mats).astype(np.float64)
            err = np.abs(got - exp).max() / np.abs(exp).max()
            assert err <= 2e-5, "mode %d relative error %g" % (m, err)
    finally:
        csf.free()


def test_root_mttkrp_4mode_6m(lib32, port):
    inds, vals, dims = _zipf((400_000, 120_000, 9_000, 300), 6_000_000, 31)
    _check_all_modes(lib32, port, inds, vals, dims, 64)


def test_root_mttkrp_3mode_5m(lib32, port):
    inds, vals, dims = _zipf((300_000, 100_000, 2_000, 1), 5_000_000, 32)
    _check_all_modes(lib32, port, inds[:3], vals, dims[:3], 64)
