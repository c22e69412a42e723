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


def test_autotuner_picks_a_shape_and_keeps_results(lib32, port):
    """The first MTTKRP of a bucket (>= 2^20 nonzeros) times the launch-shape
    candidates and records the fastest (sb_mttkrp_tune_table grows); that
    call and the next (which reuses the shape) both match the oracle, and so
    does the heuristic shape with the tuner off."""
    import ctypes as C
    L = lib32.L
    L.sb_mttkrp_autotune.argtypes = [C.c_int]
    L.sb_mttkrp_tune_table.argtypes = [C.POINTER(C.c_int), C.c_int]
    L.sb_mttkrp_tune_table.restype = C.c_int
    inds, vals, dims = _zipf((200_000, 60_000, 4_000, 100), 2_500_000, 35)
    R = 48                       # a rank bucket no other test tunes
    rng = np.random.default_rng(8)
    mats = [rng.random((d, R), dtype=np.float32) for d in dims]
    i64 = [x.astype(np.uint64) for x in inds]
    m64 = [m.astype(np.float64) for m in mats]
    exp = port.mttkrp_coo(i64, vals.astype(np.float64), np.array(dims, np.uint64), 0, m64)
    csf = lib32.csf_convert(inds, vals, sb.CSF_ALLMODE)
    tab = (C.c_int * (8 * 128))()
    try:
        n0 = L.sb_mttkrp_tune_table(tab, 128)
        for _ in range(2):
            got = lib32.mttkrp(csf, 0, mats).astype(np.float64)
            assert np.abs(got - exp).max() / np.abs(exp).max() <= 2e-5
        n1 = L.sb_mttkrp_tune_table(tab, 128)
        assert n1 == n0 + 1
        e = list(tab[8 * n0: 8 * n0 + 8])
        assert e[0] == 1 and e[1] == 4 and e[2] == 0 and e[3] == 5     # FP32, 4 levels, root, R 48
        assert e[5] in (1, 4) and e[6] in (4, 8, 16, 32) and e[7] > 0
        L.sb_mttkrp_autotune(0)
        got = lib32.mttkrp(csf, 0, mats).astype(np.float64)
        assert np.abs(got - exp).max() / np.abs(exp).max() <= 2e-5
    finally:
        L.sb_mttkrp_autotune(1)
        csf.free()
