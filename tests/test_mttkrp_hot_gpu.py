"""The hot-row root MTTKRP (k_csf_root_hot): for a tree of at least 2^22
nonzeros (FP32, rank 64) the root MTTKRP reads the plan's most-fetched
factor rows from shared memory and every other row from global memory.

Checked here, on 3- and 4-mode Zipf tensors large enough to use it, one CSF
per mode (every MTTKRP writes the root of its own tree):
* the plan is built and used (sb_mttkrp_plan_build reports it usable);
* every mode's MTTKRP matches the oracle's FP64 COO MTTKRP within 2e-5
  relative (max-abs error / max-abs value), with the hot-row kernel
  (sb_mttkrp_root_hot(1)), the plain root kernel (0, the default) and the
  plain root kernel with L1 prefetch of the leaf rows (2) on the same trees;
* a tree below the size threshold, and an FP32 tree of rank 32, take the
  plain kernel and stay within the same bound."""
import ctypes as C

import numpy as np
import pytest

import splatt_b200 as sb
import splatt_synth as S

pytestmark = pytest.mark.gpu


def _bind(L):
    L.sb_mttkrp_root_hot.argtypes = [C.c_int]
    L.sb_mttkrp_root_hot.restype = None
    L.sb_mttkrp_plan_build.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.sb_mttkrp_plan_build.restype = C.c_int


def _zipf(dims, nnz, seed):
    import torch
    dinds, dvals, nd = S.zipf_tensor_torch(torch, list(dims), nnz, 1.2, seed)
    inds = [x.cpu().numpy().astype(np.uint32) for x in dinds]
    return inds, dvals.cpu().numpy(), nd


def _check_all_modes(lib32, port, inds, vals, dims, R, hot_flags, expect_plan):
    L = lib32.L
    _bind(L)
    rng = np.random.default_rng(7)
    mats = [rng.random((d, R), dtype=np.float32) for d in dims]
    csf = lib32.csf_convert(inds, vals, sb.CSF_ALLMODE)
    i64 = [x.astype(np.uint64) for x in inds]
    v64 = vals.astype(np.float64)
    m64 = [m.astype(np.float64) for m in mats]
    nmodes = len(dims)
    try:
        for t in range(nmodes):
            used = C.c_int(-1)
            assert L.sb_mttkrp_plan_build(C.c_void_p(csf.ptr[t].dev), C.byref(used)) == 0
            assert used.value == expect_plan
        exp = [port.mttkrp_coo(i64, v64, np.array(dims, np.uint64), m, m64)
               for m in range(nmodes)]
        for hot in hot_flags:
            L.sb_mttkrp_root_hot(hot)
            for m in range(nmodes):
                got = lib32.mttkrp(csf, m, mats).astype(np.float64)
                err = np.abs(got - exp[m]).max() / np.abs(exp[m]).max()
                assert err <= 2e-5, "hot %d mode %d relative error %g" % (hot, m, err)
    finally:
        L.sb_mttkrp_root_hot(0)
        csf.free()


def test_root_hot_4mode(lib32, port):
    inds, vals, dims = _zipf((400_000, 120_000, 9_000, 300), 6_000_000, 31)
    _check_all_modes(lib32, port, inds, vals, dims, 64, (1, 0, 2), 1)


def test_root_hot_3mode(lib32, port):
    inds, vals, dims = _zipf((300_000, 100_000, 2_000, 1), 5_000_000, 32)
    inds, dims = inds[:3], dims[:3]
    _check_all_modes(lib32, port, inds, vals, dims, 64, (1, 0, 2), 1)


def test_root_hot_not_used_below_threshold_or_other_rank(lib32, port):
    inds, vals, dims = _zipf((40_000, 12_000, 900, 30), 600_000, 33)
    _check_all_modes(lib32, port, inds, vals, dims, 64, (1,), 0)
    inds, vals, dims = _zipf((400_000, 120_000, 9_000, 300), 5_000_000, 34)
    _check_all_modes(lib32, port, inds, vals, dims, 32, (1,), 1)
