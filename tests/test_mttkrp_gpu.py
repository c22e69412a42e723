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


def test_csf_convert_device_fp32(lib32, port):
    """splatt_b200_csf_convert_device (COO already on the device, no host
    mirror) + splatt_b200_mttkrp_device, FP32, every mode, vs the oracle."""
    import ctypes
    import torch
    import splatt_b200 as sb
    inds, vals, dims = D.zipf4()
    L = lib32.L
    L.splatt_b200_csf_convert_device.argtypes = [
        ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
        ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int,
        ctypes.POINTER(ctypes.POINTER(lib32.Csf)), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    L.splatt_b200_csf_convert_device.restype = ctypes.c_int
    di = [torch.from_numpy(x.astype(np.int32)).cuda() for x in inds]
    dv = torch.from_numpy(vals.astype(np.float32)).cuda()
    opts = lib32.opts(csf_alloc=sb.CSF_ALLMODE)
    csf = ctypes.POINTER(lib32.Csf)()
    d64 = (ctypes.c_uint64 * 4)(*[int(x) for x in dims])
    dp = (ctypes.c_void_p * 4)(*[x.data_ptr() for x in di])
    torch.cuda.synchronize()
    lib32.check(L.splatt_b200_csf_convert_device(4, len(vals), d64, dp, ctypes.c_void_p(dv.data_ptr()),
                                                 1, ctypes.byref(csf), opts, 0), "convert_device")
    mats = _mats(dims, 64, 11)
    dm = [torch.from_numpy(x.astype(np.float32)).cuda() for x in mats]
    mp = (ctypes.c_void_p * 4)(*[x.data_ptr() for x in dm])
    for m in range(4):
        out = torch.empty(int(dims[m]), 64, device="cuda", dtype=torch.float32)
        torch.cuda.synchronize()
        lib32.check(L.splatt_b200_mttkrp_device(m, 64, csf, opts, mp, 64,
                                                ctypes.c_void_p(out.data_ptr()), 64, 1),
                    "mttkrp_device")
        L.sb_sync()
        ref = port.mttkrp_coo(inds, vals, dims, m, [x.astype(np.float32).astype(np.float64)
                                                    for x in mats])
        assert _relerr(out.cpu().numpy().astype(np.float64), ref) <= 2e-5, m
    L.splatt_free_csf(csf, opts)
