"""The FP32 precision mode's Gram on the tensor cores (sb_gram with split TF32
products, k_gram_tc.cu): G = A^T A of an FP32 factor, against a PyTorch FP64
reference of the same op on the same input.  Ranks that are multiples of 4
with 16-byte rows take the TMA-fed kernel, the others the thread-loaded one;
both are covered.

Tolerance: max |G - G_ref| / max |G_ref| <= 2e-5.  The split keeps each
element to ~2^-22 relative; the tensor core accumulates in FP32 over at most
4096 rows per CTA and the CTAs add in FP64."""
import ctypes as C

import numpy as np
import pytest

import splatt_b200 as sb

pytestmark = pytest.mark.gpu

SB_F32, SB_GRAM_TF32X3 = 1, 1


def _gram(lib, A, R, ld, precision):
    import torch
    L = lib.L
    L.sb_gram.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_int]
    L.sb_gram.restype = C.c_int
    G = torch.full((R, R), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = L.sb_gram(A.data_ptr(), SB_F32, A.shape[0], R, ld, G.data_ptr(), precision)
    assert rc == 0
    L.sb_sync()
    return G


@pytest.mark.parametrize("I,R,pad", [(1, 1, 0), (7, 5, 3), (32, 16, 0), (33, 31, 1), (1000, 32, 0),
                                     (4096, 33, 0), (4097, 48, 5), (100003, 64, 0),
                                     (2000003, 64, 0), (300000, 8, 0), (50000, 64, 4),
                                     (70001, 40, 0), (129, 4, 0)])
def test_gram_tc_vs_fp64(lib32, I, R, pad):
    import torch
    g = torch.Generator(device="cuda").manual_seed(I * 131 + R)
    ld = R + pad
    full = torch.randn(I, ld, device="cuda", dtype=torch.float32, generator=g)
    full[:, R:] = float("nan")            # padding columns must never be read
    A = full[:, :R]
    ref = torch.triu(A.double().T @ A.double())     # sb_gram fills the upper triangle
    for _ in range(2):                    # two calls in a row: no state carried over
        got = _gram(lib32, full, R, ld, SB_GRAM_TF32X3)
        assert not torch.isnan(got).any()
        assert float(torch.tril(got, -1).abs().max() if R > 1 else 0.0) == 0.0
        err = float((got - ref).abs().max() / ref.abs().max())
        assert err <= 2e-5, (I, R, err)
    # and against the FP64-accumulating CUDA-core path on the same FP32 input
    plain = _gram(lib32, full, R, ld, 0)
    assert float((got - plain).abs().max() / plain.abs().max()) <= 2e-5


def test_gram_tc_ranks_beyond_64_use_cuda_cores(lib32):
    import torch
    A = torch.randn(5000, 80, device="cuda", dtype=torch.float32)
    got = _gram(lib32, A, 80, 80, SB_GRAM_TF32X3)
    ref = torch.triu(A.double().T @ A.double())
    assert float((got - ref).abs().max() / ref.abs().max()) <= 1e-6
