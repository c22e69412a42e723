"""splatt_b200_gram_noalloc: the Gram entry point that allocates nothing.

It exists for callers that must not call cudaMalloc / cudaFree (a process
whose device memory is already split between its own pools, or a plug-in
whose host application owns the allocator).  Its partial sums live in a
fixed device array shared by every call, so this test checks, through the
C ABI, calls in a row with different shapes and types (up to the rank
limit, and with a row stride wider than the rank) against the
regular allocating Gram entry point (sb_gram) at the tolerance the other
FP64 kernel tests use (1e-12 relative), and the rejection of ranks above
the array's limit.  The file sorts last so a failure here leaves every other
test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(L):
    L.splatt_b200_gram_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint32,
                                           C.c_uint32, C.c_void_p, C.c_void_p]
    L.splatt_b200_gram_noalloc.restype = C.c_int
    L.sb_gram.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32,
                          C.c_void_p, C.c_int]
    L.sb_gram.restype = C.c_int
    L.sb_sync.restype = C.c_int


def test_gram_noalloc_matches_allocating_gram(lib64):
    import torch
    L = lib64.L
    _bind(L)
    stream = C.c_void_p(L.splatt_b200_get_stream())
    gen = torch.Generator(device="cuda").manual_seed(5)
    # calls in a row: each must not see the previous one's partials.  The
    # shapes reach the array's limits: rank 64 (every thread of a block
    # holds up to 9 upper-triangle pairs), rank 63 (not a power of two) and
    # a row stride wider than the rank (a 5000 x 72 buffer read as rank 64)
    for nrows, rank, ld, dt, vt in [(5000, 32, 32, torch.float64, 0),
                                    (777, 16, 16, torch.float32, 1),
                                    (9000, 64, 64, torch.float64, 0),
                                    (3001, 63, 63, torch.float32, 1),
                                    (5000, 64, 72, torch.float64, 0)]:
        buf = torch.randn(nrows, ld, dtype=dt, device="cuda", generator=gen)
        g_new = torch.full((rank, rank), float("nan"), dtype=torch.float64, device="cuda")
        g_ref = torch.zeros((rank, rank), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert L.splatt_b200_gram_noalloc(C.c_void_p(buf.data_ptr()), vt, nrows, rank, ld,
                                          C.c_void_p(g_new.data_ptr()), stream) == 1
        assert L.sb_gram(C.c_void_p(buf.data_ptr()), vt, nrows, rank, ld,
                         C.c_void_p(g_ref.data_ptr()), 0) == 0
        assert L.sb_sync() == 0
        upper = np.triu(np.ones((rank, rank), bool))
        a, b = g_new.cpu().numpy()[upper], g_ref.cpu().numpy()[upper]
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
        host = buf[:, :rank].double().cpu().numpy()
        assert np.abs(a - (host.T @ host)[upper]).max() <= 1e-12 * np.abs(b).max()


def test_gram_noalloc_rejects_rank_above_limit(lib64):
    import torch
    L = lib64.L
    _bind(L)
    A = torch.zeros((4, 65), dtype=torch.float64, device="cuda")
    G = torch.zeros((65, 65), dtype=torch.float64, device="cuda")
    rc = L.splatt_b200_gram_noalloc(C.c_void_p(A.data_ptr()), 0, 4, 65, 65,
                                    C.c_void_p(G.data_ptr()), C.c_void_p(L.splatt_b200_get_stream()))
    assert rc == 2
