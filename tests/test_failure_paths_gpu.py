"""Failure paths of the device code, made to happen without faulting the GPU.

* Every grid-barrier wait of the fused streaming kernel is bounded.  With the
  deadline shortened to 1 ns (sb_set_wait_deadline_ns), the first wait that
  polls the barrier word 64 times gives up: it sets the launch's error word,
  every block returns, and splatt_b200_stream_push reports
  SPLATT_ERROR_DEVICE within a fraction of the default 2 s deadline.  The
  context stays usable: the deadline is restored and a fresh stream then
  matches the oracle (time rows within 1e-9 relative).
* A non-positive pivot in the regularised normal equations' Cholesky
  (a rank-deficient Gram: a zero factor column with no regularisation) is
  reported in the kernel's status word as the failing pivot + 1; the kernel
  does not trap, and the next factorisation on the same context succeeds.
  The reference prints "DPOTRF returned %d" and carries on
  (src/matrix.c:118-121).
"""
import ctypes as C
import time

import numpy as np
import pytest

import splatt_b200 as sb
import splatt_synth as S

pytestmark = pytest.mark.gpu


def _set_deadline(lib, ns):
    f = lib.L.sb_set_wait_deadline_ns
    f.argtypes = [C.c_uint64]
    f.restype = C.c_int
    assert f(ns) == 0


def test_grid_barrier_wait_expires_as_device_error(lib64, port):
    inds, vals, dims = S.stream_tensor(300, 200, 4, 0, 400, 0.5, 1.1, seed=4)
    si, sv, offs, _ = sb.parse_stream(inds, vals, dims, 2)
    a, b = int(offs[0]), int(offs[1])
    st = sb.Stream(lib64, 3, 2, dims, 16, exec_=sb.FUSED)
    _set_deadline(lib64, 1)
    try:
        t0 = time.perf_counter()
        with pytest.raises(sb.SplattError):
            st.push([x[a:b] for x in si], sv[a:b])
        elapsed = time.perf_counter() - t0
    finally:
        _set_deadline(lib64, 0)
    lib64.L.splatt_b200_stream_status.argtypes = [C.c_void_p]
    assert lib64.L.splatt_b200_stream_status(st.h) == sb.SPLATT_ERROR_DEVICE
    assert elapsed < 1.0, elapsed
    st.free()
    got = lib64.stream_run(inds, vals, dims, 2, 16, seed=11, exec_=sb.FUSED)
    ref = port.stream(inds, vals, dims, 2, 16, seed=11)
    assert np.abs(got["time"] - ref["time"]).max() <= 1e-9 * np.abs(ref["time"]).max()
    assert (got["outer"] == ref["outer"]).all()


def _chol(lib, G, R):
    import torch
    f = lib.L.sb_form_gram_chol
    f.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                  C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    Lt = torch.empty(R, R, dtype=torch.float64, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    grams = (C.c_void_p * 1)(G.data_ptr())
    torch.cuda.synchronize()
    rc = f(grams, 1, 1, R, 0.0, 0, Lt.data_ptr(), None, status.data_ptr())
    lib.L.sb_sync()
    return rc, int(status.item()), Lt


def test_cholesky_nonpositive_pivot_is_a_status(lib64):
    import torch
    R = 8
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.rand(50, R, dtype=torch.float64, device="cuda", generator=g)
    A[:, 3] = 0.0
    G = torch.triu(A.T @ A).contiguous()
    rc, status, _ = _chol(lib64, G, R)
    assert rc == 0
    assert status == 4                      # pivot 3 (0-based) + 1
    A[:, 3] = 1.0
    G = torch.triu(A.T @ A).contiguous()
    rc, status, Lt = _chol(lib64, G, R)
    assert rc == 0 and status == 0
    full = (A.T @ A)
    assert float((Lt.T @ Lt - full).abs().max() / full.abs().max()) <= 1e-12
