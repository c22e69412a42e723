"""Streaming CPD per-slice update on the device vs the oracle (pinned to the
reference's StreamCPD): time row of every slice, final factors, outer
iteration counts and the per-slice ("local-1") error.

FP64 (plain and fused executors): time rows and factors within 1e-9
relative max error, identical outer-iteration counts, local error^2 within
1e-9.  FP32 + FP64-solve precision: |delta error^2| <= 1e-4 per slice
against the FP64 oracle (the fit-tolerance bar for the FP32 mode)."""
import numpy as np
import pytest

import splatt_b200 as sb
import splatt_synth as S

pytestmark = pytest.mark.gpu


def _data(seed=4, T=12, I=300, J=200, med=400):
    return S.stream_tensor(I, J, T, 0, med, 0.5, 1.1, seed=seed)


@pytest.mark.parametrize("exec_", [sb.PLAIN, sb.FUSED])
@pytest.mark.parametrize("R", [8, 16, 32])
def test_stream_fp64_matches_oracle(lib64, port, exec_, R):
    inds, vals, dims = _data()
    got = lib64.stream_run(inds, vals, dims, 2, R, seed=11, exec_=exec_, errs=True)
    ref = port.stream(inds, vals, dims, 2, R, seed=11)
    assert got["time"].shape == ref["time"].shape
    scale = np.abs(ref["time"]).max()
    assert np.abs(got["time"] - ref["time"]).max() <= 1e-9 * scale
    assert (got["outer"] == ref["outer"]).all()
    for m in (0, 1):
        a, b = got["factors"][m], ref["factors"][m]
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 1e-9 * max(np.abs(b).max(), 1.0)
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= 1e-9


def test_stream_other_mode_orders(lib64, port):
    # streamed mode first and in the middle, rank 64
    inds, vals, dims = _data(seed=7, T=6)
    for sm in (0, 1):
        perm = [2, 0, 1] if sm == 0 else [0, 2, 1]
        pi = [inds[p] for p in perm]
        pd = dims[perm]
        got = lib64.stream_run(pi, vals, pd, sm, 64, seed=3, exec_=sb.FUSED)
        ref = port.stream(pi, vals, pd, sm, 64, seed=3)
        assert np.abs(got["time"] - ref["time"]).max() <= 1e-9 * np.abs(ref["time"]).max()


def test_stream_fp32_fit_within_1e4(lib64, port):
    inds, vals, dims = _data(seed=5, T=10)
    got = lib64.stream_run(inds, vals, dims, 2, 16, seed=2, precision=sb.FP32,
                           exec_=sb.FUSED, errs=True)
    ref = port.stream(inds, vals, dims, 2, 16, seed=2)
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= 1e-4
