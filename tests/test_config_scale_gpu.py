"""Parity at the benchmark workloads' own sizes (not only on toy tensors).

* plain CPD-ALS on the full 1000x800x600, 500,000-nonzero, rank-16,
  20-iteration workload (FP64, TWOMODE CSF) against the oracle: fit within
  1e-10, lambda and factors within 1e-8 relative (the bars of the small CPD
  tests; ALS amplifies last-ulp reorderings of the sums);
* the static MTTKRP of the 4-mode 2Mx500Kx50Kx1K Zipf(1.2) distribution at a
  10M-nonzero subset (FP32 values and factors, uint32 indices, rank 64, one
  CSF per mode) against the oracle's FP64 COO MTTKRP: every mode within 2e-5
  relative (max-abs error / max-abs value).  At this size a hot root row sums
  over a million nonzeros, so the atomics on split nodes and the chunked
  accumulation order are exercised far beyond the small cases;
* the first slices of the 20000x10000x500 streaming workload (rank 32, frob
  1e-2, forgetting 0.95, FP64, fused executor) against the oracle: time rows
  within 1e-9 relative, identical outer-iteration counts, local error^2
  within 1e-9.
"""
import numpy as np
import pytest

import splatt_b200 as sb
import splatt_synth as S

pytestmark = pytest.mark.gpu

C1 = dict(dims=(1000, 800, 600), nnz=500_000, rank=16, its=20)
C3 = dict(dims=(2_000_000, 500_000, 50_000, 1_000), zipf=1.2, rank=64)
C2 = dict(I=20000, J=10000, T=500, total_nnz=50_000_000, median=80000, sigma=0.8, zipf=1.1,
          rank=32, reg=1e-2, forget=0.95)


def test_c1_full_workload_cpd_matches_oracle(lib64, port):
    inds, vals, dims = S.uniform_tensor(list(C1["dims"]), C1["nnz"], seed=2024)
    csf = lib64.csf_convert(inds, vals, sb.CSF_TWOMODE)
    got = lib64.cpd(csf, C1["rank"], niters=C1["its"], tol=0.0, seed=2024)
    csf.free()
    ref = port.cpd(inds, vals, dims, C1["rank"], C1["its"], 0.0, 2024)
    assert abs(got["fit"] - ref["fit"]) <= 1e-10, (got["fit"], ref["fit"])
    assert np.abs(got["lam"] - ref["lam"]).max() <= 1e-8 * np.abs(ref["lam"]).max()
    for a, b in zip(got["factors"], ref["factors"]):
        assert np.abs(a - b).max() <= 1e-8 * max(np.abs(b).max(), 1.0)


def test_c3_distribution_10m_subset_mttkrp_matches_oracle(lib32, port):
    import torch
    dinds, dvals, dims = S.zipf_tensor_torch(torch, C3["dims"], 10_000_000, C3["zipf"], 2024)
    inds = [x.cpu().numpy().astype(np.uint32) for x in dinds]
    vals = dvals.cpu().numpy()
    del dinds, dvals
    nnz = len(vals)
    assert nnz >= 10_000_000
    R = C3["rank"]
    rng = np.random.default_rng(3)
    mats = [rng.random((d, R), dtype=np.float32) for d in dims]
    csf = lib32.csf_convert(inds, vals, sb.CSF_ALLMODE)
    i64 = [x.astype(np.uint64) for x in inds]
    v64 = vals.astype(np.float64)
    m64 = [m.astype(np.float64) for m in mats]
    for m in range(4):
        got = lib32.mttkrp(csf, m, mats)
        exp = port.mttkrp_coo(i64, v64, np.array(dims, np.uint64), m, m64)
        err = np.abs(got.astype(np.float64) - exp).max() / np.abs(exp).max()
        assert err <= 2e-5, "mode %d relative error %g" % (m, err)
    csf.free()


def test_c2_first_slices_stream_matches_oracle(lib64, port):
    T = 6
    inds, vals, dims = S.stream_tensor(C2["I"], C2["J"], C2["T"], C2["total_nnz"], C2["median"],
                                       C2["sigma"], C2["zipf"], seed=2024, sort_slices=True,
                                       max_t=T, exact=True)
    dims = np.array([dims[0], dims[1], T], np.uint64)
    got = lib64.stream_run(inds, vals, dims, 2, C2["rank"], forget=C2["forget"], reg=C2["reg"],
                           seed=2024, exec_=sb.FUSED, errs=True)
    ref = port.stream(inds, vals, dims, 2, C2["rank"], C2["forget"], C2["reg"], 200, seed=2024)
    assert got["time"].shape == ref["time"].shape == (T, C2["rank"])
    assert np.abs(got["time"] - ref["time"]).max() <= 1e-9 * np.abs(ref["time"]).max()
    assert (got["outer"] == ref["outer"]).all(), (got["outer"], ref["outer"])
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= 1e-9
