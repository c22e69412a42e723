"""Streaming CPD per-slice update on the device vs the oracle (pinned to the
reference's StreamCPD): time row of every slice, final factors, outer
iteration counts and the per-slice ("local-1") error.

FP64 (plain and fused executors): time rows and factors within 1e-9
relative max error, identical outer-iteration counts, local error^2 within
1e-9; the same with the non-negative max-column-norm prox on the
non-streamed modes (`--con=nonneg`), whose factors must stay >= 0, and with
lasso on them (`--reg=l1,L`, ADMM in independent 50-row chunks).  FP32 + FP64-solve precision: |delta error^2| <= 1e-4 per slice
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


@pytest.mark.parametrize("exec_", [sb.PLAIN, sb.FUSED])
@pytest.mark.parametrize("R", [8, 48])
def test_stream_nonneg_fp64_matches_oracle(lib64, port, exec_, R):
    inds, vals, dims = _data(seed=6, T=10)
    got = lib64.stream_run(inds, vals, dims, 2, R, seed=13, exec_=exec_, errs=True, nonneg=True)
    ref = port.stream(inds, vals, dims, 2, R, seed=13, nonneg=True)
    scale = np.abs(ref["time"]).max()
    assert np.abs(got["time"] - ref["time"]).max() <= 1e-9 * scale
    assert (got["outer"] == ref["outer"]).all()
    for m in (0, 1):
        a, b = got["factors"][m], ref["factors"][m]
        assert a.shape == b.shape
        assert a.min() >= 0.0
        assert np.abs(a - b).max() <= 1e-9 * max(np.abs(b).max(), 1.0)
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= 1e-9


def test_stream_nonneg_fp32_fit_within_1e4(lib64, port):
    inds, vals, dims = _data(seed=8, T=10)
    got = lib64.stream_run(inds, vals, dims, 2, 16, seed=4, precision=sb.FP32,
                           exec_=sb.FUSED, errs=True, nonneg=True)
    ref = port.stream(inds, vals, dims, 2, 16, seed=4, nonneg=True)
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= 1e-4
    for m in (0, 1):
        assert got["factors"][m].min() >= 0.0


def test_stream_set_prox_rejects(lib64):
    st = sb.Stream(lib64, 3, 2, [10, 10, 4], 8)
    with pytest.raises(sb.SplattError):
        st.set_prox(2, sb.PROX_MAXCOLNORM_NONNEG)      # the streamed mode
    with pytest.raises(sb.SplattError):
        st.set_prox(0, 7)
    with pytest.raises(sb.SplattError):
        st.set_prox(0, sb.PROX_LASSO, -1.0)
    st.set_prox(1, sb.PROX_MAXCOLNORM_NONNEG)
    st.free()


def _cpd_stream_file(lib, path, rank, sm, seed, nonneg, frob_on_time=True):
    """splatt_cpd_stream on a .tns with `--con=nonneg` / `--reg=frob,1e-2,sm`
    registered as the reference's CLI registers them; returns the status."""
    import ctypes as C
    L, it = lib.L, lib.it
    L.splatt_cpd_stream.argtypes = [C.c_char_p, it, it, C.c_double,
                                    C.POINTER(lib.CpdOpts), C.c_void_p]
    L.splatt_cpd_stream.restype = C.c_int
    L.splatt_register_frob.argtypes = [C.POINTER(lib.CpdOpts), lib.vt, C.POINTER(it), it]
    L.splatt_register_nonneg.argtypes = [C.POINTER(lib.CpdOpts), C.POINTER(it), it]
    L.splatt_alloc_global_opts.restype = C.c_void_p
    L.splatt_free_global_opts.argtypes = [C.c_void_p]
    o = L.splatt_alloc_cpd_opts()
    o.contents.max_iterations = 200
    if nonneg:
        L.splatt_register_nonneg(o, (it * 8)(*range(8)), 8)
    if frob_on_time:
        L.splatt_register_frob(o, 1e-2, (it * 1)(sm), 1)
    g = L.splatt_alloc_global_opts()
    (C.c_int * 3).from_address(g)[2] = seed            # random_seed
    try:
        return L.splatt_cpd_stream(str(path).encode(), rank, sm, 0.95, o, g)
    finally:
        L.splatt_free_cpd_opts(o)
        L.splatt_free_global_opts(g)


def test_cpd_stream_file_nonneg(lib64, port, tmp_path, monkeypatch):
    """splatt_cpd_stream maps NON-NEGATIVE on the non-streamed modes to the
    non-negative max-column-norm (StreamCPD.cc:325-337): mode%d.mat matches
    the oracle in the original row order; without it the factors keep
    negative entries; NON-NEGATIVE left on the streamed mode is refused."""
    inds, vals, dims = _data(seed=9, T=6)
    f = tmp_path / "x.tns"
    with open(f, "w") as fh:
        for n in range(len(vals)):
            fh.write("%d %d %d %.17g\n" % (inds[0][n] + 1, inds[1][n] + 1, inds[2][n] + 1,
                                           vals[n]))
    monkeypatch.chdir(tmp_path)
    R = 8
    assert _cpd_stream_file(lib64, f, R, 2, 11, False) == sb.SPLATT_SUCCESS
    plain = [np.loadtxt("mode%d.mat" % (m + 1)) for m in (0, 1)]
    assert min(x.min() for x in plain) < 0.0
    assert _cpd_stream_file(lib64, f, R, 2, 11, True) == sb.SPLATT_SUCCESS
    got = [np.loadtxt("mode%d.mat" % (m + 1)) for m in (0, 1)]
    ref = port.stream(inds, vals, dims, 2, R, seed=11, nonneg=True)
    _, _, _, iperm = sb.parse_stream(inds, vals, dims, 2)
    for m in (0, 1):
        b = ref["factors"][m]
        a = got[m][iperm[m][:len(b)].astype(np.int64)]
        assert got[m].min() >= 0.0
        # mode%d.mat is printed with 9 significant digits
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)
    assert _cpd_stream_file(lib64, f, R, 2, 11, True, frob_on_time=False) != sb.SPLATT_SUCCESS


@pytest.mark.parametrize("exec_", [sb.PLAIN, sb.FUSED])
@pytest.mark.parametrize("R", [8, 48])
def test_stream_lasso_fp64_matches_oracle(lib64, port, exec_, R):
    """`--reg=l1,0.01`.  The multiplier leaves 13-61% of the factor entries
    at zero on this tensor (larger ones zero everything, which would test
    nothing; the test checks for both cases).  Tolerance 1e-8 here (1e-9
    for the column-norm proxes): the threshold's on/off decisions near
    |p| = lambda / rho amplify the last-bit difference between the kernel's
    solve (explicit inverse of G + rho I) and the oracle's Cholesky solve."""
    tol = 1e-8
    inds, vals, dims = _data(seed=10, T=8)
    got = lib64.stream_run(inds, vals, dims, 2, R, seed=17, exec_=exec_, errs=True, lasso=0.01)
    ref = port.stream(inds, vals, dims, 2, R, seed=17, lasso=0.01)
    scale = np.abs(ref["time"]).max()
    assert scale > 0.0
    assert np.abs(got["time"] - ref["time"]).max() <= tol * scale
    assert (got["outer"] == ref["outer"]).all()
    nz, total = 0, 0
    for m in (0, 1):
        a, b = got["factors"][m], ref["factors"][m]
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1.0)
        nz += int((b == 0.0).sum())
        total += b.size
    assert 0 < nz < total                            # active, not degenerate
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= tol


def test_stream_lasso_fp32_fit_within_1e4(lib64, port):
    inds, vals, dims = _data(seed=12, T=8)
    got = lib64.stream_run(inds, vals, dims, 2, 16, seed=6, precision=sb.FP32,
                           exec_=sb.FUSED, errs=True, lasso=0.01)
    ref = port.stream(inds, vals, dims, 2, 16, seed=6, lasso=0.01)
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= 1e-4


def test_cpd_stream_file_lasso(lib64, port, tmp_path, monkeypatch):
    """`--reg=l1,0.01 --reg=frob,1e-2,3` through splatt_cpd_stream."""
    import ctypes as C
    inds, vals, dims = _data(seed=14, T=6)
    f = tmp_path / "x.tns"
    with open(f, "w") as fh:
        for n in range(len(vals)):
            fh.write("%d %d %d %.17g\n" % (inds[0][n] + 1, inds[1][n] + 1, inds[2][n] + 1,
                                            vals[n]))
    monkeypatch.chdir(tmp_path)
    L, it = lib64.L, lib64.it
    L.splatt_register_lasso.argtypes = [C.POINTER(lib64.CpdOpts), lib64.vt, C.POINTER(it), it]
    L.splatt_register_frob.argtypes = [C.POINTER(lib64.CpdOpts), lib64.vt, C.POINTER(it), it]
    L.splatt_cpd_stream.argtypes = [C.c_char_p, it, it, C.c_double,
                                    C.POINTER(lib64.CpdOpts), C.c_void_p]
    L.splatt_cpd_stream.restype = C.c_int
    L.splatt_alloc_global_opts.restype = C.c_void_p
    L.splatt_free_global_opts.argtypes = [C.c_void_p]
    o = L.splatt_alloc_cpd_opts()
    o.contents.max_iterations = 200
    L.splatt_register_lasso(o, 0.01, (it * 8)(*range(8)), 8)
    L.splatt_register_frob(o, 1e-2, (it * 1)(2), 1)
    g = L.splatt_alloc_global_opts()
    (C.c_int * 3).from_address(g)[2] = 11
    try:
        assert L.splatt_cpd_stream(str(f).encode(), 8, 2, 0.95, o, g) == sb.SPLATT_SUCCESS
    finally:
        L.splatt_free_cpd_opts(o)
        L.splatt_free_global_opts(g)
    ref = port.stream(inds, vals, dims, 2, 8, seed=11, lasso=0.01)
    assert np.abs(ref["time"]).max() > 0.0
    _, _, _, iperm = sb.parse_stream(inds, vals, dims, 2)
    for m in (0, 1):
        got = np.loadtxt("mode%d.mat" % (m + 1))
        b = ref["factors"][m]
        a = got[iperm[m][:len(b)].astype(np.int64)]
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)


@pytest.mark.parametrize("sm", [0, 1, 2])
def test_cpd_stream_file_device_ingest(lib64, port, tmp_path, monkeypatch, sm):
    """splatt_cpd_stream prepares the stream on the device (order by time then
    the following modes, first-appearance relabel, slice bounds): with the
    time mode first, in the middle and last, mode%d.mat and the time factor
    match the oracle, which prepares it like ParserSimple."""
    inds, vals, dims = _data(seed=15, T=7)
    perm = {0: [2, 0, 1], 1: [0, 2, 1], 2: [0, 1, 2]}[sm]
    pi = [inds[p] for p in perm]
    pd = dims[perm]
    f = tmp_path / "x.tns"
    with open(f, "w") as fh:
        for n in range(len(vals)):
            fh.write(" ".join(str(int(x[n]) + 1) for x in pi) + " %.17g\n" % vals[n])
    monkeypatch.chdir(tmp_path)
    assert _cpd_stream_file(lib64, f, 8, sm, 21, False) == sb.SPLATT_SUCCESS
    ref = port.stream(pi, vals, pd, sm, 8, seed=21)
    _, _, _, iperm = sb.parse_stream(pi, vals, pd, sm)
    for m in range(3):
        got = np.loadtxt("mode%d.mat" % (m + 1))
        if m == sm:
            b = ref["time"]
            a = got[:len(b)]
        else:
            b = ref["factors"][m]
            a = got[iperm[m][:len(b)].astype(np.int64)]
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0), m


@pytest.mark.parametrize("exec_", [sb.PLAIN, sb.FUSED])
@pytest.mark.parametrize("R", [8, 48])
def test_stream_rowsimp_fp64_matches_oracle(lib64, port, exec_, R):
    """`--con=rowsimp`: each non-streamed factor row projected onto the
    probability simplex (simplex.cc:34-66), ADMM in 50-row chunks.

    Tolerance 1e-8 here (1e-9 elsewhere): the projection's threshold is a
    difference of running sums that cancels, so the last-bit difference
    between the kernel's solve (explicit inverse of G + rho I) and the
    oracle's Cholesky solve grows over the chunk iterations; at R = 48 the
    two differ by ~1.2e-9 (measured), with identical iteration counts."""
    tol = 1e-8
    inds, vals, dims = _data(seed=16, T=6)
    got = lib64.stream_run(inds, vals, dims, 2, R, seed=19, exec_=exec_, errs=True, rowsimp=True)
    ref = port.stream(inds, vals, dims, 2, R, seed=19, rowsimp=True)
    scale = np.abs(ref["time"]).max()
    assert np.abs(got["time"] - ref["time"]).max() <= tol * scale
    assert (got["outer"] == ref["outer"]).all()
    for m in (0, 1):
        a, b = got["factors"][m], ref["factors"][m]
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1.0)
        assert a.min() >= 0.0 and np.abs(a.sum(axis=1) - 1.0).max() <= 1e-9
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= tol


NTF = {"ntf_lasso": (16, 0.01), "ntf_frob": (18, 0.1)}


@pytest.mark.parametrize("exec_", [sb.PLAIN, sb.FUSED])
@pytest.mark.parametrize("R", [8, 48])
@pytest.mark.parametrize("con", list(NTF))
def test_stream_ntf_fp64_matches_oracle(lib64, port, exec_, R, con):
    """`--reg=ntf-l1,0.01` (nonneg_lasso.c:30-45: v > L/rho ? v - L/rho : 0)
    and `--reg=ntf-frob,0.1` (nonneg_frob.c:31-49: max(v rho / (L + rho),
    0)), both row-separable, ADMM in 50-row chunks.  The multipliers leave
    5-75% of the factor entries at zero on these tensors (ntf-l1 at 0.1 and
    ntf-frob at 1.0 zero nearly all).  Tolerance 1e-8, as for lasso: the
    prox's on/off decisions at the threshold amplify the last-bit difference
    between the kernel's solve and the oracle's Cholesky solve."""
    tol = 1e-8
    seed, mult = NTF[con]
    kw = {con: mult}
    inds, vals, dims = _data(seed=seed, T=8)
    got = lib64.stream_run(inds, vals, dims, 2, R, seed=17, exec_=exec_, errs=True, **kw)
    ref = port.stream(inds, vals, dims, 2, R, seed=17, **kw)
    scale = np.abs(ref["time"]).max()
    assert scale > 0.0
    assert np.abs(got["time"] - ref["time"]).max() <= tol * scale
    assert (got["outer"] == ref["outer"]).all()
    nz, total = 0, 0
    for m in (0, 1):
        a, b = got["factors"][m], ref["factors"][m]
        assert a.shape == b.shape
        assert a.min() >= 0.0
        assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1.0)
        nz += int((b == 0.0).sum())
        total += b.size
    assert 0 < nz < total                            # active, not degenerate
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= tol


def test_cpd_stream_file_ntf_frob(lib64, port, tmp_path, monkeypatch):
    """`--reg=ntf-frob,0.1 --reg=frob,1e-2,3` through splatt_cpd_stream: the
    NTF registration (described "NTF-L1-REG", like ntf-l1's) maps to the
    NTF-Frobenius prox on the non-streamed modes."""
    import ctypes as C
    inds, vals, dims = _data(seed=18, T=6)
    f = tmp_path / "x.tns"
    with open(f, "w") as fh:
        for n in range(len(vals)):
            fh.write("%d %d %d %.17g\n" % (inds[0][n] + 1, inds[1][n] + 1, inds[2][n] + 1,
                                            vals[n]))
    monkeypatch.chdir(tmp_path)
    L, it = lib64.L, lib64.it
    L.splatt_register_ntf_frob.argtypes = [C.POINTER(lib64.CpdOpts), lib64.vt, C.POINTER(it), it]
    L.splatt_register_frob.argtypes = [C.POINTER(lib64.CpdOpts), lib64.vt, C.POINTER(it), it]
    L.splatt_cpd_stream.argtypes = [C.c_char_p, it, it, C.c_double,
                                    C.POINTER(lib64.CpdOpts), C.c_void_p]
    L.splatt_cpd_stream.restype = C.c_int
    L.splatt_alloc_global_opts.restype = C.c_void_p
    L.splatt_free_global_opts.argtypes = [C.c_void_p]
    o = L.splatt_alloc_cpd_opts()
    o.contents.max_iterations = 200
    L.splatt_register_ntf_frob(o, 0.1, (it * 8)(*range(8)), 8)
    L.splatt_register_frob(o, 1e-2, (it * 1)(2), 1)
    g = L.splatt_alloc_global_opts()
    (C.c_int * 3).from_address(g)[2] = 11
    try:
        assert L.splatt_cpd_stream(str(f).encode(), 8, 2, 0.95, o, g) == sb.SPLATT_SUCCESS
    finally:
        L.splatt_free_cpd_opts(o)
        L.splatt_free_global_opts(g)
    ref = port.stream(inds, vals, dims, 2, 8, seed=11, ntf_frob=0.1)
    assert np.abs(ref["time"]).max() > 0.0
    _, _, _, iperm = sb.parse_stream(inds, vals, dims, 2)
    for m in (0, 1):
        got = np.loadtxt("mode%d.mat" % (m + 1))
        b = ref["factors"][m]
        a = got[iperm[m][:len(b)].astype(np.int64)]
        assert a.min() >= 0.0
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)


def test_stream_window_errors_match_oracle(lib64, port):
    """splatt_b200_stream_window_errsq (the driver's "global" / "local-10"
    figures, StreamCPD.cc:77-86) after the last slice, for windows of 1, 10,
    all and more than all slices, against the oracle's restatement
    (orc_stream_window_errsq) at 1e-9; a window of one slice equals the
    per-slice local error."""
    import ctypes as C
    import torch
    inds, vals, dims = _data(seed=12, T=24)
    si, sv, offs, _ = sb.parse_stream(inds, vals, dims, 2)
    T = len(offs) - 1
    sb.srand(5)
    st = sb.Stream(lib64, 3, 2, dims, 16, exec_=sb.FUSED)
    for t in range(T):
        a, b = int(offs[t]), int(offs[t + 1])
        st.push([x[a:b] for x in si], sv[a:b])
    local1 = st.local_errsq()
    facs = st.factors(T)
    dind = [torch.from_numpy(x.astype(np.int32)).cuda() for x in si]
    dval = torch.from_numpy(np.ascontiguousarray(sv, dtype=np.float64)).cuda()
    f = lib64.L.splatt_b200_stream_window_errsq
    f.argtypes = [C.c_void_p, lib64.it, C.POINTER(C.c_void_p), C.c_void_p, lib64.it]
    f.restype = C.c_double
    torch.cuda.synchronize()
    for k in (1, 10, T, 3 * T):
        w0 = max(0, T - k)
        lo, hi = int(offs[w0]), int(offs[T])
        ptrs = (C.c_void_p * 3)(*[x.data_ptr() + 4 * lo for x in dind])
        got = f(C.c_void_p(st.h), hi - lo, ptrs, C.c_void_p(dval.data_ptr() + 8 * lo), k)
        want = port.window_errsq(inds, vals, dims, 2, facs[2], facs[:2], k)
        assert got >= 0.0 and abs(got - want) <= 1e-9, (k, got, want)
        if k == 1:
            assert abs(got - local1) <= 1e-12
    st.free()


@pytest.mark.parametrize("exec_", [sb.PLAIN, sb.FUSED])
@pytest.mark.parametrize("R", [8, 40])
def test_stream_colsimp_fp64_matches_oracle(lib64, port, exec_, R):
    """`--con=colsimp`: each non-streamed factor's columns projected onto the
    probability simplex inside a single-chunk ADMM (simplex.cc:113-150), the
    threshold of every column found by grid-wide rounds.  Time rows and
    factors within 1e-8 relative of the oracle (the projection's support
    decisions at the threshold amplify the last-bit differences of the
    solve, as for the other threshold proxes), identical outer-iteration
    counts; every column of the final factors is non-negative and sums
    to 1.  At rank 40 the same amplification separates the oracle from the
    compiled reference itself by 9.8e-8 relative on this stream (its last
    slice: 1.2e-5 absolute), so the bar there is 5e-7."""
    inds, vals, dims = _data(seed=15, T=8)
    got = lib64.stream_run(inds, vals, dims, 2, R, seed=19, exec_=exec_, errs=True, colsimp=True)
    ref = port.stream(inds, vals, dims, 2, R, seed=19, colsimp=True)
    tol = 1e-8 if R <= 8 else 5e-7
    assert np.abs(got["time"] - ref["time"]).max() <= tol * np.abs(ref["time"]).max()
    assert (got["outer"] == ref["outer"]).all()
    for m in (0, 1):
        a, b = got["factors"][m], ref["factors"][m]
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1.0)
        assert a.min() >= 0.0
        assert np.abs(a.sum(axis=0) - 1.0).max() <= 1e-9
    assert np.abs(got["local_errsq"] - ref["local_errsq"]).max() <= \
        tol * max(1.0, np.abs(ref["local_errsq"]).max())


def test_cpd_stream_file_colsimp(lib64, port, tmp_path, monkeypatch):
    """`splatt cpd x.tns --stream=3 --con=colsimp --reg=frob,1e-2,3` through
    splatt_cpd_stream: mode%d.mat matches the oracle in the original row
    order (printed with 9 significant digits)."""
    import ctypes as C
    inds, vals, dims = _data(seed=16, T=6)
    f = tmp_path / "x.tns"
    with open(f, "w") as fh:
        for n in range(len(vals)):
            fh.write("%d %d %d %.17g\n" % (inds[0][n] + 1, inds[1][n] + 1, inds[2][n] + 1,
                                            vals[n]))
    monkeypatch.chdir(tmp_path)
    L, it = lib64.L, lib64.it
    L.splatt_register_colsimp.argtypes = [C.POINTER(lib64.CpdOpts), C.POINTER(it), it]
    L.splatt_register_frob.argtypes = [C.POINTER(lib64.CpdOpts), lib64.vt, C.POINTER(it), it]
    L.splatt_cpd_stream.argtypes = [C.c_char_p, it, it, C.c_double,
                                    C.POINTER(lib64.CpdOpts), C.c_void_p]
    L.splatt_cpd_stream.restype = C.c_int
    L.splatt_alloc_global_opts.restype = C.c_void_p
    L.splatt_free_global_opts.argtypes = [C.c_void_p]
    o = L.splatt_alloc_cpd_opts()
    o.contents.max_iterations = 200
    L.splatt_register_colsimp(o, (it * 8)(*range(8)), 8)
    L.splatt_register_frob(o, 1e-2, (it * 1)(2), 1)
    g = L.splatt_alloc_global_opts()
    (C.c_int * 3).from_address(g)[2] = 11
    try:
        assert L.splatt_cpd_stream(str(f).encode(), 8, 2, 0.95, o, g) == sb.SPLATT_SUCCESS
    finally:
        L.splatt_free_cpd_opts(o)
        L.splatt_free_global_opts(g)
    ref = port.stream(inds, vals, dims, 2, 8, seed=11, colsimp=True)
    _, _, _, iperm = sb.parse_stream(inds, vals, dims, 2)
    for m in (0, 1):
        got = np.loadtxt("mode%d.mat" % (m + 1))
        b = ref["factors"][m]
        a = got[iperm[m][:len(b)].astype(np.int64)]
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)
