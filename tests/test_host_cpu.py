"""Host logic of the C ABI that decides before any device call, run without a
GPU: the tiling schemes splatt_csf_convert refuses, the NTF registrations,
and the constraint mapping of splatt_cpd_stream (StreamCPD.cc:325-337) for
what it refuses: ADMM constraints on the streamed mode, constraints with no
streaming counterpart, a missing file."""
import ctypes as C

import numpy as np
import pytest

import splatt_b200 as sb


@pytest.fixture(scope="module")
def lib():
    return sb.Lib(64)                 # loaded, never initialised on a device


def test_csf_convert_refuses_unbuilt_tile_schemes(lib):
    inds = [np.array([0, 1, 2], np.uint64), np.array([1, 0, 2], np.uint64),
            np.array([2, 2, 0], np.uint64)]
    vals = np.array([1.0, 2.0, 3.0])
    for scheme in (2, 3):                              # SYNCTILE, COOPTILE
        opts = lib.opts(csf_alloc=sb.CSF_ALLMODE)
        opts[sb.OPT["TILE"]] = float(scheme)
        keep, arr = lib._idx_ptrs(inds)
        out = C.POINTER(lib.Csf)()
        rc = lib.L.splatt_csf_convert(lib.it(3), lib.it(3), arr,
                                      vals.ctypes.data_as(C.POINTER(lib.vt)), C.byref(out), opts)
        assert rc == sb.SPLATT_ERROR_BADINPUT, scheme


def _stream_call(lib, path, register):
    L, it = lib.L, lib.it
    L.splatt_cpd_stream.argtypes = [C.c_char_p, it, it, C.c_double, C.POINTER(lib.CpdOpts),
                                    C.c_void_p]
    L.splatt_cpd_stream.restype = C.c_int
    o = L.splatt_alloc_cpd_opts()
    try:
        register(L, o, it)
        return L.splatt_cpd_stream(str(path).encode(), 4, 2, 0.95, o, None)
    finally:
        L.splatt_free_cpd_opts(o)


@pytest.fixture
def tns(tmp_path):
    f = tmp_path / "t.tns"
    f.write_text("1 1 1 1.0\n2 1 1 2.0\n1 2 2 3.0\n2 2 2 4.0\n")
    return f


def test_cpd_stream_refuses_admm_constraint_on_streamed_mode(lib, tns):
    def reg(L, o, it):
        L.splatt_register_nonneg.argtypes = [C.POINTER(lib.CpdOpts), C.POINTER(it), it]
        L.splatt_register_nonneg(o, (it * 1)(2), 1)
    assert _stream_call(lib, tns, reg) == sb.SPLATT_ERROR_BADINPUT


def test_cpd_stream_refuses_frob_on_non_streamed_mode(lib, tns):
    def reg(L, o, it):
        L.splatt_register_frob.argtypes = [C.POINTER(lib.CpdOpts), lib.vt, C.POINTER(it), it]
        L.splatt_register_frob(o, 1e-2, (it * 1)(0), 1)
    assert _stream_call(lib, tns, reg) == sb.SPLATT_ERROR_BADINPUT


def test_cpd_stream_refuses_unknown_constraint(lib, tns):
    def reg(L, o, it):
        L.splatt_alloc_constraint.restype = C.c_void_p
        L.splatt_alloc_constraint.argtypes = [C.c_int]
        L.splatt_register_constraint.argtypes = [C.POINTER(lib.CpdOpts), it, C.c_void_p]
        c = L.splatt_alloc_constraint(1)                 # SPLATT_CON_ADMM
        con_t = dict(lib.CpdOpts._fields_)["constraints"]._type_._type_
        C.cast(c, C.POINTER(con_t)).contents.description = b"SMOOTH-COL (1.0e-02)"
        L.splatt_register_constraint(o, 1, c)
    assert _stream_call(lib, tns, reg) == sb.SPLATT_ERROR_BADINPUT


def test_cpd_stream_refuses_missing_file(lib, tmp_path):
    assert _stream_call(lib, tmp_path / "none.tns", lambda L, o, it: None) == \
        sb.SPLATT_ERROR_BADINPUT


def test_ntf_registrations(lib):
    """splatt_register_ntf_lasso / _ntf_frob (nonneg_lasso.c:67-100,
    nonneg_frob.c:74-105): ADMM, row-separable, the multiplier in `data`, both
    described "NTF-L1-REG (L)" as in the reference, told apart by their prox
    function."""
    L, it = lib.L, lib.it
    for f in (L.splatt_register_ntf_lasso, L.splatt_register_ntf_frob):
        f.argtypes = [C.POINTER(lib.CpdOpts), lib.vt, C.POINTER(it), it]
        f.restype = C.c_int
    o = L.splatt_alloc_cpd_opts()
    try:
        assert L.splatt_register_ntf_lasso(o, 0.01, (it * 1)(0), 1) == sb.SPLATT_SUCCESS
        assert L.splatt_register_ntf_frob(o, 0.25, (it * 1)(1), 1) == sb.SPLATT_SUCCESS
        a, b = o.contents.constraints[0].contents, o.contents.constraints[1].contents
        for c, mult in ((a, 0.01), (b, 0.25)):
            assert c.solve_type == 1 and c.row_separable
            assert c.description == ("NTF-L1-REG (%0.1e)" % mult).encode()
            assert C.cast(c.data, C.POINTER(lib.vt))[0] == mult
        assert a.prox and b.prox and a.prox != b.prox
    finally:
        L.splatt_free_cpd_opts(o)


def test_cpd_stream_refuses_ntf_on_streamed_mode(lib, tns):
    def reg(L, o, it):
        L.splatt_register_ntf_frob.argtypes = [C.POINTER(lib.CpdOpts), lib.vt, C.POINTER(it), it]
        L.splatt_register_ntf_frob(o, 0.1, (it * 1)(2), 1)
    assert _stream_call(lib, tns, reg) == sb.SPLATT_ERROR_BADINPUT


def test_colsimp_and_smooth_register_and_smooth_is_refused(lib, tns):
    """splatt_register_colsimp / _smooth (SPLATT's cpd.h:297-300, 349-353)
    register with SPLATT's descriptions; splatt_cpd_stream refuses smooth on
    a non-streamed mode before any device work (the reference's streaming
    driver leaves smooth's workspace uninitialised)."""
    L, it = lib.L, lib.it
    L.splatt_register_colsimp.argtypes = [C.POINTER(lib.CpdOpts), C.POINTER(it), it]
    L.splatt_register_smooth.argtypes = [C.POINTER(lib.CpdOpts), lib.vt, C.POINTER(it), it]
    o = L.splatt_alloc_cpd_opts()
    try:
        assert L.splatt_register_colsimp(o, (it * 1)(0), 1) == sb.SPLATT_SUCCESS
        assert L.splatt_register_smooth(o, 0.5, (it * 1)(1), 1) == sb.SPLATT_SUCCESS
        a, b = o.contents.constraints[0].contents, o.contents.constraints[1].contents
        assert a.description == b"COL-SIMPLEX" and not a.row_separable
        assert b.description == b"SMOOTH-COL (5.0e-01)"
        assert C.cast(b.data, C.POINTER(lib.vt))[0] == 0.5
    finally:
        L.splatt_free_cpd_opts(o)
    def reg(L, o, it):
        L.splatt_register_smooth(o, 0.5, (it * 1)(0), 1)
    assert _stream_call(lib, tns, reg) == sb.SPLATT_ERROR_BADINPUT


def test_version_and_default_opts(lib):
    """The reference's API tests (tests/api_test.c:38-89): the version is
    SPLATT's 2.0.0; the option defaults are SPLATT's (src/opts.c:14-75) with
    one thread, the value SPLATT itself gives inside a parallel region."""
    L = lib.L
    for f in (L.splatt_version_major, L.splatt_version_minor, L.splatt_version_subminor):
        f.restype = C.c_int
    assert (L.splatt_version_major(), L.splatt_version_minor(),
            L.splatt_version_subminor()) == (2, 0, 0)
    o = L.splatt_default_opts()
    try:
        assert o[sb.OPT["TOLERANCE"]] == 1e-5 and o[sb.OPT["NITER"]] == 50
        assert o[sb.OPT["CSF_ALLOC"]] == sb.CSF_TWOMODE and o[sb.OPT["TILE"]] == sb.NOTILE
        assert o[sb.OPT["TILELEVEL"]] == 1 and o[sb.OPT["PRIVTHRESH"]] == 0.02
        assert o[sb.OPT["NTHREADS"]] == 1
    finally:
        L.splatt_free_opts(o)


def _bin(path, dims, inds, vals, nnz=None, iw=8, vw=8):
    """A .bin tensor (src/io.c:388-474 layout: int32 magic 0, idx width, val
    width, nmodes, dims, nnz, the index arrays mode by mode, the values);
    `nnz` overrides the stored count."""
    it = np.uint64 if iw == 8 else np.uint32
    with open(path, "wb") as f:
        f.write(np.int32(0).tobytes())
        f.write(np.array([iw, vw], np.uint64).tobytes())
        f.write(np.array([len(dims)], it).tobytes())
        f.write(np.array(dims, it).tobytes())
        f.write(np.array([len(vals) if nnz is None else nnz], it).tobytes())
        for x in inds:
            f.write(np.asarray(x, it).tobytes())
        f.write(np.asarray(vals, np.float64 if vw == 8 else np.float32).tobytes())


def _load(lib, path):
    L = lib.L
    L.splatt_coord_load.argtypes = [C.c_char_p, C.POINTER(lib.Coord)]
    L.splatt_coord_load.restype = C.c_int
    c = lib.Coord()
    return L.splatt_coord_load(str(path).encode(), C.byref(c)), c


def test_coord_load_binary_and_its_refusals(lib, tmp_path):
    """The binary reader (src/io.c:118-196 layout) loads a well-formed file at
    both widths, and refuses, without reading past its buffers, a count
    larger than the file holds (one that would overflow the allocation size
    among them), a truncated payload, and an index outside its dimension."""
    dims = [4, 3, 5]
    inds = [np.array([0, 3, 1]), np.array([2, 0, 1]), np.array([4, 4, 0])]
    vals = np.array([1.5, -2.0, 0.25])
    for iw, vw in ((8, 8), (4, 4)):
        p = tmp_path / ("ok%d.bin" % iw)
        _bin(p, dims, inds, vals, iw=iw, vw=vw)
        rc, c = _load(lib, p)
        assert rc == sb.SPLATT_SUCCESS and c.nnz == 3 and list(c.dims[:3]) == dims
        for m in range(3):
            assert np.ctypeslib.as_array(c.ind[m], (3,)).tolist() == inds[m].tolist()
        assert np.ctypeslib.as_array(c.vals, (3,)).tolist() == vals.tolist()
    bad = tmp_path / "bad.bin"
    for nnz in (1 << 62, (1 << 61) + 1, 4):            # more than the payload holds
        _bin(bad, dims, inds, vals, nnz=nnz)
        assert _load(lib, bad)[0] == sb.SPLATT_ERROR_BADINPUT, nnz
    _bin(bad, dims, [x[:2] for x in inds], vals[:2], nnz=3)  # truncated
    assert _load(lib, bad)[0] == sb.SPLATT_ERROR_BADINPUT
    out = [inds[0], np.array([2, 3, 1]), inds[2]]             # 3 >= dims[1]
    _bin(bad, dims, out, vals)
    assert _load(lib, bad)[0] == sb.SPLATT_ERROR_BADINPUT


@pytest.mark.parametrize("nmodes,sm", [(3, 2), (3, 0), (3, 1), (4, 1), (4, 3)])
def test_parse_stream_matches_oracle(port, nmodes, sm):
    """The Python mirror's host preparation of a stream (parse_stream) equals
    the oracle's ParserSimple restatement (ParserSimple.cc:13-79): order,
    first-appearance labels and values, exactly; its slice offsets bound each
    time index and its iperm maps labels back to the original indices."""
    rng = np.random.default_rng(100 + 10 * nmodes + sm)
    dims = np.array([37, 23, 11, 9][:nmodes], np.uint64)
    dims[sm] = 6
    n = 400
    coords = set()
    while len(coords) < n:                              # distinct coordinates
        coords.add(tuple(int(rng.integers(0, int(d))) for d in dims))
    coords = sorted(coords, key=lambda c: rng.random())
    inds = [np.array([c[m] for c in coords], np.uint64) for m in range(nmodes)]
    vals = rng.lognormal(size=n)
    s_inds, s_vals, offs, iperm = sb.parse_stream(inds, vals, dims, sm)
    o_inds, o_vals = port.stream_prepare(inds, vals, dims, sm)
    for m in range(nmodes):
        assert np.array_equal(s_inds[m], o_inds[m]), m
    assert np.array_equal(s_vals, o_vals)
    t = s_inds[sm]
    for k in range(len(offs) - 1):
        assert (t[offs[k]:offs[k + 1]] == k).all()
    # iperm[m][label] is the original index: the relabelled tensor maps back
    order = np.lexsort([inds[(sm + k) % nmodes] for k in range(nmodes)][::-1])
    for m in range(nmodes):
        if m != sm:
            assert np.array_equal(iperm[m][s_inds[m].astype(np.int64)], inds[m][order]), m


def test_csf_convert_and_load_refuse_bad_shapes(lib, tmp_path):
    """splatt_csf_convert / splatt_csf_load refuse, before any device call:
    fewer than 2 or more than 8 modes, no nonzeros, missing pointers, a
    missing or empty file (SPLATT_ERROR_BADINPUT)."""
    L = lib.L
    inds = [np.array([0, 1], np.uint64) for _ in range(9)]
    vals = np.array([1.0, 2.0])
    keep, arr = lib._idx_ptrs(inds)
    vp = vals.ctypes.data_as(C.POINTER(lib.vt))
    opts = lib.opts()
    out = C.POINTER(lib.Csf)()
    for nmodes, nnz in ((1, 2), (9, 2), (3, 0)):
        assert L.splatt_csf_convert(lib.it(nmodes), lib.it(nnz), arr, vp, C.byref(out),
                                    opts) == sb.SPLATT_ERROR_BADINPUT, (nmodes, nnz)
    assert L.splatt_csf_convert(lib.it(3), lib.it(2), None, vp, C.byref(out),
                                opts) == sb.SPLATT_ERROR_BADINPUT
    assert L.splatt_csf_convert(lib.it(3), lib.it(2), arr, vp, C.byref(out),
                                None) == sb.SPLATT_ERROR_BADINPUT
    L.splatt_csf_load.argtypes = [C.c_char_p, C.POINTER(lib.it), C.POINTER(C.POINTER(lib.Csf)),
                                  C.POINTER(C.c_double)]
    L.splatt_csf_load.restype = C.c_int
    n = lib.it()
    empty = tmp_path / "empty.tns"
    empty.write_text("# nothing\n")
    for path in (tmp_path / "none.tns", empty):
        assert L.splatt_csf_load(str(path).encode(), C.byref(n), C.byref(out),
                                 opts) == sb.SPLATT_ERROR_BADINPUT, path


def test_cpd_stream_refuses_rank_out_of_range(lib, tns):
    """The streaming kernels take ranks 1..64: splatt_cpd_stream refuses
    others up front with SPLATT_ERROR_BADINPUT (not an allocation error)."""
    L, it = lib.L, lib.it
    L.splatt_cpd_stream.argtypes = [C.c_char_p, it, it, C.c_double, C.POINTER(lib.CpdOpts),
                                    C.c_void_p]
    L.splatt_cpd_stream.restype = C.c_int
    for rank in (0, 65, 1000):
        assert L.splatt_cpd_stream(str(tns).encode(), rank, 2, 0.95, None,
                                   None) == sb.SPLATT_ERROR_BADINPUT, rank
