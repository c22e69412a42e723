"""Tensor files read onto the device (sb_read_tensor_device: text parsed by
the device, binary widths converted there) against the host reader
(splatt_coord_load, which restates tt_read, src/io.c:62-196): the same mode
count, dims, nonzero count, 0-based indices and values, bit for bit, on
files that exercise the text format's corners -- comment and blank lines,
1- and 0-indexed modes, a last line without newline, CRLF line ends, the
reference's own "%f" values, 17-digit and exponent forms, signs -- and on
binary files of both index and value widths.  Lines the device cannot parse
exactly go to the host, so the result is exact either way.

Then the same files through splatt_csf_load (device read, empty slices
dropped on the device, CSF built there): the CSF equals the oracle's CSF of
the host-read tensor after tt_remove_empty."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

import splatt_b200 as sb

pytestmark = pytest.mark.gpu


def _read_device(lib, path):
    L, it = lib.L, lib.it
    f = L.sb_read_tensor_device
    f.argtypes = [C.c_char_p, C.POINTER(it), C.POINTER(it), C.POINTER(it),
                  C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    f.restype = C.c_int
    L.sb_d2h.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    L.sb_free.argtypes = [C.c_void_p]
    n, nnz = it(), it()
    dims = (it * 8)()
    dinds = (C.c_void_p * 8)()
    dval = C.c_void_p()
    rc = f(str(path).encode(), C.byref(n), C.byref(nnz), dims, dinds, C.byref(dval))
    if rc != 0:
        return rc, None
    N, Z = int(n.value), int(nnz.value)
    inds = []
    for m in range(N):
        h = np.zeros(Z, np.uint32)
        assert L.sb_d2h(h.ctypes.data, dinds[m], Z * 4) == 0
        inds.append(h.astype(np.uint64))
        L.sb_free(dinds[m])
    v = np.zeros(Z, lib.val_dtype)
    assert L.sb_d2h(v.ctypes.data, dval, Z * v.itemsize) == 0
    L.sb_free(dval)
    return 0, dict(inds=inds, vals=v, dims=[int(dims[m]) for m in range(N)])


def _read_host(lib, path):
    Coord = sb.coord_struct(64)
    L = lib.L
    L.splatt_coord_load.argtypes = [C.c_char_p, C.POINTER(Coord)]
    L.splatt_coord_load.restype = C.c_int
    c = Coord()
    assert L.splatt_coord_load(str(path).encode(), C.byref(c)) == sb.SPLATT_SUCCESS
    N, Z = int(c.nmodes), int(c.nnz)
    return dict(inds=[np.ctypeslib.as_array(c.ind[m], (Z,)).copy() for m in range(N)],
                vals=np.ctypeslib.as_array(c.vals, (Z,)).copy(),
                dims=[int(c.dims[m]) for m in range(N)])


def _same(a, b):
    assert a["dims"] == b["dims"]
    assert len(a["inds"]) == len(b["inds"])
    for x, y in zip(a["inds"], b["inds"]):
        assert np.array_equal(x, y)
    assert a["vals"].dtype == b["vals"].dtype
    assert np.array_equal(a["vals"].view(np.uint64), b["vals"].view(np.uint64))


TEXT_CASES = {
    "fixed_1based": "# a comment\n1 1 1 0.500000\n2 3 1 1.250000\n\n3 2 2 -7.000000\n"
                    "# another\n1 2 3 123456.789012\n",
    "zero_based_mode_and_no_newline": "0 1 1 1.5\n4 2 1 2.5\n2 3 2 3\n0 1 2 4.0",
    "crlf": "1 1 1 0.25\r\n2 2 2 0.5\r\n3 1 2 1e-3\r\n",
    "forms": "1 1 1 1e5\n2 1 1 2.5E+2\n1 2 1 -0.000123\n2 2 2 .5\n1 1 2 7.\n"
             "2 1 2 +3.25\n1 2 2 0.1\n2 2 1 1.0000000000000002\n",
    "digits17": "\n".join("%d %d %d %.17g" % (i % 7 + 1, i % 5 + 1, i % 3 + 1,
                                             np.sin(i + 0.5) * 10 ** (i % 9 - 4))
                          for i in range(200)) + "\n",
    "specials": "1 1 1 0x1p-2\n2 1 1 inf\n1 2 1 1e400\n2 2 1 4.9e-324\n",
}


@pytest.mark.parametrize("name", sorted(TEXT_CASES))
def test_text_reader_matches_host(lib64, tmp_path, name):
    p = tmp_path / (name + ".tns")
    p.write_bytes(TEXT_CASES[name].encode())
    rc, got = _read_device(lib64, p)
    assert rc == 0
    _same(got, _read_host(lib64, p))


def test_text_reader_large_seeded(lib64, tmp_path):
    """100,000 lines of the reference's own output format ("%f" values,
    1-based indices): every line takes the device's exact path."""
    rng = np.random.default_rng(3)
    n = 100_000
    idx = [rng.integers(1, d + 1, n) for d in (5000, 3000, 700)]
    vals = rng.lognormal(0, 2, n)
    p = tmp_path / "big.tns"
    with open(p, "w") as fh:
        for k in range(n):
            fh.write("%d %d %d %f\n" % (idx[0][k], idx[1][k], idx[2][k], vals[k]))
    rc, got = _read_device(lib64, p)
    assert rc == 0
    _same(got, _read_host(lib64, p))


def _write_bin(path, iw, vw, inds, vals, dims):
    with open(path, "wb") as fh:
        fh.write(struct.pack("<i", 0))
        fh.write(struct.pack("<QQ", iw, vw))
        ic = "<I" if iw == 4 else "<Q"
        fh.write(struct.pack(ic, len(inds)))
        for d in dims:
            fh.write(struct.pack(ic, d))
        fh.write(struct.pack(ic, len(vals)))
        for x in inds:
            fh.write(np.asarray(x, np.uint32 if iw == 4 else np.uint64).tobytes())
        fh.write(np.asarray(vals, np.float32 if vw == 4 else np.float64).tobytes())


@pytest.mark.parametrize("iw,vw", [(8, 8), (4, 4), (8, 4), (4, 8)])
def test_binary_reader_matches_host(lib64, tmp_path, iw, vw):
    rng = np.random.default_rng(iw * 10 + vw)
    dims = [900, 40, 17, 3]
    n = 5000
    inds = [rng.integers(0, d, n) for d in dims]
    vals = rng.normal(0, 1, n)
    p = tmp_path / "t.bin"
    _write_bin(p, iw, vw, inds, vals, dims)
    rc, got = _read_device(lib64, p)
    assert rc == 0
    _same(got, _read_host(lib64, p))
    # an index outside its dimension is refused
    inds[1][7] = dims[1]
    _write_bin(p, iw, vw, inds, vals, dims)
    rc, _ = _read_device(lib64, p)
    assert rc == 3


def test_csf_load_removes_empty_slices_on_device(lib64, port, tmp_path):
    """splatt_csf_load: device read + tt_remove_empty on the device + CSF:
    every tree equals the oracle's CSF of the compacted tensor, and the
    dims are the compacted ones."""
    import splatt_synth as S
    rng = np.random.default_rng(9)
    dims = [60, 45, 30]
    n = 2000
    # every third index of mode 0 and odd indices of mode 2 never used
    i0 = rng.choice(np.arange(0, 60, 3), n)
    i1 = rng.integers(0, 45, n)
    i2 = rng.choice(np.arange(0, 30, 2), n)
    key = (i0 * 45 + i1) * 30 + i2
    _, first = np.unique(key, return_index=True)
    first.sort()
    inds = [i0[first].astype(np.uint64), i1[first].astype(np.uint64), i2[first].astype(np.uint64)]
    vals = rng.random(len(first)) + 0.5
    p = tmp_path / "gappy.tns"
    with open(p, "w") as fh:
        for k in range(len(vals)):
            fh.write("%d %d %d %.17g\n" % (inds[0][k] + 1, inds[1][k] + 1, inds[2][k] + 1, vals[k]))
    ci, cv, cd = S.compact_empty(inds, vals, np.array([int(x.max()) + 1 for x in inds]))
    L = lib64.L
    L.splatt_csf_load.argtypes = [C.c_char_p, C.POINTER(lib64.it),
                                  C.POINTER(C.POINTER(lib64.Csf)), C.POINTER(C.c_double)]
    L.splatt_csf_load.restype = C.c_int
    nm = lib64.it()
    out = C.POINTER(lib64.Csf)()
    opts = lib64.opts(csf_alloc=sb.CSF_TWOMODE)
    assert L.splatt_csf_load(str(p).encode(), C.byref(nm), C.byref(out), opts) == 1
    got = sb.CsfSet(lib64, out, opts, 2)
    ref = port.csf(ci, cv, cd, sb.CSF_TWOMODE)
    for t in range(2):
        g, r = got.tree(t), ref.tensor(t)
        assert [int(x) for x in g["dims"]] == [int(x) for x in cd]
        for l in range(2):
            assert np.array_equal(g["fptr"][l], r["fptr"][l]), (t, l)
        for l in range(1, 3):
            assert np.array_equal(g["fids"][l], r["fids"][l]), (t, l)
        assert np.array_equal(g["vals"], r["vals"]), t
    got.free()
