"""The reference's own test tensors (tests/tensors/*.tns in the SPLATT source
tree: the inputs of its csf_test.c and mttkrp_test.c), read where that tree
and the compiled reference are present, skipped elsewhere.  No GPU.

  * the library's reader (splatt_coord_load, host only) gives exactly the
    coordinates, dims and values of the reference's tt_read, including the
    per-mode 0 / 1 index base (src/io.c:278-345), and reads back exactly the
    .bin files the reference's own writer makes of them at both widths
    (its binary round trip, tests/io_test.c:58-90), and its empty-slice
    removal equals the reference's tt_remove_empty (src/sptensor.c:190-252)
    on the test tensors and on synthetic ones with gaps in every mode;
  * the oracle's CSF trees (every allocation scheme, untiled and dense-tiled,
    and the reference's own dense-tile case, tests/csf_densetile_test.c) are
    bit-exact against the reference's csf_alloc on them;
  * the oracle's MTTKRP matches the reference's splatt_mttkrp on them at
    rank 3, every mode (its own test: tests/mttkrp_test.c:14-88, 1e-10)."""
import ctypes as C
import os

import numpy as np
import pytest

from oracles import REF_SRC, Ref, have_ref
from splatt_b200 import coord_struct

TENSORS = os.path.join(REF_SRC, "tests", "tensors")
FILES = ["small.tns", "small4.tns", "small4_zeroidx.tns", "med.tns", "med4.tns", "med5.tns"]

_COORD = coord_struct(64)      # splatt_coord of the 64-bit build

pytestmark = pytest.mark.skipif(not (have_ref(64) and os.path.isdir(TENSORS)),
                                reason="reference tree or its build not present")


@pytest.mark.parametrize("name", FILES)
def test_coord_load_matches_reference_reader(name):
    import splatt_b200 as sb
    path = os.path.join(TENSORS, name)
    inds, vals, dims = Ref(64).tt_read(path)
    L = sb.Lib(64).L
    L.splatt_coord_load.argtypes = [C.c_char_p, C.POINTER(_COORD)]
    L.splatt_coord_load.restype = C.c_int
    c = _COORD()
    assert L.splatt_coord_load(path.encode(), C.byref(c)) == sb.SPLATT_SUCCESS
    n, nnz = int(c.nmodes), int(c.nnz)
    assert n == len(inds) and nnz == len(vals)
    assert [int(c.dims[m]) for m in range(n)] == [int(x) for x in dims]
    for m in range(n):
        assert np.array_equal(np.ctypeslib.as_array(c.ind[m], (nnz,)), inds[m]), m
    assert np.array_equal(np.ctypeslib.as_array(c.vals, (nnz,)), vals)


@pytest.mark.parametrize("width", [64, 32])
@pytest.mark.parametrize("name", FILES)
def test_coord_load_reads_reference_binary(name, width, tmp_path):
    """The reference's binary round trip (tests/io_test.c:58-90): its own
    tt_write_binary writes each test tensor (64-bit and 32-bit builds, so
    both index and value widths of the .bin header); splatt_coord_load reads
    back exactly what the reference read from the text file."""
    if not have_ref(width):
        pytest.skip("oracle/_ref not built")
    import splatt_b200 as sb
    binp = tmp_path / "t.bin"
    inds, vals, dims = Ref(width).tt_read(os.path.join(TENSORS, name), write_bin=binp)
    L = sb.Lib(64).L
    L.splatt_coord_load.argtypes = [C.c_char_p, C.POINTER(_COORD)]
    L.splatt_coord_load.restype = C.c_int
    c = _COORD()
    assert L.splatt_coord_load(str(binp).encode(), C.byref(c)) == sb.SPLATT_SUCCESS
    n, nnz = int(c.nmodes), int(c.nnz)
    assert n == len(inds) and nnz == len(vals)
    assert [int(c.dims[m]) for m in range(n)] == [int(x) for x in dims]
    for m in range(n):
        assert np.array_equal(np.ctypeslib.as_array(c.ind[m], (nnz,)), inds[m]), m
    # the values at the writer's width, widened exactly
    assert np.array_equal(np.ctypeslib.as_array(c.vals, (nnz,)), vals.astype(np.float64))


@pytest.mark.parametrize("name", FILES)
def test_fixture_csf_port_vs_ref(port, name):
    ref = Ref(64)
    inds, vals, dims = ref.tt_read(os.path.join(TENSORS, name))
    n = len(inds)
    for alloc in (0, 1, 2):
        p = port.csf(inds, vals, dims, alloc)
        q = ref.csf(inds, vals, dims, alloc)
        assert p.count == q.count
        for t in range(p.count):
            a, b = p.tensor(t), q.tensor(t)
            assert (a["dim_perm"] == b["dim_perm"]).all() and (a["nfibs"] == b["nfibs"]).all()
            for l in range(n):
                if l < n - 1:
                    assert np.array_equal(a["fptr"][l], b["fptr"][l]), (name, alloc, t, l)
                if l > 0:
                    assert np.array_equal(a["fids"][l], b["fids"][l]), (name, alloc, t, l)
            assert np.array_equal(a["vals"], b["vals"])
        p.free()
        q.free()
        tp = port.csf_tiled(inds, vals, dims, alloc, 2, 2)
        tq = ref.csf_tiled(inds, vals, dims, alloc, 2, 2)
        assert len(tp) == len(tq)
        for t in range(len(tp)):
            assert len(tp[t]) == len(tq[t])
            for k in range(len(tp[t])):
                a, b = tp[t][k], tq[t][k]
                assert (a["nfibs"] == b["nfibs"]).all(), (name, alloc, t, k)
                for l in range(n - 1):
                    assert np.array_equal(a["fptr"][l], b["fptr"][l]), (name, alloc, t, k, l)
                assert np.array_equal(a["vals"], b["vals"])


@pytest.mark.parametrize("nthreads", [5, 1])
def test_fixture_densetile_as_reference_test(port, nthreads):
    """The reference's own dense-tile test (tests/csf_densetile_test.c:24-110):
    med4.tns, ONEMODE, DENSETILE with 5 and 1 threads at the default tile
    level 1.  Its checks (tile count, nonzeros summing over tiles) plus every
    tile's arrays against the reference's csf_alloc."""
    ref = Ref(64)
    inds, vals, dims = ref.tt_read(os.path.join(TENSORS, "med4.tns"))
    n = len(inds)
    tp = port.csf_tiled(inds, vals, dims, 0, nthreads, 1)
    tq = ref.csf_tiled(inds, vals, dims, 0, nthreads, 1)
    assert len(tp) == len(tq) == 1
    if nthreads == 1:
        assert len(tp[0]) == 1
    assert sum(int(t["nfibs"][n - 1]) for t in tp[0]) == len(vals)
    assert len(tp[0]) == len(tq[0])
    for k, (a, b) in enumerate(zip(tp[0], tq[0])):
        assert (a["nfibs"] == b["nfibs"]).all(), k
        for l in range(n):
            if l < n - 1:
                assert np.array_equal(a["fptr"][l], b["fptr"][l]), (k, l)
            # root ids are stored only when there are several tiles
            # (csf.c:260-264); one tile keeps them implicit, as untiled
            if l > 0 or len(tq[0]) > 1:
                assert np.array_equal(a["fids"][l], b["fids"][l]), (k, l)
        assert np.array_equal(a["vals"], b["vals"]), k


@pytest.mark.parametrize("name", FILES)
def test_fixture_mttkrp_port_vs_ref(port, name):
    ref = Ref(64)
    inds, vals, dims = ref.tt_read(os.path.join(TENSORS, name))
    rng = np.random.default_rng(5)
    mats = [rng.random((int(d), 3)) for d in dims]
    q = ref.csf(inds, vals, dims, 2)
    for m in range(len(inds)):
        want, _ = ref.mttkrp(q, m, mats)
        got = port.mttkrp_coo(inds, vals, dims, m, mats)
        assert np.abs(got - want).max() <= 1e-10, (name, m)
    q.free()


@pytest.mark.parametrize("alloc", [0, 1, 2])
@pytest.mark.parametrize("name", FILES)
def test_fixture_mttkrp_as_reference_tests(port, name, alloc):
    """The reference's six CSF MTTKRP tests (tests/mttkrp_test.c:173-290):
    ONE/TWO/ALL trees, untiled and dense-tiled at every depth up to the mode
    count, 7 threads, rank 3, every output mode, against the COO MTTKRP gold
    within its 1e-10 (here the oracle's COO MTTKRP is the gold); the oracle's
    tiled trees at those settings (up to depth 3) are bit-exact against the
    reference's."""
    ref = Ref(64)
    inds, vals, dims = ref.tt_read(os.path.join(TENSORS, name))
    n = len(inds)
    rng = np.random.default_rng(9)
    mats = [rng.random((int(d), 3)) for d in dims]
    gold = [port.mttkrp_coo(inds, vals, dims, m, mats) for m in range(n)]
    for level in range(0, n + 1):
        outs = ref.mttkrp_tiled(inds, vals, dims, alloc, 7, level, mats)
        for m in range(n):
            assert np.abs(outs[m] - gold[m]).max() <= 1e-10, (name, alloc, level, m)
        if level > 3:                   # 7**level tiles per tree: arrays up to 343
            continue
        tp = port.csf_tiled(inds, vals, dims, alloc, 7, level)
        tq = ref.csf_tiled(inds, vals, dims, alloc, 7, level)
        assert [len(t) for t in tp] == [len(t) for t in tq], (name, alloc, level)
        for t in range(len(tp)):
            for a, b in zip(tp[t], tq[t]):
                assert (a["nfibs"] == b["nfibs"]).all(), (name, alloc, level, t)
                for l in range(1, n):
                    assert np.array_equal(a["fids"][l], b["fids"][l]), (name, alloc, level, t, l)
                assert np.array_equal(a["vals"], b["vals"]), (name, alloc, level, t)


@pytest.mark.parametrize("alloc", [0, 1, 2])
@pytest.mark.parametrize("name", FILES)
def test_fixture_mttkrp_fp32_as_reference_tests(port, name, alloc):
    """The same six tests in the reference's 32-bit build (uint32 indices,
    float values): its CSF MTTKRP, untiled and dense-tiled at every depth,
    7 threads, against the FP64 COO gold within its FP32 tolerance, 9e-3
    absolute (tests/mttkrp_test.c:25-27)."""
    if not have_ref(32):
        pytest.skip("oracle/_ref 32-bit build absent")
    ref = Ref(32)
    inds, vals, dims = ref.tt_read(os.path.join(TENSORS, name))
    n = len(inds)
    rng = np.random.default_rng(9)
    mats = [rng.random((int(d), 3)).astype(np.float32) for d in dims]
    i64 = [x.astype(np.uint64) for x in inds]
    gold = [port.mttkrp_coo(i64, vals.astype(np.float64), dims.astype(np.uint64), m,
                            [x.astype(np.float64) for x in mats]) for m in range(n)]
    for level in range(0, n + 1):
        outs = ref.mttkrp_tiled(inds, vals, dims, alloc, 7, level, mats)
        for m in range(n):
            assert np.abs(outs[m] - gold[m]).max() <= 9e-3, (name, alloc, level, m)


def _gappy_tns(path, seed, nmodes, dims, nnz, zero_based=False):
    """A seeded tensor whose indices skip whole slices in every mode (only
    every third index of mode 0 is used, a random half of the others)."""
    rng = np.random.default_rng(seed)
    cols = []
    for m in range(nmodes):
        if m == 0:
            pool = np.arange(0, dims[m], 3)
        else:
            pool = np.sort(rng.choice(dims[m], max(1, dims[m] // 2), replace=False))
        cols.append(rng.choice(pool, nnz))
    base = 0 if zero_based else 1
    with open(path, "w") as f:
        for n in range(nnz):
            f.write(" ".join(str(int(c[n]) + base) for c in cols) +
                    " %.17g\n" % rng.lognormal())


@pytest.mark.parametrize("case", [("small4.tns", None), ("gap3", (3, [40, 25, 30], 300)),
                                  ("gap4", (4, [31, 12, 50, 9], 500)),
                                  ("gap3z", (3, [20, 20, 20], 100))])
def test_remove_empty_matches_reference(case, tmp_path):
    """Empty-slice removal (tt_remove_empty, src/sptensor.c:190-252), which
    splatt_csf_load applies after reading (src/csf.c:18-36): the library's
    host routine gives the reference's relabelled indices, dims, removed
    count and local -> global index maps, mode by mode."""
    import splatt_b200 as sb
    name, spec = case
    if spec is None:
        path = os.path.join(TENSORS, name)
    else:
        path = str(tmp_path / (name + ".tns"))
        _gappy_tns(path, 7, spec[0], spec[1], spec[2], zero_based=name.endswith("z"))
    inds, vals, dims, maps, removed = Ref(64).tt_read(path, remove_empty=True)
    L = sb.Lib(64).L
    L.splatt_coord_load.argtypes = [C.c_char_p, C.POINTER(_COORD)]
    L.sb_remove_empty.argtypes = [C.POINTER(_COORD)]
    L.sb_remove_empty.restype = C.c_uint64
    c = _COORD()
    assert L.splatt_coord_load(path.encode(), C.byref(c)) == sb.SPLATT_SUCCESS
    assert int(L.sb_remove_empty(C.byref(c))) == removed
    if spec is not None:
        assert removed > 0
    n, nnz = int(c.nmodes), int(c.nnz)
    assert [int(c.dims[m]) for m in range(n)] == [int(x) for x in dims]
    for m in range(n):
        assert np.array_equal(np.ctypeslib.as_array(c.ind[m], (nnz,)), inds[m]), m
        if maps[m] is None:
            assert not c.indmap[m], m
        else:
            got = np.ctypeslib.as_array(c.indmap[m], (int(c.dims[m]),))
            assert np.array_equal(got, maps[m]), m
    assert np.array_equal(np.ctypeslib.as_array(c.vals, (nnz,)), vals)


@pytest.mark.parametrize("width", [64, 32])
def test_fill_rand_matches_reference(width):
    """Factor initialisation draws (fill_rand / rand_val, src/util.c:16-40):
    the library's host fill gives the reference's values bit for bit after
    the same srand, at both value widths (both call the process's rand())."""
    if not have_ref(width):
        pytest.skip("oracle/_ref not built")
    import splatt_b200 as sb
    ref = Ref(width)
    lib = sb.Lib(width)
    for seed, n in ((1, 1), (7, 1000), (12345, 4097)):
        want = np.zeros(n, ref.val_dtype)
        ref.lib.ref_fill_rand(C.c_uint(seed), ref._vp(want), ref._ix(n))
        got = np.zeros(n, ref.val_dtype)
        sb.srand(seed)
        lib.L.sb_fill_rand(got.ctypes.data_as(C.c_void_p), lib.it(n))
        assert np.array_equal(got, want), (seed, n)
        assert np.abs(got).max() <= 3.0
        if n > 1:
            assert (got < 0).any() and (got > 0).any()
