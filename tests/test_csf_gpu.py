"""CSF construction on the device is bit-exact against the oracle (which is
pinned to the reference's csf_alloc): dim_perm, nfibs, fptr, fids, vals for
ONEMODE / TWOMODE / ALLMODE on 3-, 4- and 5-mode tensors (the reference's
tests/csf_test.c:31-61 structure checks, extended to every level)."""
import numpy as np
import pytest

import datasets as D

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(D.ALL))
@pytest.mark.parametrize("alloc", [0, 1, 2])
def test_csf_bit_exact(lib64, port, name, alloc):
    inds, vals, dims = D.ALL[name]()
    got = lib64.csf_convert(inds, vals, alloc)
    ref = port.csf(inds, vals, dims, alloc)
    assert got.count == ref.count
    for t in range(got.count):
        g, r = got.tree(t), ref.tensor(t)
        assert (g["dim_perm"] == r["dim_perm"]).all()
        assert (g["nfibs"] == r["nfibs"]).all()
        n = len(inds)
        for l in range(n):
            if l < n - 1:
                assert np.array_equal(g["fptr"][l], r["fptr"][l]), (t, l)
            if l > 0:
                assert np.array_equal(g["fids"][l], r["fids"][l]), (t, l)
        assert g["root_null"]          # untiled root ids stay NULL, as in SPLATT
        assert np.array_equal(g["vals"], r["vals"])
        # nfibs[0] == root dimension when no slice is empty (csf_test.c:41)
        assert g["nfibs"][0] == dims[g["dim_perm"][0]]
    ref.free()


def test_csf_frobsq(lib64):
    inds, vals, dims = D.med3()
    got = lib64.csf_convert(inds, vals, 1)
    assert abs(lib64.frobsq(got) - float(np.sum(vals * vals))) <= 1e-12 * float(np.sum(vals * vals))


def test_csf_rejects_out_of_range(lib64):
    import splatt_b200 as sb
    inds, vals, dims = D.small3()
    bad = [i.copy() for i in inds]
    # convert infers dims from the data, so a bad index cannot occur there;
    # an empty tensor is rejected
    with pytest.raises(sb.SplattError):
        lib64.csf_convert([b[:0] for b in bad], vals[:0], 1)


@pytest.mark.parametrize("name", ["small3", "zipf3", "small4", "zipf4", "small5"])
@pytest.mark.parametrize("alloc", [0, 1, 2])
@pytest.mark.parametrize("tile", [(4, 1), (3, 2), (2, 8)])
def test_csf_dense_tiled_bit_exact(lib64, port, name, alloc, tile):
    """SPLATT_DENSETILE trees (src/csf.c:427-501, src/tile.c:260-340): every
    tile of every tree bit-exact against the oracle (pinned to the
    reference's csf_alloc), empty tiles included; TWOMODE's second tree is
    untiled; root ids are kept exactly when a tree has several tiles."""
    inds, vals, dims = D.ALL[name]()
    got = lib64.csf_convert(inds, vals, alloc, tile=tile)
    ref = port.csf_tiled(inds, vals, dims, alloc, tile[0], tile[1])
    n = len(inds)
    assert got.count == len(ref)
    for t in range(got.count):
        assert got.ntiles(t) == len(ref[t]), t
        for k in range(got.ntiles(t)):
            g, r = got.tree(t, k), ref[t][k]
            assert (g["dim_perm"] == r["dim_perm"]).all()
            assert (g["nfibs"] == r["nfibs"]).all(), (t, k)
            for l in range(n):
                if l < n - 1:
                    assert np.array_equal(g["fptr"][l], r["fptr"][l]), (t, k, l)
                if l > 0 and r["nfibs"][l]:
                    assert np.array_equal(g["fids"][l], r["fids"][l]), (t, k, l)
            if got.ntiles(t) > 1 and r["nfibs"][0]:
                assert np.array_equal(g["fids"][0], r["fids"][0]), (t, k)
            else:
                assert g["root_null"]
            assert np.array_equal(g["vals"], r["vals"])


@pytest.mark.parametrize("alloc", [0, 1, 2])
@pytest.mark.parametrize("tile", [(4, 1), (3, 2)])
def test_mttkrp_dense_tiled(lib64, port, alloc, tile):
    """splatt_mttkrp on dense-tiled trees sums the tiles: every mode vs the
    oracle at the plain FP64 bar."""
    inds, vals, dims = D.zipf4()
    csf = lib64.csf_convert(inds, vals, alloc, tile=tile)
    rng = np.random.default_rng(3)
    mats = [rng.random((int(d), 16)) * 2 - 1 for d in dims]
    for m in range(len(inds)):
        got = lib64.mttkrp(csf, m, mats)
        ref = port.mttkrp_coo(inds, vals, dims, m, mats)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), m


def test_cpd_dense_tiled_matches_untiled(lib64):
    """splatt_cpd on dense-tiled trees: the same decomposition as untiled
    (the MTTKRP sums tiles in another order, so FP64-rounding close)."""
    inds, vals, dims = D.med3()
    a = lib64.cpd(lib64.csf_convert(inds, vals, 1), 8, niters=10, seed=5)
    b = lib64.cpd(lib64.csf_convert(inds, vals, 1, tile=(4, 2)), 8, niters=10, seed=5)
    assert abs(a["fit"] - b["fit"]) <= 1e-9
    for x, y in zip(a["factors"], b["factors"]):
        assert np.abs(x - y).max() <= 1e-7 * max(np.abs(y).max(), 1.0)
