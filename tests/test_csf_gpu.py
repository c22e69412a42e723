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
