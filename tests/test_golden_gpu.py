"""The CUDA path against the committed outputs of the compiled reference
(tests/golden/ref_golden.npz, made by tests/golden/make_golden.py from
oracle/_ref), directly: the same inputs, the reference's own results.

Each check is the composition of two verified links: the CUDA path against
the oracle (the other GPU tests) and the oracle against these fixtures
(tests/test_golden_cpu.py).  The tolerances are the sums of those links'
bounds: CSF arrays bit-exact; MTTKRP 2e-12 relative; CPD fit 2e-10 absolute,
factors 2e-8 relative; streaming time rows and factors 2e-9 relative
(2e-8 with lasso or the row simplex, whose thresholds amplify last-bit
differences)."""
import hashlib
import os

import numpy as np
import pytest

import datasets as D
import splatt_synth as S

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "ref_golden.npz"))
STREAM = dict(args=(300, 200, 10, 0, 400, 0.5, 1.1), seed=4, mode=2, rank=8, rseed=11)
CONS = {"none": ({}, 2e-9), "nonneg": (dict(nonneg=True), 2e-9),
        "lasso": (dict(lasso=0.01), 2e-8), "rowsimp": (dict(rowsimp=True), 2e-8),
        "ntf_lasso": (dict(ntf_lasso=0.01), 2e-8), "ntf_frob": (dict(ntf_frob=0.1), 2e-8),
        "colsimp": (dict(colsimp=True), 2e-8)}


def _digest(inds, vals):
    h = hashlib.sha256()
    for x in inds:
        h.update(np.ascontiguousarray(x, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(vals, dtype=np.float64).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", ["small3", "small4"])
def test_golden_csf_and_mttkrp_gpu(lib64, name):
    inds, vals, dims = D.ALL[name]()
    assert _digest(inds, vals) == str(G["%s/digest" % name]), "input generator changed"
    n = len(inds)
    for alloc in (0, 1, 2):
        got = lib64.csf_convert(inds, vals, alloc)
        for t in range(got.count):
            g = got.tree(t)
            k = "%s/csf%d/t%d" % (name, alloc, t)
            assert (g["dim_perm"] == G[k + "/dim_perm"]).all(), k
            assert (g["nfibs"] == G[k + "/nfibs"]).all(), k
            for l in range(n):
                if l < n - 1:
                    assert np.array_equal(g["fptr"][l], G[k + "/fptr%d" % l]), (k, l)
                if l > 0:
                    assert np.array_equal(g["fids"][l], G[k + "/fids%d" % l]), (k, l)
            assert np.array_equal(g["vals"], G[k + "/vals"]), k
    rng = np.random.default_rng(3)
    mats = [rng.random((int(d), 3)) for d in dims]
    csf = lib64.csf_convert(inds, vals, 2)
    for m in range(n):
        want = G["%s/mttkrp%d" % (name, m)]
        got = lib64.mttkrp(csf, m, mats)
        assert np.abs(got - want).max() <= 2e-12 * np.abs(want).max(), m


def test_golden_cpd_gpu(lib64):
    inds, vals, dims = D.small3()
    csf = lib64.csf_convert(inds, vals, 1)
    c = lib64.cpd(csf, 4, niters=10, tol=0.0, seed=7)
    assert abs(c["fit"] - float(G["cpd/fit"])) <= 2e-10
    for m, f in enumerate(c["factors"]):
        want = G["cpd/factor%d" % m]
        assert np.abs(f - want).max() <= 2e-8 * max(np.abs(want).max(), 1.0), m


@pytest.mark.parametrize("con", list(CONS))
def test_golden_stream_gpu(lib64, con):
    kw, tol = CONS[con]
    inds, vals, dims = S.stream_tensor(*STREAM["args"], seed=STREAM["seed"])
    assert _digest(inds, vals) == str(G["stream/digest"]), "input generator changed"
    r = lib64.stream_run(inds, vals, dims, STREAM["mode"], STREAM["rank"],
                         seed=STREAM["rseed"], **kw)
    want = G["stream/%s/time" % con]
    assert r["time"].shape == want.shape
    assert np.abs(r["time"] - want).max() <= tol * np.abs(want).max()
    for m in (0, 1):
        w = G["stream/%s/factor%d" % (con, m)]
        assert r["factors"][m].shape == w.shape, m
        assert np.abs(r["factors"][m] - w).max() <= tol * max(np.abs(w).max(), 1.0), m
