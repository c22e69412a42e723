"""The oracle against committed outputs of the compiled reference
(tests/golden/ref_golden.npz, made by tests/golden/make_golden.py): CSF trees
bit-exact, MTTKRP at rank 3, CPD-ALS fit and factors, the streaming CPD
with each supported constraint, and the streaming driver's error reports.
Needs no reference build, so it pins the
oracle wherever the test suite runs.  No GPU."""
import hashlib
import os

import numpy as np
import pytest

import datasets as D
import splatt_synth as S
from oracles import PROX_KINDS

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "ref_golden.npz"))
STREAM = dict(args=(300, 200, 10, 0, 400, 0.5, 1.1), seed=4, mode=2, rank=8, rseed=11)
CONS = {"none": {}, "nonneg": dict(nonneg=True), "lasso": dict(lasso=0.01),
        "rowsimp": dict(rowsimp=True),
        "ntf_lasso": dict(ntf_lasso=0.01), "ntf_frob": dict(ntf_frob=0.1),
        "colsimp": dict(colsimp=True)}
WINDOW = dict(args=(300, 200, 60, 0, 150, 0.5, 1.1), seed=6, mode=2, rank=8, rseed=11)


def _digest(inds, vals):
    h = hashlib.sha256()
    for x in inds:
        h.update(np.ascontiguousarray(x, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(vals, dtype=np.float64).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", ["small3", "small4"])
def test_golden_csf_and_mttkrp(port, name):
    inds, vals, dims = D.ALL[name]()
    assert _digest(inds, vals) == str(G["%s/digest" % name]), "input generator changed"
    n = len(inds)
    for alloc in (0, 1, 2):
        v = port.csf(inds, vals, dims, alloc)
        for t in range(v.count):
            tr = v.tensor(t)
            k = "%s/csf%d/t%d" % (name, alloc, t)
            assert (tr["dim_perm"] == G[k + "/dim_perm"]).all()
            assert (tr["nfibs"] == G[k + "/nfibs"]).all()
            for l in range(n):
                if l < n - 1:
                    assert np.array_equal(tr["fptr"][l], G[k + "/fptr%d" % l]), (k, l)
                if l > 0:
                    assert np.array_equal(tr["fids"][l], G[k + "/fids%d" % l]), (k, l)
            assert np.array_equal(tr["vals"], G[k + "/vals"])
        v.free()
    rng = np.random.default_rng(3)
    mats = [rng.random((int(d), 3)) for d in dims]
    for m in range(n):
        want = G["%s/mttkrp%d" % (name, m)]
        got = port.mttkrp_coo(inds, vals, dims, m, mats)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), m


def test_golden_cpd(port):
    inds, vals, dims = D.small3()
    c = port.cpd(inds, vals, dims, 4, 10, 0.0, 7)
    assert abs(c["fit"] - float(G["cpd/fit"])) <= 1e-12
    for m, f in enumerate(c["factors"]):
        want = G["cpd/factor%d" % m]
        assert np.abs(f - want).max() <= 1e-12 * max(np.abs(want).max(), 1.0), m


@pytest.mark.parametrize("con", list(CONS))
def test_golden_stream(port, con):
    inds, vals, dims = S.stream_tensor(*STREAM["args"], seed=STREAM["seed"])
    assert _digest(inds, vals) == str(G["stream/digest"]), "input generator changed"
    r = port.stream(inds, vals, dims, STREAM["mode"], STREAM["rank"], seed=STREAM["rseed"],
                    **CONS[con])
    want = G["stream/%s/time" % con]
    assert r["time"].shape == want.shape
    assert np.abs(r["time"] - want).max() <= 1e-10 * np.abs(want).max()
    for m in (0, 1):
        w = G["stream/%s/factor%d" % (con, m)]
        assert np.abs(r["factors"][m] - w).max() <= 1e-10 * max(np.abs(w).max(), 1.0), m


def test_golden_stream_reports(port):
    """global, local-10 and final-err at the last batch (StreamCPD.cc:509-528,
    553-556), printed by the reference with 5 decimals."""
    inds, vals, dims = S.stream_tensor(*WINDOW["args"], seed=WINDOW["seed"])
    assert _digest(inds, vals) == str(G["window/digest"]), "input generator changed"
    r = port.stream(inds, vals, dims, WINDOW["mode"], WINDOW["rank"], seed=WINDOW["rseed"])
    T = r["time"].shape[0]
    got = [port.window_errsq(inds, vals, dims, WINDOW["mode"], r["time"], r["factors"], k)
           for k in (T, 10, T)]
    assert np.abs(np.array(got) - G["window/reports"]).max() <= 6e-6


PROX_CASES = [(37, 8, 0.1, 1.0), (120, 16, 0.01, 0.5), (3, 33, 0.5, 2.0)]


@pytest.mark.parametrize("kind", list(PROX_KINDS))
def test_golden_prox(port, kind):
    """Each ADMM constraint's proximal operator, bit-exact against the
    reference's own routine on seeded blocks."""
    for n, (I, R, lam, rho) in enumerate(PROX_CASES):
        mat = G["prox/in%d" % n]
        assert mat.shape == (I, R)
        assert np.array_equal(port.prox(PROX_KINDS[kind], mat, lam, rho),
                              G["prox/%s/%d" % (kind, n)]), n
