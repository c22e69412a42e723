"""Regenerate tests/golden/ref_golden.npz: outputs of the compiled reference
(oracle/_ref, built by `make -C oracle ref` from the SPLATT sources) on small
seeded inputs, so that the oracle stays pinned where the reference is not
built (tests/test_golden_cpu.py).

    python tests/golden/make_golden.py

Inputs are regenerated from their seeds by tests/datasets.py and
splatt_synth; a digest of each input is stored beside the outputs so a
change of generator is detected instead of compared against."""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "splatt-stream_b200"))

import datasets as D  # noqa: E402
import splatt_synth as S  # noqa: E402
from oracles import PROX_KINDS, Ref  # noqa: E402

CSF_SETS = ["small3", "small4"]
STREAM = dict(args=(300, 200, 10, 0, 400, 0.5, 1.1), seed=4, mode=2, rank=8, rseed=11)
STREAM_CONS = {"none": {}, "nonneg": dict(nonneg=True), "lasso": dict(lasso=0.01),
               "rowsimp": dict(rowsimp=True),
               "ntf_lasso": dict(ntf_lasso=0.01), "ntf_frob": dict(ntf_frob=0.1),
               "colsimp": dict(colsimp=True)}
# the streaming driver's error reports at the last batch (global, local-10,
# final-err), on a stream long enough that local-10 is not the whole history
WINDOW = dict(args=(300, 200, 60, 0, 150, 0.5, 1.1), seed=6, mode=2, rank=8, rseed=11)
# the ADMM constraints' proximal operators on seeded blocks: (rows, cols, lambda, rho)
PROX = dict(seed=5, cases=[(37, 8, 0.1, 1.0), (120, 16, 0.01, 0.5), (3, 33, 0.5, 2.0)])


def digest(inds, vals):
    h = hashlib.sha256()
    for x in inds:
        h.update(np.ascontiguousarray(x, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(vals, dtype=np.float64).tobytes())
    return h.hexdigest()


def main():
    ref = Ref(64)
    out = {}
    for name in CSF_SETS:
        inds, vals, dims = D.ALL[name]()
        out["%s/digest" % name] = np.array(digest(inds, vals))
        for alloc in (0, 1, 2):
            v = ref.csf(inds, vals, dims, alloc)
            for t in range(v.count):
                tr = v.tensor(t)
                k = "%s/csf%d/t%d" % (name, alloc, t)
                out[k + "/dim_perm"] = tr["dim_perm"]
                out[k + "/nfibs"] = tr["nfibs"]
                for l in range(len(inds)):
                    if tr["fptr"][l] is not None:
                        out[k + "/fptr%d" % l] = tr["fptr"][l].astype(np.uint32)
                    if l > 0:
                        out[k + "/fids%d" % l] = tr["fids"][l].astype(np.uint32)
                out[k + "/vals"] = tr["vals"]
            v.free()
        rng = np.random.default_rng(3)
        mats = [rng.random((int(d), 3)) for d in dims]
        q = ref.csf(inds, vals, dims, 2)
        for m in range(len(inds)):
            out["%s/mttkrp%d" % (name, m)] = ref.mttkrp(q, m, mats)[0]
        q.free()
    inds, vals, dims = D.small3()
    c = ref.cpd(inds, vals, dims, 4, 10, 0.0, 7)
    out["cpd/fit"] = np.array(c["fit"])
    for m, f in enumerate(c["factors"]):
        out["cpd/factor%d" % m] = f
    out["cpd/lambda"] = np.asarray(c["lam"])
    sinds, svals, sdims = S.stream_tensor(*STREAM["args"], seed=STREAM["seed"])
    out["stream/digest"] = np.array(digest(sinds, svals))
    for con, kw in STREAM_CONS.items():
        r = ref.stream(sinds, svals, sdims, STREAM["mode"], STREAM["rank"], seed=STREAM["rseed"],
                       **kw)
        out["stream/%s/time" % con] = r["time"]
        for m in (0, 1):
            out["stream/%s/factor%d" % (con, m)] = r["factors"][m]
    rng = np.random.default_rng(PROX["seed"])
    for n, (I, R, lam, rho) in enumerate(PROX["cases"]):
        mat = rng.normal(0, 0.5, (I, R))
        out["prox/in%d" % n] = mat
        for name, k in PROX_KINDS.items():
            out["prox/%s/%d" % (name, n)] = ref.prox(k, mat, lam, rho)
    winds, wvals, wdims = S.stream_tensor(*WINDOW["args"], seed=WINDOW["seed"])
    out["window/digest"] = np.array(digest(winds, wvals))
    r = ref.stream(winds, wvals, wdims, WINDOW["mode"], WINDOW["rank"], seed=WINDOW["rseed"])
    last = max(k for k in r["reports"] if k != "final")
    out["window/reports"] = np.array([r["reports"][last]["global_"],
                                      r["reports"][last]["local10"], r["reports"]["final"]])
    np.savez_compressed(os.path.join(HERE, "ref_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
