"""The `splatt cpd` command (splatt-stream_b200/splatt): the reference's
command-line front end (src/cmds/cmd_cpd.c) over this library.

CPU: usage and argument errors exit non-zero before any device work.
GPU: `splatt cpd X.tns --stream=3 --reg=frob,1e-2,3` writes mode%d.mat that
match the oracle's streaming factors and time rows (printed with 9
significant digits: 1e-7 relative), and the plain `splatt cpd X.tns` writes
lambda.mat and mode%d.mat that match the oracle's CPD-ALS from the same
seed (1e-7 relative; lambda, printed with 7 significant digits, 1e-6)."""
import os
import subprocess

import numpy as np
import pytest

import datasets as D
import splatt_b200 as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "splatt-stream_b200", "splatt")


def _run(args, cwd=None):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


def _write_tns(path, inds, vals):
    with open(path, "w") as fh:
        for n in range(len(vals)):
            fh.write(" ".join("%d" % (x[n] + 1) for x in inds) + " %.17g\n" % vals[n])


def test_cli_usage_and_argument_errors(tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("the command is built by splatt-stream_b200/build.py")
    r = _run([])
    assert r.returncode != 0 and "usage" in r.stderr
    r = _run(["cpd", "--help"])
    assert r.returncode == 0 and "--stream" in r.stdout
    r = _run(["frobnicate"])
    assert r.returncode != 0 and "unknown command" in r.stderr
    f = tmp_path / "x.tns"
    f.write_text("1 1 1 1.0\n")
    r = _run(["cpd", str(f), "--con=bogus"])
    assert r.returncode != 0 and "constraint 'bogus' not found" in r.stderr
    r = _run(["cpd", str(f), "--reg=frob"])
    assert r.returncode != 0 and "require 'MULT'" in r.stderr
    r = _run(["cpd", str(f), "--csf=four"])
    assert r.returncode != 0 and "not recognized" in r.stderr
    r = _run(["cpd"])
    assert r.returncode != 0


@pytest.mark.gpu
def test_cli_stream_matches_oracle(port, tmp_path):
    import splatt_synth as S
    inds, vals, dims = S.stream_tensor(300, 200, 6, 0, 400, 0.5, 1.1, seed=9)
    _write_tns(tmp_path / "x.tns", inds, vals)
    r = _run(["cpd", "x.tns", "--stream=3", "--reg=frob,1e-2,3", "-r", "8", "-i", "200",
              "--seed", "11"], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    ref = port.stream(inds, vals, dims, 2, 8, seed=11)
    _, _, _, iperm = sb.parse_stream(inds, vals, dims, 2)
    for m in (0, 1):
        got = np.loadtxt(tmp_path / ("mode%d.mat" % (m + 1)))
        b = ref["factors"][m]
        a = got[iperm[m][:len(b)].astype(np.int64)]
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)
    t = np.loadtxt(tmp_path / "mode3.mat")
    assert np.abs(t - ref["time"]).max() <= 1e-7 * np.abs(ref["time"]).max()


@pytest.mark.gpu
def test_cli_cpd_matches_oracle(port, tmp_path):
    inds, vals, dims = D.small3()
    _write_tns(tmp_path / "x.tns", inds, vals)
    r = _run(["cpd", "x.tns", "-r", "6", "-i", "10", "--tol", "0", "--seed", "5", "-s", "out"],
             cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    ref = port.cpd(inds, vals, dims, 6, 10, 0.0, 5)
    lam = np.loadtxt(tmp_path / "out.lambda.mat")
    # lambda.mat is printed "%le" (7 significant digits, src/io.c:771)
    assert np.abs(lam - ref["lam"]).max() <= 1e-6 * np.abs(ref["lam"]).max()
    for m in range(3):
        a = np.loadtxt(tmp_path / ("out.mode%d.mat" % (m + 1)))
        b = ref["factors"][m]
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)


def _reports(stdout):
    """The driver's report lines: {batch: (global, local-1, local-10)} and
    final-err."""
    import re
    rep, fin = {}, None
    for line in stdout.splitlines():
        m = re.match(r"batch\s+(\d+):.*global: ([-+0-9.eE]+) local-1: ([-+0-9.eE]+) "
                     r"local-10: ([-+0-9.eE]+)", line)
        if m:
            rep[int(m.group(1))] = tuple(float(m.group(k)) for k in (2, 3, 4))
        m = re.match(r"final-err: ([-+0-9.eE]+)", line)
        if m:
            fin = float(m.group(1))
    return rep, fin


@pytest.mark.gpu
def test_cli_stream_reports_match_reference_golden(port, tmp_path):
    """The streaming driver's report lines (StreamCPD.cc:509-534, 553-556)
    from `splatt cpd --stream`: local-1 on every batch against the oracle's
    per-slice error, and global / local-10 at the last batch and final-err
    against the reference's own printed values stored in the golden
    fixtures (both printed with 5 decimals: within 1e-5)."""
    import splatt_synth as S
    G = np.load(os.path.join(ROOT, "tests", "golden", "ref_golden.npz"))
    W = dict(args=(300, 200, 60, 0, 150, 0.5, 1.1), seed=6, mode=2, rank=8, rseed=11)
    inds, vals, dims = S.stream_tensor(*W["args"], seed=W["seed"])
    _write_tns(tmp_path / "x.tns", inds, vals)
    r = _run(["cpd", "x.tns", "--stream=3", "--reg=frob,1e-2,3", "-r", "8", "-i", "200",
              "--seed", "11"], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    rep, fin = _reports(r.stdout)
    T = int(dims[2])
    assert sorted(rep) == list(range(1, T + 1))
    ref = port.stream(inds, vals, dims, 2, 8, seed=11)
    local1 = np.array([rep[t + 1][1] for t in range(T)])
    assert np.abs(local1 - ref["local_errsq"]).max() <= 1e-5
    assert all(rep[t][0] == -1.0 and rep[t][2] == -1.0 for t in range(1, T))
    want = G["window/reports"]                    # global, local-10, final-err
    got = np.array([rep[T][0], rep[T][2], fin])
    assert np.abs(got - want).max() <= 1e-5, (got, want)
