#!/usr/bin/env python
"""Benchmark of the SPLATT-stream hot path on B200.

Default workload (N=1 line): streaming CPD of a synthetic 3-mode tensor
20000 x 10000 x 500 whose third mode is time (500 slices streamed in order,
~50M nonzeros, per-slice nnz lognormal(median 80K, sigma 0.8), Zipf(1.1)
indices, lognormal(0,1) values), rank 32, frob regularisation 1e-2 on the
time mode, forgetting 0.95.  A step is one time slice's full update.

Reported per slice: fused FP64 (headline `value`, device-resident slices),
fused FP32+FP64-solve, the plain FP64 per-phase path (the denominator of the
fused-vs-plain speed-up), p50/p99 latency, `e2e` through the host-buffer
C-ABI (splatt_b200_stream_push), the live roofline of the fused slice
kernel, and the reference's OpenMP CPU path on a bounded sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload stream|cpd]

Multi-GPU (torchrun): every rank streams its own independent tensor (weak
scaling, no data-path collective); timing is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "splatt-stream_b200"))
# the CPU-baseline leg drives the oracle / compiled reference (test code)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

C2 = dict(I=20000, J=10000, T=500, total_nnz=50_000_000, median=80000, sigma=0.8, zipf=1.1,
          rank=32, reg=1e-2, forget=0.95)
C3 = dict(dims=(2_000_000, 500_000, 50_000, 1_000), nnz=400_000_000, zipf=1.2, rank=64)
C5 = dict(streams=64, I=50_000, J=20_000, rank=32, reg=1e-2, forget=0.95, rate=200.0,
          median=50_000, sigma=1.0, zipf=1.1, budget=120 * 10**9)
# slices timed (and warm-up slices run) at most by the CPU reference arm
REF_MAX_STEPS = 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="stream",
                    choices=["stream", "mttkrp", "serve", "cpd", "batch"])
    ap.add_argument("--serve-horizon", type=float, default=0.5,
                    help="seconds of Poisson arrivals in the serving measurement")
    ap.add_argument("--serve-slices", type=int, default=6,
                    help="distinct pre-generated slices per served stream (cycled)")
    ap.add_argument("--serve-sat", type=int, default=12,
                    help="slices per stream in the saturated serving measurement")
    ap.add_argument("--serve-chain", type=int, default=4,
                    help="batch capacity in slices per stream (a stream's waiting slices "
                         "run as a chain within one launch)")
    ap.add_argument("--no-mttkrp", action="store_true",
                    help="skip the static-MTTKRP sub-measurement of the stream workload")
    ap.add_argument("--mttkrp-scale", type=float, default=1.0,
                    help="fraction of the 400M nonzeros of the static-MTTKRP tensor")
    ap.add_argument("--cpu-slices", type=int, default=8,
                    help="slices of the stream timed on the CPU baseline (after the warm-up "
                         "slices; the parity block compares every slice that run covers)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--slices", type=int, default=None,
                    help="stream only the first SLICES slices (the whole-stream figures and the "
                         "precision study then cover those; for profiling runs)")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the precision study of the stream workload")
    ap.add_argument("--no-serve", action="store_true",
                    help="skip the serving sub-measurement of the stream workload")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 256-stream batched sub-measurement of the stream workload")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--seed", type=int, default=2024)
    return ap.parse_args()


# --------------------------------------------------------------------------
# distributed plumbing
# --------------------------------------------------------------------------
def dist_init(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def dist_max(pg, x):
    """Max over ranks (timers: the job takes as long as its slowest rank)."""
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(pg):
    if pg is not None:
        pg.barrier()


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """Per-launch DRAM bytes of a kernel from its committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.strip().startswith("traffic_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].strip())
                except ValueError:
                    return None
    return None


# --------------------------------------------------------------------------
# the streaming workload
# --------------------------------------------------------------------------
def make_stream(seed, max_t):
    """The first `max_t` slices (all when None) of the seeded streaming
    tensor; every slice holds exactly its lognormal target count of distinct
    nonzeros (50M over the 500 slices).  A prefix of the stream is the same
    whatever `max_t` is, so the reference arm and the B200 arm see the same
    slices."""
    import splatt_b200 as sb
    import splatt_synth as S
    inds, vals, dims = S.stream_tensor(C2["I"], C2["J"], C2["T"], C2["total_nnz"], C2["median"],
                                       C2["sigma"], C2["zipf"], seed=seed, sort_slices=True,
                                       max_t=max_t, exact=True)
    return prepare_stream(inds, vals, dims)


def prepare_stream(inds, vals, dims):
    """ParserSimple's preparation (host) of a stream whose slices are sorted
    by (mode 1, mode 2): relabelled indices, slice offsets and the per-slice
    dims the streaming driver sees."""
    import splatt_b200 as sb
    s_inds, s_vals, offs, _ = sb.parse_stream(inds, vals, dims, 2, presorted=True)
    T = len(offs) - 1
    sdims = []
    prev = [0, 0]
    for t in range(T):
        a, b = int(offs[t]), int(offs[t + 1])
        d = []
        for q, m in enumerate((0, 1)):
            mx = int(s_inds[m][a:b].max()) + 1
            prev[q] = max(prev[q], mx)
            d.append(prev[q])
        sdims.append((d[0], d[1], 1))
    return dict(inds=s_inds, vals=s_vals, offs=offs, dims=dims, sdims=sdims, T=T,
                raw=(inds, vals))


def bench_ingest(lib, data, torch, reps=3):
    """ParserSimple's preparation of the whole streamed tensor on the device
    (sb_stream_prepare: order by time then the other modes, first-appearance
    relabel, slice bounds), as splatt_cpd_stream runs it; checked against the
    host preparation the stream bench itself uses."""
    import ctypes as C
    inds, vals = data["raw"]
    dims = [int(x) for x in data["dims"]]
    dims[2] = int(data["T"])                 # the slices actually generated
    N, nnz, T = len(inds), len(vals), dims[2]
    dI = [torch.from_numpy(np.ascontiguousarray(x, dtype=np.int32)).cuda() for x in inds]
    dV = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float64)).cuda()
    oI = [torch.empty(nnz, dtype=torch.int32, device="cuda") for _ in range(N)]
    oV = torch.empty(nnz, dtype=torch.float64, device="cuda")
    maps = [torch.empty(max(dims[m], 1), dtype=torch.int32, device="cuda") for m in range(N)]
    L = lib.L
    f = L.sb_stream_prepare
    P = C.POINTER
    f.argtypes = [C.c_uint32, C.c_uint64, P(C.c_uint64), P(C.c_void_p), C.c_void_p, C.c_int,
                  C.c_uint32, P(C.c_void_p), C.c_void_p, P(C.c_void_p), P(C.c_uint64),
                  P(C.c_uint64), P(C.c_uint64)]
    f.restype = C.c_int
    d64 = (C.c_uint64 * N)(*dims)
    ip = (C.c_void_p * N)(*[x.data_ptr() for x in dI])
    op = (C.c_void_p * N)(*[x.data_ptr() for x in oI])
    mp = (C.c_void_p * N)(*[x.data_ptr() for x in maps])
    nlab = np.zeros(N, np.uint64)
    offs = np.zeros(T + 1, np.uint64)
    seen = np.zeros(N * T, np.uint64)
    U = P(C.c_uint64)
    orig = L.splatt_b200_get_stream()
    L.splatt_b200_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    secs = []
    try:
        for r in range(reps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rc = f(N, nnz, d64, ip, C.c_void_p(dV.data_ptr()), 0, 2, op,
                   C.c_void_p(oV.data_ptr()), mp, nlab.ctypes.data_as(U),
                   offs.ctypes.data_as(U), seen.ctypes.data_as(U))
            torch.cuda.synchronize()
            if rc != 0:
                return {"error": "sb_stream_prepare returned %d" % rc}
            if r:
                secs.append(time.perf_counter() - t0)
    finally:
        L.splatt_b200_set_stream(C.c_void_p(orig))
    ok = bool(np.array_equal(offs, np.asarray(data["offs"], dtype=np.uint64)))
    for m in range(N):
        ok = ok and bool(np.array_equal(oI[m].cpu().numpy().astype(np.uint64),
                                        np.asarray(data["inds"][m], dtype=np.uint64)))
    ok = ok and bool(np.array_equal(oV.cpu().numpy(), np.asarray(data["vals"], dtype=np.float64)))
    t = float(np.median(secs))
    return {"what": "ParserSimple preparation of the whole tensor on the device "
                    "(splatt_cpd_stream's ingest): sort by (time, mode 1, mode 2), "
                    "first-appearance relabel, slice bounds",
            "nnz": nnz, "slices": T, "seconds": t, "mnnz_per_s": nnz / t / 1e6,
            "matches_host_parser": ok}


def alg_bytes_slice(nnz, rows, outer, inner, vbytes):
    """Algorithmic bytes of one slice update: per outer iteration the COO
    MTTKRP of each mode reads nnz (value + 3 uint32 indices) and writes
    nothing beyond the output rows; each non-streamed mode m moves
    rows_m*R*s bytes 6 times per ADMM iteration (M, P, D, aux, init, solve
    pass) and 5 times per outer iteration (Gram, historical GEMM, delta)."""
    R = C2["rank"]
    b = outer * nnz * (vbytes + 3 * 4) * 3
    for m in (0, 1):
        b += rows[m] * R * vbytes * (6 * inner[m] + 5 * outer)
    return b


def run_device(lib, data, torch, nslices, precision, exec_, seed, flush, stats=True):
    """Slices 0..nslices-1 from device-resident COO through
    splatt_b200_stream_push_device; one pair of CUDA events per slice on the
    library stream, the L2 flushed between slices (outside the events).
    With `stats`, each slice's outer/ADMM iterations, rows and local error^2
    are read after its end event.  Returns (seconds per slice, records, time
    rows of every slice)."""
    import splatt_b200 as sb
    st = torch.cuda.Stream()
    orig = lib.L.splatt_b200_get_stream()
    lib.L.splatt_b200_set_stream(C_void(st.cuda_stream))
    vdt = torch.float64 if precision == sb.FP64 else torch.float32
    dev = torch.device("cuda")
    ii = [torch.from_numpy(data["inds"][m].astype(np.int32)).to(dev) for m in (0, 1)]
    vv = torch.from_numpy(data["vals"]).to(dev, vdt)
    dummy = torch.zeros(8, dtype=torch.int32, device=dev)
    sb.srand(seed)
    s = sb.Stream(lib, 3, 2, data["dims"], C2["rank"], C2["forget"], C2["reg"], 200, precision,
                  exec_)
    offs = data["offs"]
    recs = []
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(nslices)]
    torch.cuda.synchronize()
    for t in range(nslices):
        a, b = int(offs[t]), int(offs[t + 1])
        ptrs = [ii[0].data_ptr() + 4 * a, ii[1].data_ptr() + 4 * a, dummy.data_ptr()]
        vptr = vv.data_ptr() + vv.element_size() * a
        with torch.cuda.stream(st):
            flush.zero_()
            evs[t][0].record(st)
            s.push_device(ptrs, vptr, b - a, data["sdims"][t])
            evs[t][1].record(st)
        if stats:
            s.sync()
            outer, inner, rows = s.stats()
            recs.append(dict(nnz=b - a, rows=rows, outer=outer, inner=inner,
                             errsq=s.local_errsq()))
    st.synchronize()
    s.sync()
    times = np.array([e0.elapsed_time(e1) * 1e-3 for e0, e1 in evs])
    trows = s.factors(nslices)[2] if stats else None
    s.free()
    lib.L.splatt_b200_set_stream(C_void(orig))
    return times, recs, trows


def C_void(x):
    import ctypes
    return ctypes.c_void_p(x)


def run_e2e(lib, data, K, W, seed, torch):
    """Through the host-buffer C-ABI: each step copies the slice from host
    memory (pinned staging inside the library), runs the update and reads
    the time row back."""
    import splatt_b200 as sb
    offs = data["offs"]
    sb.srand(seed)
    s = sb.Stream(lib, 3, 2, data["dims"], C2["rank"], C2["forget"], C2["reg"], 200, sb.FP64,
                  sb.FUSED)
    keep = [np.ascontiguousarray(x) for x in data["inds"]]
    times, h2d = [], 0
    for t in range(W + K):
        a, b = int(offs[t]), int(offs[t + 1])
        sl = [x[a:b] for x in keep]
        vals = data["vals"][a:b]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.push(sl, vals)
        t1 = time.perf_counter()
        if t >= W:
            times.append(t1 - t0)
            h2d += (b - a) * (2 * 4 + 8)
    s.free()
    return np.array(times), h2d // max(K, 1)


def cpu_baseline(data, nslices, ref_ok, warm, seed):
    """The reference's OpenMP streaming CPD (oracle/_ref) on the first
    `warm + nslices` slices of the same stream with the same factor seed, all
    host threads; the first `warm` slices are warm-up and only the next
    `nslices` are timed (each slice's batch_time as the reference prints it).
    Returns (the cpu_baseline object, the run's per-slice outputs)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracles
    offs = data["offs"]
    total = warm + nslices
    n = int(offs[total])
    # the stream's original coordinates (slices in time order, the same
    # nonzeros as data["inds"][:, :n]): the reference's ParserSimple then
    # assigns the labels the B200 arm's prepared stream carries.  (Feeding it
    # the already relabelled indices would make it relabel them again, by
    # first appearance in a different order, and give later slices' new rows
    # other random initial values.)
    raw_inds, raw_vals = data["raw"]
    inds = [np.asarray(raw_inds[m][:n]) for m in range(3)]
    vals = np.asarray(raw_vals[:n])
    dims = np.array([int(inds[0].max()) + 1, int(inds[1].max()) + 1, total], np.uint64)
    cores = os.cpu_count() or 1
    if ref_ok:
        ref = oracles.Ref(64, nthreads=cores)
        out = ref.stream(inds, vals, dims, 2, C2["rank"], C2["forget"], C2["reg"], 200, seed=seed)
        secs = np.asarray(out["batch_secs"])[warm:total]
        kind, how = "reference", "per-slice batch_time"
    else:
        port = oracles.Port()
        t0 = time.perf_counter()
        port.stream(inds, vals, dims, 2, C2["rank"], C2["forget"], C2["reg"], 200, seed=seed,
                    max_slices=warm)
        t1 = time.perf_counter()
        out = port.stream(inds, vals, dims, 2, C2["rank"], C2["forget"], C2["reg"], 200,
                          seed=seed)
        t2 = time.perf_counter()
        # the whole run less a run of the warm-up slices alone
        secs = np.array([max((t2 - t1) - (t1 - t0), 1e-9) / nslices] * nslices)
        kind, cores, how = "port", 1, "wall time of the run less that of the warm-up slices"
    cb = dict(value=float(nslices / secs.sum()), unit="slices/s", cores=cores, kind=kind,
              sample="slices %d-%d (%d nnz through slice %d) of the same stream and factor "
                     "seed, after %d untimed warm-up slices; rank %d, %s"
                     % (warm, total - 1, n, total - 1, warm, C2["rank"], how),
              p99_ms=float(np.percentile(secs, 99) * 1e3))
    return cb, out


def _fits(recs):
    return 1.0 - np.sqrt(np.maximum(np.array([r["errsq"] for r in recs]), 0.0))


def _drift(fa, fb, W):
    """Per-slice |fit_a - fit_b| after the warm-up slices: max per decile of
    the stream, overall max and the first slice above 1e-4; and the
    difference of the deciles' mean fits."""
    d = np.abs(fa - fb)[W:]
    over = np.nonzero(d > 1e-4)[0]
    return {"max_by_decile": [float(x.max()) for x in np.array_split(d, 10)],
            "max_abs": float(d.max()), "mean_abs": float(d.mean()),
            "first_slice_over_1e-4": int(W + over[0]) if over.size else None,
            "mean_fit_diff_by_decile": [float(abs(x.mean() - y.mean())) for x, y in
                                        zip(np.array_split(fa[W:], 10),
                                            np.array_split(fb[W:], 10))]}


def precision_study(lib, data, torch, args, flush, W, r64, r32, rp):
    """How far the FP32 mode's per-slice fit moves from the FP64 run's over
    the whole stream, beside how far two FP64 runs that differ only in
    summation order (the fused and the plain executors) move apart, on the
    workload's random values and on a planted stream of exact rank 32 plus
    10% noise (splatt_synth.planted_stream), where the factorisation has a
    well-defined optimum."""
    import splatt_b200 as sb
    import splatt_synth as S
    T = data["T"]
    f64, f32 = _fits(r64), _fits(r32)
    out = {"random_values": {"fp32_vs_fp64": _drift(f32, f64, W),
                             "fit_fp64_by_decile": [float(x.mean()) for x in
                                                    np.array_split(f64[W:], 10)]}}
    if rp is not None:
        out["random_values"]["fp64_plain_vs_fp64_fused"] = _drift(_fits(rp), f64, W)
    pi, pv, pd = S.planted_stream(C2["I"], C2["J"], T, C2["rank"], 50, 50, 0.7, 0.1,
                                  args.seed + 1)
    dp = prepare_stream(pi, pv, pd)
    _, q64, _ = run_device(lib, dp, torch, T, sb.FP64, sb.FUSED, args.seed, flush)
    _, q32, _ = run_device(lib, dp, torch, T, sb.FP32, sb.FUSED, args.seed, flush)
    _, qp, _ = run_device(lib, dp, torch, T, sb.FP64, sb.PLAIN, args.seed, flush)
    g64, g32 = _fits(q64), _fits(q32)
    out["planted_rank32_noise0.1"] = {
        "data": "20000x10000x%d stream of exact rank 32 plus 10%% noise: 32 blocks of 50 x 50 "
                "(rows x columns), each active in a slice with probability 0.7, factor entries "
                "U(0.5, 1.5); %d nonzeros" % (T, len(pv)),
        "fp32_vs_fp64": _drift(g32, g64, W),
        "fp64_plain_vs_fp64_fused": _drift(_fits(qp), g64, W),
        "fit_fp64_by_decile": [float(x.mean()) for x in np.array_split(g64[W:], 10)]}
    out["note"] = ("per-slice local fit 1 - sqrt(relative error^2); slices %d-%d; the FP64 "
                   "plain-vs-fused pair differs only in the order of FP64 sums" % (W, T - 1))
    return out


def stream_config(W, K, seed):
    """The `config` object of the streaming line, the same in both arms."""
    return {"workload": "streaming CPD: 3-mode 20000x10000x500 (time = mode 3), 50M nnz "
                        "(per-slice lognormal, median 80K, sigma 0.8), Zipf(1.1), rank 32, "
                        "frob 1e-2, forget 0.95",
            "slices_timed": "%d-%d" % (W, W + K - 1), "seed": seed}


def stream_parity(recs, trows, ref_out, nref):
    """The B200 FP64 run against the reference's own run over the slices both
    ran: the reference's printed local-1 error^2 (5 decimals), its outer
    iteration counts (its "delta:" lines) and its time rows."""
    g_err = np.array([r["errsq"] for r in recs[:nref]])
    r_err = np.asarray(ref_out["local_errsq"])[:nref]
    g_out = [int(r["outer"]) for r in recs[:nref]]
    r_out = [int(x) for x in np.asarray(ref_out.get("outer", []))[:nref]]
    rt = np.asarray(ref_out["time"])[:nref]
    by_slice = np.abs(trows[:nref] - rt).max(axis=1) / np.abs(rt).max()
    trel = float(by_slice.max())
    d = float(np.abs(g_err - r_err).max())
    ok = d <= 1e-5 and g_out == r_out and trel <= 1e-9
    return {"against": "reference (oracle/_ref, StreamCPD::compute), same stream and factor seed",
            "slices": "0-%d" % (nref - 1),
            "local1_errsq_max_abs_diff": d, "local1_tolerance": 1e-5,
            "local1_note": "the reference prints local-1 to 5 decimals",
            "outer_gpu": g_out, "outer_reference": r_out, "outer_identical": g_out == r_out,
            "time_rows_max_rel_diff": trel, "time_rows_tolerance": 1e-9,
            "time_rows_rel_diff_by_slice": [float(x) for x in by_slice], "ok": bool(ok)}


def bench_stream(args, world, rank, local, pg):
    import torch
    import splatt_b200 as sb
    W = max(3, args.warmup)
    K = args.steps if args.steps is not None else 20
    data = make_stream(args.seed + 7919 * rank, args.slices)
    T = data["T"]
    K = max(1, min(K, T - W))
    lib = sb.Lib(64)
    lib.init(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    # untimed warm run (module load, allocations)
    run_device(lib, data, torch, 2, sb.FP64, sb.FUSED, args.seed, flush, stats=False)

    clocks = ClockSampler(local)
    dist_barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    # the whole stream: slices W..W+K-1 are the headline window; all slices
    # after the W warm-up ones give the whole-stream figures
    t64, r64, trows64 = run_device(lib, data, torch, T, sb.FP64, sb.FUSED, args.seed, flush)
    torch.cuda.synchronize()
    clk = clocks.stop()
    dist_barrier(pg)
    win = slice(W, W + K)
    total64 = dist_max(pg, float(t64[win].sum()))
    t32, r32, _ = run_device(lib, data, torch, T, sb.FP32, sb.FUSED, args.seed, flush)
    total32 = dist_max(pg, float(t32[win].sum()))
    e64 = np.array([r["errsq"] for r in r64])
    e32 = np.array([r["errsq"] for r in r32])
    fit64 = 1.0 - np.sqrt(np.maximum(e64, 0.0))
    dfit = np.abs((1.0 - np.sqrt(np.maximum(e32, 0.0))) - fit64)[W:]
    plain, rp = None, None
    if not args.no_plain:
        # the plain per-phase executor over the whole stream: its first K
        # slices after warm-up time the denominator of the fused speed-up,
        # all of them give the FP64-vs-FP64 drift (a different summation
        # order) of the precision study
        Kp = min(K, 60)
        tp, rp, _ = run_device(lib, data, torch, T, sb.FP64, sb.PLAIN, args.seed, flush)
        totp = dist_max(pg, float(tp[W:W + Kp].sum()))
        plain = dict(value=world * Kp / totp, unit="slices/s", steps=Kp,
                     slices_timed="%d-%d" % (W, W + Kp - 1),
                     p50_ms=float(np.percentile(tp[W:W + Kp], 50) * 1e3),
                     p99_ms=float(np.percentile(tp[W:W + Kp], 99) * 1e3))
    study = None if args.no_precision else precision_study(lib, data, torch, args, flush, W, r64,
                                                            r32, rp)
    te, h2d = run_e2e(lib, data, K, W, args.seed, torch)
    tote = dist_max(pg, float(te.sum()))

    # roofline of the fused slice kernel (one launch per slice)
    peak, peak_kind = measured_peaks()
    alg = [alg_bytes_slice(r["nnz"], r["rows"], r["outer"], r["inner"], 8) for r in r64]
    achieved = float(np.sum(alg[W:W + K]) / t64[win].sum() / 1e9)
    traffic = profile_traffic("stream_fused_c2.md")
    roof = dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s",
                frac=achieved / peak, traffic=traffic, peak_source=peak_kind,
                kernel="k_stream_fused<double, false>",
                note="per-slice algorithmic bytes (COO MTTKRP + ADMM/Gram/historical "
                     "passes over the factor rows) / per-slice event time, headline window; "
                     "factor state (~8 MB) is L2-resident, so the slice is latency-bound")
    ws = t64[W:]
    every = np.arange(W, T, 25)
    whole = {"slices": "%d-%d" % (W, T - 1), "value": float(ws.size / ws.sum()),
             "unit": "slices/s", "p50_ms": float(np.percentile(ws, 50) * 1e3),
             "p99_ms": float(np.percentile(ws, 99) * 1e3),
             "every_25th_slice": {"slices": [int(x) for x in every],
                                  "value": float(every.size / t64[every].sum()),
                                  "ms": [float(t64[x] * 1e3) for x in every]},
             "value_by_decile": [float(x.size / x.sum()) for x in np.array_split(ws, 10)],
             "outer_iterations": {"mean": float(np.mean([r["outer"] for r in r64[W:]])),
                                  "max": int(max(r["outer"] for r in r64[W:]))},
             "rows_at_end": [int(r64[-1]["rows"][0]), int(r64[-1]["rows"][1])],
             "roofline_frac": float(np.sum(alg[W:]) / ws.sum() / 1e9 / peak),
             "fp32_value": float(t32[W:].size / t32[W:].sum())}
    line = {
        "metric": "streamed slices/sec (streaming CPD, 20000x10000x500, rank 32)",
        "value": world * K / total64,
        "unit": "slices/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": total64 / K * 1e3,
        "p50_ms": float(np.percentile(t64[win], 50) * 1e3),
        "p99_ms": float(np.percentile(t64[win], 99) * 1e3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded; Zipf(1.1) indices, lognormal values; per rank)",
        "config": stream_config(W, K, args.seed),
        "setup": {"executor": "fused persistent slice kernel (one cooperative launch per "
                              "slice), device-resident slices",
                  "nnz_realised": int(len(data["vals"])), "slices": T,
                  "l2": "flushed between slices (256 MB write, outside the timed events)",
                  "parallelism": "replicas" if world > 1 else "1 GPU"},
        "whole_stream": whole,
        "fp32": {"value": world * K / total32, "unit": "slices/s",
                 "p50_ms": float(np.percentile(t32[win], 50) * 1e3),
                 "p99_ms": float(np.percentile(t32[win], 99) * 1e3),
                 "dtype": "f32 factors/MTTKRP, f64 Gram/Cholesky/solve/norms",
                 "fit_vs_fp64": {
                     "max_abs_first_100": float(dfit[:100].max()),
                     "max_abs": float(dfit.max()), "mean_abs": float(dfit.mean()),
                     "first_slice_over_1e-4": (int(W + np.argmax(dfit > 1e-4))
                                               if (dfit > 1e-4).any() else None),
                     "max_abs_by_decile": [float(x.max()) for x in np.array_split(dfit, 10)
                                           if x.size],
                     "slices": "%d-%d" % (W, T - 1),
                     "note": "per-slice local fit 1 - sqrt(relative error^2) of the FP32 run "
                             "minus that of the FP64 run, both from the same initial factors"}},
        "fit_fp64": {"mean": float(fit64[W:].mean()), "last": float(fit64[-1])},
        "precision_study": study,
        "plain_fp64": plain,
        "e2e": {"value": world * K / tote, "unit": "slices/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": C2["rank"] * 8 + 48,
                "path": "splatt_b200_stream_push (host COO -> pinned -> device, time row back)"},
        "roofline": roof,
        "gpu_launches": K,
        "clocks": clk,
    }
    if plain:
        line["speedup_fused_vs_plain_fp64"] = line["value"] / plain["value"]
    if rank == 0 and not args.no_cpu_baseline:
        from oracles import have_ref  # noqa
        nref = max(1, min(args.cpu_slices, K))
        cb, ref_out = cpu_baseline(data, nref, have_ref(64), W, args.seed)
        line["cpu_baseline"] = cb
        if have_ref(64):
            line["parity"] = stream_parity(r64, trows64, ref_out, W + nref)
    if rank == 0:
        try:
            line["ingest"] = bench_ingest(lib, data, torch)
        except Exception as e:          # keep the streaming line if this part fails
            line["ingest"] = {"error": str(e)[:300]}
    if not args.no_mttkrp:
        del flush
        torch.cuda.empty_cache()
        lib32 = sb.Lib(32)
        lib32.init(local)
        try:
            mk = bench_mttkrp(args, torch, lib32, args.mttkrp_scale)
        except Exception as e:          # keep the streaming line if this part fails
            line["static_mttkrp"] = {"error": str(e)[:300]}
            return line
        line["static_mttkrp"] = dict(
            workload="static CSF MTTKRP, 4-mode %s, %d nnz, Zipf(1.2), FP32, rank 64, "
                     "one CSF per mode, all modes in turn" % ("x".join(map(str, mk["dims"])),
                                                              mk["nnz"]),
            value=mk["gbs"], unit="GB/s (algorithmic)", frac=mk["gbs"] / peak,
            ms_per_mode=mk["ms_per_mode"], gbs_per_mode=mk["gbs_per_mode"],
            csf_build_s=mk["csf_build_s"], kernel="k_csf_root<float,4,16,4>",
            nfibs=mk["nfibs"], gram=mk.get("gram"),
            traffic=profile_traffic("mttkrp_csf_c3.md"))
        del lib32
        torch.cuda.empty_cache()
    if not args.no_serve:
        try:
            sv = bench_serve(args, world, rank, local, pg)
            line["serve"] = {k: sv[k] for k in (
                "metric", "value", "unit", "p50_ms", "p99_ms", "dtype", "config",
                "saturated_fp32", "poisson_200_per_stream_fp32", "poisson_half_capacity_fp32",
                "saturated_fp64", "plain_fp64_per_slice", "speedup_vs_plain_fp64",
                "accuracy_planted", "fit_vs_fp64", "clocks")}
        except Exception as e:          # keep the streaming line if this part fails
            line["serve"] = {"error": str(e)[:300]}
        torch.cuda.empty_cache()
    if not args.no_batch:
        try:
            bargs = argparse.Namespace(**vars(args))
            bargs.steps, bargs.warmup = 2, 3
            bt = bench_batch(bargs, world, rank, local, pg)
            line["batch"] = {k: bt[k] for k in (
                "metric", "value", "unit", "steps", "warmup", "ms_per_step", "dtype", "config",
                "outer_iterations_last_step", "gpu_launches", "clocks")}
        except Exception as e:
            line["batch"] = {"error": str(e)[:300]}
    return line


# --------------------------------------------------------------------------
# static CSF MTTKRP: 4-mode 2M x 500K x 50K x 1K, 400M nnz, Zipf(1.2), FP32,
# rank 64, one CSF per mode (ALLMODE), MTTKRP of every mode in turn
# --------------------------------------------------------------------------
def gen_zipf_gpu(torch, dims, nnz, s, seed, device="cuda"):
    """Seeded bounded-Zipf(s) 4-mode coordinates, duplicates dropped, empty
    slices compacted, values U(0,1] (splatt_synth.zipf_tensor_torch)."""
    import splatt_synth as S
    return S.zipf_tensor_torch(torch, dims, nnz, s, seed, device=device)


def mttkrp_alg_bytes(nnz, nfibs, dims, out_mode, R, s=4, x=4):
    """Algorithmic bytes of one CSF MTTKRP launch: leaf vals + ids, fptr/fids
    of the upper levels (root ids not stored untiled), every input factor
    once, the output once."""
    b = nnz * (s + x)
    N = len(dims)
    for l in range(N - 1):
        b += (nfibs[l] + 1) * x + (nfibs[l] * x if l > 0 else 0)
    b += sum(dims[m] * R * s for m in range(N) if m != out_mode)
    b += dims[out_mode] * R * s
    return b


def bench_mttkrp(args, torch, lib, scale, K=3, W=2):
    import ctypes
    import splatt_b200 as sb
    t0 = time.perf_counter()
    inds, vals, dims = gen_zipf_gpu(torch, C3["dims"], int(C3["nnz"] * scale), C3["zipf"],
                                    args.seed)
    nnz = int(vals.numel())
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    R = C3["rank"]
    L = lib.L
    L.splatt_b200_csf_convert_device.argtypes = [
        ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
        ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int,
        ctypes.POINTER(ctypes.POINTER(lib.Csf)), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    L.splatt_b200_csf_convert_device.restype = ctypes.c_int
    opts = lib.opts(csf_alloc=sb.CSF_ALLMODE)
    d64 = (ctypes.c_uint64 * 4)(*dims)
    dptr = (ctypes.c_void_p * 4)(*[x.data_ptr() for x in inds])
    csf = ctypes.POINTER(lib.Csf)()
    t0 = time.perf_counter()
    lib.check(L.splatt_b200_csf_convert_device(4, nnz, d64, dptr, ctypes.c_void_p(vals.data_ptr()),
                                                1, ctypes.byref(csf), opts, 0), "csf_convert_device")
    torch.cuda.synchronize()
    t_csf = time.perf_counter() - t0
    del inds, vals
    nfibs = [[int(csf[m].pt.contents.nfibs[l]) for l in range(4)] for m in range(4)]
    g = torch.Generator(device="cuda").manual_seed(1)
    mats = [torch.rand(d, R, device="cuda", dtype=torch.float32, generator=g) for d in dims]
    outs = [torch.empty(d, R, device="cuda", dtype=torch.float32) for d in dims]
    mp = (ctypes.c_void_p * 4)(*[m.data_ptr() for m in mats])
    st = torch.cuda.Stream()
    orig = L.splatt_b200_get_stream()
    L.splatt_b200_set_stream(C_void(st.cuda_stream))
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(4)] for _ in range(K)]
    torch.cuda.synchronize()
    for it in range(W + K):
        for m in range(4):
            with torch.cuda.stream(st):
                if it >= W:
                    ev[it - W][m][0].record(st)
                rc = L.splatt_b200_mttkrp_device(lib.it(m), lib.it(R), csf, opts, mp, lib.it(R),
                                                 C_void(outs[m].data_ptr()), lib.it(R), 1)
                if it >= W:
                    ev[it - W][m][1].record(st)
            lib.check(rc, "mttkrp_device")
    st.synchronize()
    L.splatt_b200_set_stream(C_void(orig))
    per_mode = np.array([[ev[k][m][0].elapsed_time(ev[k][m][1]) * 1e-3 for m in range(4)]
                         for k in range(K)])
    t_mode = per_mode.mean(axis=0)
    alg = [mttkrp_alg_bytes(nnz, nfibs[m], dims, m, R) for m in range(4)]
    gram = bench_gram(torch, lib, mats[0], K=K, W=W)
    L.splatt_free_csf(csf, opts)
    del mats, outs
    torch.cuda.empty_cache()
    return dict(nnz=nnz, dims=dims, nfibs=nfibs, ms_per_mode=[float(x * 1e3) for x in t_mode],
                alg_bytes_per_mode=alg, gbs_per_mode=[a / t / 1e9 for a, t in zip(alg, t_mode)],
                gbs=float(sum(alg) / t_mode.sum() / 1e9), seconds_all_modes=float(t_mode.sum()),
                gen_s=t_gen, csf_build_s=t_csf, gram=gram)


def bench_gram(torch, lib, A, K=5, W=2):
    """G = A^T A of one FP32 factor (rows x R, larger than L2) through sb_gram:
    the tensor-core path (split TF32 products, k_gram_tc) and the FP64
    CUDA-core path, CUDA events on the library stream."""
    import ctypes
    L = lib.L
    L.sb_gram.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32,
                          ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int]
    L.sb_gram.restype = ctypes.c_int
    I, R = int(A.shape[0]), int(A.shape[1])
    G = torch.empty(R, R, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    orig = L.splatt_b200_get_stream()
    L.splatt_b200_set_stream(C_void(st.cuda_stream))
    out = {}
    ref = torch.triu(A.double().T @ A.double())
    for name, prec in (("tensor_core_split_tf32", 1), ("fp64_cuda_core", 0)):
        ts = []
        for it in range(W + K):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(st):
                e0.record(st)
                rc = L.sb_gram(A.data_ptr(), 1, I, R, R, G.data_ptr(), prec)
                e1.record(st)
            if rc != 0:                       # internal sb_* calls return 0 on success
                raise RuntimeError("sb_gram failed with %d" % rc)
            st.synchronize()
            if it >= W:
                ts.append(e0.elapsed_time(e1) * 1e-3)
        t = float(np.mean(ts))
        err = float((G - ref).abs().max() / ref.abs().max())
        out[name] = dict(ms=t * 1e3, gbs=I * R * 4 / t / 1e9, rel_err_vs_fp64=err)
    L.splatt_b200_set_stream(C_void(orig))
    out["shape"] = [I, R]
    out["note"] = ("algorithmic bytes = rows x R x 4 (the factor read once); the split products "
                   "run 2 MMAs (M=128: hi and lo rows, N=R) per 8 rows")
    return out


def mttkrp_cpu_baseline(torch, seed, nnz, device="cuda"):
    """The reference's FP32 / 32-bit-index build (oracle/_ref) on a subset of
    the same distribution: splatt_csf_alloc (ALLMODE), then splatt_mttkrp of
    every mode, all host threads.  Returns algorithmic GB/s."""
    import oracles
    inds, vals, dims = gen_zipf_gpu(torch, C3["dims"], nnz, C3["zipf"], seed, device=device)
    nnz = int(vals.numel())
    inds = [x.cpu().numpy().astype(np.uint32) for x in inds]
    vals = vals.cpu().numpy()
    cores = os.cpu_count() or 1
    ref = oracles.Ref(32, nthreads=cores)
    h = ref.csf(inds, vals, np.array(dims, np.uint32), 2)
    R = C3["rank"]
    rng = np.random.default_rng(1)
    mats = [rng.random((d, R), dtype=np.float32) for d in dims]
    secs, alg = 0.0, 0
    for m in range(4):
        nf = [int(x) for x in h.tensor(m)["nfibs"]]
        _, t = ref.mttkrp(h, m, mats)
        secs += t
        alg += mttkrp_alg_bytes(nnz, nf, dims, m, R)
    h.free()
    return dict(value=alg / secs / 1e9, unit="GB/s", cores=cores, kind="reference",
                sample="%d-nnz subset (same Zipf(1.2) 4-mode distribution), all 4 modes, "
                       "FP32/uint32 reference build" % nnz, seconds=secs)


def bench_reference(args, world, rank):
    """--impl reference: the reference's own CPU streaming CPD (compiled
    from its sources, oracle/_ref) on a bounded sample of the same workload."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracles import have_ref
    # a step is one slice; the CPU run is bounded (about 6 s per slice on 16
    # host threads), so at most REF_MAX_STEPS slices are timed after W >= 3
    # untimed warm-up slices of the same stream; with the B200 arm's own
    # --steps/--warmup (up to REF_MAX_STEPS) both arms time the same slices
    # of the same stream from the same initial factors
    W = min(max(3, args.warmup), REF_MAX_STEPS)
    K = args.steps if args.steps is not None else 20
    K = max(1, min(K, REF_MAX_STEPS, C2["T"] - W))
    data = make_stream(args.seed, W + K)
    cb, out = cpu_baseline(data, K, have_ref(64), W, args.seed)
    errs = np.asarray(out["local_errsq"])[W:W + K]
    return {
        "impl": "reference",
        "metric": "streamed slices/sec (streaming CPD, 20000x10000x500, rank 32)",
        "value": cb["value"], "unit": "slices/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": 1e3 / cb["value"], "p99_ms": cb["p99_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; Zipf(1.1) indices, lognormal values; per rank)",
        "config": stream_config(W, K, args.seed),
        "cpu_baseline": cb,
        "local1_errsq": [float(x) for x in errs],
        "outer": [int(x) for x in np.asarray(out.get("outer", []))[W:W + K]],
        "e2e": {"value": cb["value"], "unit": "slices/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def bench_mttkrp_workload(args, world, rank, local, pg):
    import torch
    import splatt_b200 as sb
    lib32 = sb.Lib(32)
    lib32.init(local)
    K = args.steps if args.steps is not None else 5
    W = max(3, args.warmup)
    clocks = ClockSampler(local)
    dist_barrier(pg)
    clocks.start()
    mk = bench_mttkrp(args, torch, lib32, args.mttkrp_scale, K=K, W=W)
    clk = clocks.stop()
    peak, peak_kind = measured_peaks()
    tot = dist_max(pg, mk["seconds_all_modes"])
    line = {
        "metric": "CSF MTTKRP HBM GB/s (algorithmic bytes, all modes)",
        "value": world * sum(mk["alg_bytes_per_mode"]) / tot / 1e9, "unit": "GB/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": tot * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Zipf(1.2) per mode, duplicates dropped, empty slices compacted)",
        "config": {"workload": "static CSF MTTKRP, 4-mode 2Mx500Kx50Kx1K, %d nnz, rank 64, "
                               "ALLMODE CSF, all modes in turn" % mk["nnz"],
                   "l2": "inputs larger than L2 (>= 3 GB per mode)"},
        "ms_per_mode": mk["ms_per_mode"], "gbs_per_mode": mk["gbs_per_mode"],
        "roofline": {"bound": "hbm", "achieved": mk["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": mk["gbs"] / peak, "traffic": profile_traffic("mttkrp_csf_c3.md"),
                     "peak_source": peak_kind, "kernel": "k_csf_root<float,4,16,4>"},
        "gpu_launches": 4 * K, "clocks": clk, "csf_build_s": mk["csf_build_s"],
        "gram": mk.get("gram"),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = mttkrp_cpu_baseline(torch, args.seed, 16_000_000)
    return line


# --------------------------------------------------------------------------
# serving: 64 streams (50K x 20K x time, rank 32), Poisson arrivals
# --------------------------------------------------------------------------
def gen_serve_slices(torch, nstreams, nslices, seed):
    """Per stream `nslices` slices: nnz lognormal(median 50K, sigma 1.0),
    Zipf(1.1) indices over [0, 50K) x [0, 20K), lognormal(0,1) values; drawn
    on the device, returned as host arrays."""
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(seed)
    cdfs = []
    for d in (C5["I"], C5["J"]):
        w = torch.arange(1, d + 1, device=dev, dtype=torch.float64).pow_(-C5["zipf"])
        c = torch.cumsum(w, 0)
        cdfs.append(c / c[-1].clone())
    out = []
    for sidx in range(nstreams):
        perms = [torch.randperm(d, device=dev, generator=g) for d in (C5["I"], C5["J"])]
        sl = []
        for t in range(nslices):
            n = int(np.exp(np.log(C5["median"]) + C5["sigma"] * torch.randn(1, generator=g,
                                                                           device=dev).item()))
            n = max(1000, min(n, 2_000_000))
            cols = []
            for c, p, d in zip(cdfs, perms, (C5["I"], C5["J"])):
                u = torch.rand(int(n * 1.4) + 16, device=dev, dtype=torch.float64, generator=g)
                cols.append(p[torch.searchsorted(c, u, right=True).clamp_(max=d - 1)])
            key = cols[0].to(torch.int64) * C5["J"] + cols[1].to(torch.int64)
            key = torch.unique(key)[:n]
            key = key[torch.randperm(key.numel(), device=dev, generator=g)]
            i = (key // C5["J"]).cpu().numpy().astype(np.uint64)
            j = (key % C5["J"]).cpu().numpy().astype(np.uint64)
            v = torch.exp(torch.randn(key.numel(), device=dev, dtype=torch.float64,
                                      generator=g)).cpu().numpy()
            sl.append(([i, j, np.zeros(len(i), np.uint64)], v))
        out.append(sl)
    return out


def serve_accuracy(torch, lib, seed, nstreams=16, T=20):
    """The serving kernel's FP32 mode against its FP64 mode at equal inputs:
    `nstreams` planted streams of the serving shape (50K x 20K x time, rank
    32; exact rank 32 plus 10% noise, 32 blocks of 50 x 50, so the fit is
    well defined) through one scheduled launch per step (k_stream_sched, the
    kernel the serving loop replays), every stream's per-slice local fit in
    both precisions from the same initial factors."""
    import splatt_b200 as sb
    import splatt_synth as S
    data = []
    for k in range(nstreams):
        pi, pv, pd = S.planted_stream(C5["I"], C5["J"], T, C5["rank"], 50, 50, 0.7, 0.1,
                                      seed + 17 * k)
        data.append(prepare_stream(pi, pv, pd))
    dev = torch.device("cuda")
    dummy = torch.zeros(4, dtype=torch.int32, device=dev)
    fits = {}
    for prec in (sb.FP64, sb.FP32):
        vdt = torch.float64 if prec == sb.FP64 else torch.float32
        batch = sb.Batch(lib, nstreams, precision=prec, max_rank=C5["rank"])
        streams, dd = [], []
        for k, d in enumerate(data):
            st = sb.Stream(lib, 3, 2, d["dims"], C5["rank"], C5["forget"], C5["reg"], 200, prec,
                           sb.FUSED)
            sb.stream_seed(st, 500 + k)
            streams.append(st)
            dd.append([torch.from_numpy(d["inds"][m].astype(np.int32)).to(dev) for m in (0, 1)] +
                      [torch.from_numpy(d["vals"]).to(dev, vdt)])
        err = np.zeros((nstreams, T))
        for t in range(T):
            torch.cuda.synchronize()
            for st, d, (i0, i1, v) in zip(streams, data, dd):
                a, b = int(d["offs"][t]), int(d["offs"][t + 1])
                batch.add(st, [i0.data_ptr() + 4 * a, i1.data_ptr() + 4 * a, dummy.data_ptr()],
                          v.data_ptr() + v.element_size() * a, b - a, d["sdims"][t])
            batch.run()
            batch.sync()
            for k, st in enumerate(streams):
                err[k, t] = st.local_errsq()
        for st in streams:
            st.free()
        batch.free()
        fits[prec] = 1.0 - np.sqrt(np.maximum(err, 0.0))
    dfit = np.abs(fits[sb.FP32] - fits[sb.FP64])
    return {"data": "%d planted streams, 50Kx20Kx%d, exact rank 32 + 10%% noise" % (nstreams, T),
            "executor": "k_stream_sched, one launch per step (the serving kernel)",
            "fit_fp64_mean_last_slice": float(fits[sb.FP64][:, -1].mean()),
            "max_abs_dfit": float(dfit.max()), "mean_abs_dfit": float(dfit.mean()),
            "max_abs_dfit_by_slice": [float(x) for x in dfit.max(axis=0)],
            "note": "per-slice local fit, FP32 run minus FP64 run of the same stream"}


def bench_serve(args, world, rank, local, pg):
    import torch
    import splatt_b200 as sb
    lib = sb.Lib(64)
    lib.init(local)
    ns = C5["streams"]
    data = gen_serve_slices(torch, ns, args.serve_slices, args.seed + 31 * rank)
    dims = (C5["I"], C5["J"], 1 << 20)
    R = C5["rank"]

    def serve(rate, horizon, precision, saturate=False, nsat=None):
        nsat = nsat or args.serve_sat
        srv = sb.Server(lib, C5["budget"], precision=precision, max_batch=ns * args.serve_chain,
                        max_rank=R)
        ids = [srv.open(3, 2, dims, R, C5["forget"], C5["reg"], 200, seed=100 + k)
               for k in range(ns)]
        # untimed: every stream's first slice (admission, first rows drawn)
        for k in range(ns):
            inds, vals = data[k][0]
            srv.submit(ids[k], inds, vals, 0.0)
        srv.drain(1.0)
        srv.reset_stats()
        base = 0
        rng = np.random.default_rng(7 + rank)
        arr = []
        for k in range(ns):
            t, q = 0.0, 0
            while True:
                t += rng.exponential(1.0 / rate) if not saturate else 0.0
                if (not saturate and t > horizon) or (saturate and q >= nsat):
                    break
                arr.append((t, k, q % args.serve_slices))
                q += 1
        arr.sort()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nxt = 0
        while nxt < len(arr):
            now = time.perf_counter() - t0
            while nxt < len(arr) and arr[nxt][0] <= now:
                at, k, q = arr[nxt]
                inds, vals = data[k][q]
                srv.submit(ids[k], inds, vals, t0 + at)
                nxt += 1
            srv.poll(time.perf_counter())
        srv.drain(0.0)
        elapsed = time.perf_counter() - t0
        st = srv.stats()
        errs = [srv.local_errsq(i) for i in ids] if saturate else None
        srv.free()
        st["completed"] -= base
        out = dict(slices=st["completed"], seconds=elapsed, slices_per_s=st["completed"] / elapsed,
                   p50_ms=st["p50"] * 1e3, p99_ms=st["p99"] * 1e3, batches=st["batches"],
                   offered_per_s=(len(arr) / horizon) if not saturate else None)
        return out, errs

    clocks = ClockSampler(local)
    # warm (graph capture, module load) and let the group-size autotuner,
    # which keeps what it learns for the process, settle for both precisions
    for _ in range(2):
        serve(C5["rate"], 0.2, sb.FP32, saturate=True)
        serve(C5["rate"], 0.2, sb.FP64, saturate=True)
    dist_barrier(pg)
    clocks.start()
    sat32, err32 = serve(C5["rate"], 0.0, sb.FP32, saturate=True)
    clk = clocks.stop()
    load32, _ = serve(C5["rate"], args.serve_horizon, sb.FP32)
    cap = sat32["slices_per_s"]
    light_rate = 0.5 * cap / ns
    light32, _ = serve(light_rate, args.serve_horizon, sb.FP32)
    sat64, err64 = serve(C5["rate"], 0.0, sb.FP64, saturate=True)
    fit = lambda e: 1.0 - np.sqrt(np.maximum(np.asarray(e), 0.0))
    dfit = np.abs(fit(err32) - fit(err64))
    # the plain FP64 per-slice GPU path on the same slices, one stream at a time
    plain_t = []
    for k in range(min(4, ns)):
        st = sb.Stream(lib, 3, 2, dims, R, C5["forget"], C5["reg"], 200, sb.FP64, sb.PLAIN)
        sb.stream_seed(st, 100 + k)
        for q in range(args.serve_slices):
            inds, vals = data[k][q]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st.push(inds, vals)
            plain_t.append(time.perf_counter() - t0)
        st.free()
    plain = len(plain_t) / float(np.sum(plain_t))
    tot = dist_max(pg, sat32["seconds"])
    line = {
        "metric": "served slices/sec (64 concurrent streams, 50Kx20Kxtime, rank 32)",
        "value": world * sat32["slices"] / tot, "unit": "slices/s", "n_gpus": world,
        "steps": sat32["slices"], "warmup": ns, "ms_per_step": tot / max(sat32["slices"], 1) * 1e3,
        "p50_ms": load32["p50_ms"], "p99_ms": load32["p99_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 factors/MTTKRP + f64 Gram/Cholesky/solve/norms",
        "data": "synthetic (seeded; each stream cycles %d pre-generated slices)" % args.serve_slices,
        "config": {"workload": "serving loop: 64 streams, 50K x 20K x time, rank 32, frob 1e-2, "
                               "Poisson arrivals, 120 GB admission budget",
                   "executor": "scheduled cooperative launch per batch (block groups claim "
                               "per-stream slice chains), CUDA-graph replayed",
                   "batch_capacity": "%d slices per stream" % args.serve_chain},
        "saturated_fp32": sat32, "poisson_200_per_stream_fp32": load32,
        "poisson_half_capacity_fp32": light32, "saturated_fp64": sat64,
        "plain_fp64_per_slice": {"value": plain, "unit": "slices/s",
                                 "ms_per_slice": 1e3 / plain,
                                 "p50_ms": float(np.percentile(plain_t, 50) * 1e3),
                                 "p99_ms": float(np.percentile(plain_t, 99) * 1e3),
                                 "note": "one slice at a time through splatt_b200_stream_push "
                                         "(PLAIN executor), 4 streams; latency = the push"},
        "speedup_vs_plain_fp64": sat32["slices_per_s"] / plain,
        "accuracy_planted": serve_accuracy(torch, lib, args.seed + 41),
        "fit_vs_fp64": {"max_abs": float(dfit.max()), "mean_abs": float(dfit.mean()),
                        "streams": int(dfit.size),
                        "note": "local fit 1 - sqrt(relative error^2) of every stream's last "
                                "served slice (slice %d of the stream), saturated FP32 run minus "
                                "saturated FP64 run, same slices and initial factors"
                                % (args.serve_sat + 1)},
        "clocks": clk,
    }
    return line


# --------------------------------------------------------------------------
# batched: 256 heterogeneous streams, one scheduled launch per step (one
# slice of every stream), FP32 factors + FP64 solve
# --------------------------------------------------------------------------
C4 = dict(streams=256, dim_lo=1_000, dim_hi=200_000, ranks=(8, 16, 32, 64), median=40_000,
          sigma=1.0, nnz_lo=1_000, nnz_hi=2_000_000, zipf=1.1, reg=1e-2, forget=0.95)


def gen_batch_streams(torch, nslices, seed):
    """Per stream: dims I, J ~ U[1K, 200K], rank from {8, 16, 32, 64}, and
    `nslices` slices (nnz lognormal(median 40K, sigma 1) clipped to [1K, 2M],
    Zipf(1.1) coordinates with scattered hot ranks, lognormal(0, 1) values),
    kept on the device as int32 / float32."""
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(seed)
    rng = np.random.default_rng(seed)
    out = []
    for k in range(C4["streams"]):
        I = int(rng.integers(C4["dim_lo"], C4["dim_hi"] + 1))
        J = int(rng.integers(C4["dim_lo"], C4["dim_hi"] + 1))
        R = int(rng.choice(C4["ranks"]))
        samp = []
        for d in (I, J):
            w = torch.arange(1, d + 1, device=dev, dtype=torch.float64).pow_(-C4["zipf"])
            c = torch.cumsum(w, 0)
            samp.append((c / c[-1].clone(), torch.randperm(d, device=dev, generator=g)))
        sl = []
        for t in range(nslices):
            n = int(np.exp(np.log(C4["median"]) + C4["sigma"] * rng.standard_normal()))
            n = max(C4["nnz_lo"], min(n, C4["nnz_hi"]))
            cols = []
            for (c, p), d in zip(samp, (I, J)):
                u = torch.rand(int(n * 1.4) + 16, device=dev, dtype=torch.float64, generator=g)
                cols.append(p[torch.searchsorted(c, u, right=True).clamp_(max=d - 1)])
            key = torch.unique(cols[0].to(torch.int64) * J + cols[1].to(torch.int64))[:n]
            key = key[torch.randperm(key.numel(), device=dev, generator=g)]
            i0 = (key // J).to(torch.int32)
            i1 = (key % J).to(torch.int32)
            v = torch.exp(torch.randn(key.numel(), device=dev, dtype=torch.float64,
                                      generator=g)).to(torch.float32)
            sd = (int(i0.max()) + 1, int(i1.max()) + 1, 1)
            sl.append((i0, i1, v, sd))
        out.append(dict(I=I, J=J, R=R, slices=sl))
    return out


def bench_batch(args, world, rank, local, pg):
    import torch
    import splatt_b200 as sb
    lib = sb.Lib(64)
    lib.init(local)
    K = args.steps if args.steps is not None else 3
    W = max(3, args.warmup)
    data = gen_batch_streams(torch, W + K, args.seed + 131 * rank)
    ns = len(data)
    batch = sb.Batch(lib, ns, precision=sb.FP32, max_rank=64)
    streams = []
    for k, d in enumerate(data):
        st = sb.Stream(lib, 3, 2, (d["I"], d["J"], 1 << 20), d["R"], C4["forget"], C4["reg"], 200,
                       sb.FP32, sb.FUSED)
        sb.stream_seed(st, 1000 + k)
        streams.append(st)
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    L = lib.L
    cs = torch.cuda.Stream()
    orig = L.splatt_b200_get_stream()
    L.splatt_b200_set_stream(C_void(cs.cuda_stream))

    def stage(t):
        for st, d in zip(streams, data):
            i0, i1, v, sd = d["slices"][t]
            batch.add(st, [i0.data_ptr(), i1.data_ptr(), dummy.data_ptr()], v.data_ptr(),
                      v.numel(), sd)

    clocks = ClockSampler(local)
    times, nnz_steps = [], []
    for t in range(W + K):
        stage(t)                                # host: new rows drawn, args staged
        torch.cuda.synchronize()
        if t == W:
            dist_barrier(pg)
            clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(cs):
            e0.record(cs)
            batch.run()
            e1.record(cs)
        batch.sync()
        if t >= W:
            times.append(e0.elapsed_time(e1) * 1e-3)
            nnz_steps.append(sum(d["slices"][t][2].numel() for d in data))
    clk = clocks.stop()
    group = batch.last_group()
    L.splatt_b200_set_stream(C_void(orig))
    outs = [st.stats()[0] for st in streams]
    for st in streams:
        st.free()
    batch.free()
    tot = dist_max(pg, float(np.sum(times)))
    ranks = [d["R"] for d in data]
    line = {
        "metric": "batched slices/sec (256 heterogeneous streams, one scheduled launch per step)",
        "value": world * ns * K / tot, "unit": "slices/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": tot / K * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factors/MTTKRP + f64 Gram/Cholesky/solve/norms",
        "data": "synthetic (seeded; per stream dims U[1K,200K], rank in {8,16,32,64}, slice nnz "
                "lognormal median 40K clipped [1K,2M], Zipf(1.1), lognormal values)",
        "config": {"workload": "256 streams x one slice each per launch, FP32 mode",
                   "executor": "k_stream_sched, one cooperative launch per step, CUDA graph",
                   "group_blocks": group, "ranks": {str(r): ranks.count(r) for r in C4["ranks"]},
                   "mean_slice_nnz": float(np.mean(nnz_steps) / ns),
                   "l2": "inputs larger than L2 (~%.0f GB of stream state)" % (
                       sum((d["I"] + d["J"]) * d["R"] * 4 * 6 for d in data) / 1e9)},
        "outer_iterations_last_step": {"max": int(max(outs)), "mean": float(np.mean(outs))},
        "gpu_launches": K,
        "clocks": clk,
    }
    return line


# --------------------------------------------------------------------------
# plain CPD-ALS: 1000 x 800 x 600, 500K uniform nonzeros, rank 16, 20
# iterations, FP64, TWOMODE CSF (the reference's CPU-runnable case)
# --------------------------------------------------------------------------
C1 = dict(dims=(1000, 800, 600), nnz=500_000, rank=16, its=20)


def count_launches(torch, fn):
    """Kernels of this library launched by one untimed call of fn (CUPTI
    activity records through torch.profiler)."""
    from torch.profiler import profile, ProfilerActivity
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    n = 0
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA and ("sb::" in e.name or
                                                                "k_" in e.name):
            n += 1
    return n


def bench_cpd(args, world, rank, local, pg):
    import torch
    import splatt_b200 as sb
    import splatt_synth as S
    R, its = C1["rank"], C1["its"]
    inds, vals, dims = S.uniform_tensor(list(C1["dims"]), C1["nnz"], seed=args.seed + 97 * rank)
    nnz = len(vals)
    lib = sb.Lib(64)
    lib.init(local)
    K = args.steps if args.steps is not None else 5
    W = max(3, args.warmup)
    csf = lib.csf_convert(inds, vals, sb.CSF_TWOMODE)
    # per-iteration algorithmic bytes: one MTTKRP per mode on the CSF that
    # serves it, plus the factor update (read M, write A), Gram and
    # normalisation passes (~4 passes over each factor)
    trees = [csf.tree(t) for t in range(2)]
    per_it = 0
    for m in range(3):
        t = 1 if (m == int(trees[0]["dim_perm"][2])) else 0
        nf = [int(x) for x in trees[t]["nfibs"]]
        per_it += mttkrp_alg_bytes(nnz, nf, list(dims), m, R, s=8, x=4)
        per_it += 4 * int(dims[m]) * R * 8
    clocks = ClockSampler(local)
    for _ in range(W):
        lib.cpd(csf, R, niters=its, tol=0.0, seed=args.seed)
    dist_barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    ts, fit = [], None
    for _ in range(K):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = lib.cpd(csf, R, niters=its, tol=0.0, seed=args.seed)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
        fit = res["fit"]
    clk = clocks.stop()
    t = dist_max(pg, float(np.mean(ts)))
    # end to end: host COO -> splatt_csf_convert (device build) -> splatt_cpd
    te = []
    for _ in range(max(1, K // 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c2 = lib.csf_convert(inds, vals, sb.CSF_TWOMODE)
        lib.cpd(c2, R, niters=its, tol=0.0, seed=args.seed)
        torch.cuda.synchronize()
        te.append(time.perf_counter() - t0)
        c2.free()
    tee = dist_max(pg, float(np.mean(te)))
    peak, peak_kind = measured_peaks()
    line = {
        "metric": "CPD-ALS iterations/sec (1000x800x600, 500K nnz, rank 16, FP64)",
        "value": world * its / t, "unit": "iterations/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, uniform coordinates, distinct, every slice non-empty)",
        "config": {"workload": "CPD-ALS, 3-mode 1000x800x600, %d nnz, rank 16, 20 iterations, "
                               "tol 0, TWOMODE CSF" % nnz,
                   "step": "one splatt_cpd call of 20 iterations",
                   "l2": "tensor and factors are L2-resident (the whole problem is ~20 MB)"},
        "fit": fit,
        "e2e": {"value": world * its / tee, "unit": "iterations/s",
                "h2d_bytes_per_step": int(nnz * (3 * 8 + 8)),
                "d2h_bytes_per_step": int(sum(dims) * R * 8 + R * 8),
                "path": "splatt_csf_convert from host COO + splatt_cpd (factors back to host)"},
        "roofline": {"bound": "hbm", "achieved": per_it * its / t / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": per_it * its / t / 1e9 / peak, "traffic": None,
                     "peak_source": peak_kind,
                     "note": "per-iteration algorithmic bytes (3 MTTKRPs + ~4 factor passes per "
                             "mode) / iteration time; the problem fits L2 and each iteration "
                             "is ~20 short launches, so it is launch- and latency-bound"},
        "gpu_launches": count_launches(torch, lambda: lib.cpd(csf, R, niters=its, tol=0.0,
                                                               seed=args.seed)),
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        import oracles
        cores = os.cpu_count() or 1
        if oracles.have_ref(64):
            ref = oracles.Ref(64, nthreads=cores).cpd(inds, vals, dims, R, its, 0.0, args.seed)
            line["cpu_baseline"] = dict(value=its / ref["secs"], unit="iterations/s", cores=cores,
                                        kind="reference", sample="the full workload (20 "
                                        "iterations), splatt_cpd timed inside the reference",
                                        fit=ref["fit"])
    csf.free()
    return line


def main():
    args = parse_args()
    world, rank, local, pg = dist_init(args.gpus)
    if args.impl == "reference":
        line = bench_reference(args, world, rank)
    elif args.workload == "mttkrp":
        line = bench_mttkrp_workload(args, world, rank, local, pg)
    elif args.workload == "serve":
        line = bench_serve(args, world, rank, local, pg)
    elif args.workload == "cpd":
        line = bench_cpd(args, world, rank, local, pg)
    elif args.workload == "batch":
        line = bench_batch(args, world, rank, local, pg)
    else:
        line = bench_stream(args, world, rank, local, pg)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
