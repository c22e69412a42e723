"""Seeded synthetic sparse tensors with the shapes and value distributions of
the SPLATT-stream workloads (no public dataset is involved).

Every generator returns ``(inds, vals, dims)`` with ``inds`` a list of
per-mode uint64 index arrays, ``vals`` float64 and ``dims`` uint64.  Duplicate
coordinates are dropped (first occurrence kept), as the workloads require; the
reference's ``tt_remove_dups`` would sum them instead, so inputs are
deduplicated before any implementation sees them.
"""
import numpy as np


def _dedup(keys):
    """Indices of the first occurrence of each distinct key, in input order."""
    _, first = np.unique(keys, return_index=True)
    first.sort()
    return first


def _zipf_sampler(n, s, rng):
    """Bounded Zipf(s) over [0, n): P(k) ~ (k+1)^-s, hot ranks scattered by a
    seeded permutation of the index space."""
    w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    perm = rng.permutation(n).astype(np.uint64)

    def draw(k):
        u = rng.random(k)
        r = np.searchsorted(cdf, u, side="right")
        return perm[np.minimum(r, n - 1)]
    return draw


def uniform_tensor(dims, nnz, seed, nonempty=True):
    """Distinct coordinates uniform per mode, values U(0,1]; when `nonempty`,
    redraw until every slice of every mode is non-empty (the plain CPD-ALS
    workload: 1000x800x600, 500,000 nonzeros)."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, dtype=np.uint64)
    while True:
        got = np.zeros((len(dims), 0), np.uint64)
        while got.shape[1] < nnz:
            need = int((nnz - got.shape[1]) * 1.3) + 16
            cand = np.stack([rng.integers(0, int(d), need, dtype=np.uint64) for d in dims])
            allc = np.concatenate([got, cand], axis=1)
            key = np.zeros(allc.shape[1], np.uint64)
            for m, d in enumerate(dims):
                key = key * np.uint64(d) + allc[m]
            got = allc[:, _dedup(key)]
        got = got[:, :nnz]
        if not nonempty or all(len(np.unique(got[m])) == int(d) for m, d in enumerate(dims)):
            break
    vals = 1.0 - rng.random(nnz)            # (0, 1]
    return [got[m].copy() for m in range(len(dims))], vals, dims


def stream_tensor(I, J, T, total_nnz, median, sigma, zipf_s, seed, time_mode=2,
                  value_dist="lognormal", min_slice=1, max_slice=None, sort_slices=False,
                  max_t=None, exact=False):
    """A 3-mode tensor whose `time_mode` is streamed: slice t has
    round(lognormal(ln median, sigma)) nonzeros rescaled so the total is about
    `total_nnz` (clipped to [min_slice, max_slice]); the two other modes are
    bounded Zipf(zipf_s) over [0, I) and [0, J); values lognormal(0, 1).
    Every time slice is non-empty.  Returns (inds, vals, dims).

    Duplicate coordinates within a slice are dropped.  By default a slice
    keeps the distinct coordinates among one draw of 1.6x its target count,
    so heavy slices come out below target; `exact` draws again until every
    slice holds exactly its target count of distinct coordinates (the total
    is then `total_nnz` up to rounding) and draws each slice's values right
    after its coordinates, so the first k slices are the same whatever
    `max_t` is."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.normal(np.log(median), sigma, T))
    if total_nnz:
        sizes *= total_nnz / sizes.sum()
    sizes = np.maximum(np.rint(sizes).astype(np.int64), min_slice)
    if max_slice:
        sizes = np.minimum(sizes, max_slice)
    zi = _zipf_sampler(I, zipf_s, rng)
    zj = _zipf_sampler(J, zipf_s, rng)
    ii, jj, tt, vv = [], [], [], []
    for t in range(T if max_t is None else min(T, max_t)):
        n = int(sizes[t])
        a = zi(int(n * 1.6) + 8)
        b = zj(len(a))
        keep = _dedup(a * np.uint64(J) + b)[:n]
        a, b = a[keep], b[keep]
        while exact and len(a) < n:
            more = max(2 * (n - len(a)), 1024)
            a = np.concatenate([a, zi(more)])
            b = np.concatenate([b, zj(more)])
            keep = _dedup(a * np.uint64(J) + b)[:n]
            a, b = a[keep], b[keep]
        if sort_slices:
            o = np.argsort(a * np.uint64(J) + b, kind="stable")
            a, b = a[o], b[o]
        ii.append(a); jj.append(b); tt.append(np.full(len(a), t, np.uint64))
        if exact:
            vv.append(rng.lognormal(0.0, 1.0, len(a)) if value_dist == "lognormal"
                      else 1.0 - rng.random(len(a)))
    ii = np.concatenate(ii); jj = np.concatenate(jj); tt = np.concatenate(tt)
    nnz = len(ii)
    if exact:
        vals = np.concatenate(vv)
    elif value_dist == "lognormal":
        vals = rng.lognormal(0.0, 1.0, nnz)
    else:
        vals = 1.0 - rng.random(nnz)
    other = [ii, jj]
    inds, dims = [], []
    k = 0
    for m in range(3):
        if m == time_mode:
            inds.append(tt); dims.append(T)
        else:
            inds.append(other[k]); dims.append(I if k == 0 else J); k += 1
    return inds, vals, np.asarray(dims, np.uint64)


def zipf_tensor(dims, nnz, s, seed):
    """Coordinates bounded Zipf(s) per mode independently, duplicates dropped,
    values U(0,1]; empty slices are then compacted in every mode (the
    reference's tt_remove_empty semantics: kept indices renumbered in order).
    The static-MTTKRP workload uses 2,000,000x500,000x50,000x1,000, 400M."""
    rng = np.random.default_rng(seed)
    samplers = [_zipf_sampler(int(d), s, rng) for d in dims]
    got = np.zeros((len(dims), 0), np.uint64)
    while got.shape[1] < nnz:
        need = int((nnz - got.shape[1]) * 1.5) + 16
        cand = np.stack([smp(need) for smp in samplers])
        allc = np.concatenate([got, cand], axis=1)
        key = np.zeros(allc.shape[1], dtype=object) if _bits(dims) > 63 else \
            np.zeros(allc.shape[1], np.uint64)
        if key.dtype == object:
            order = np.lexsort(allc[::-1])
            srt = allc[:, order]
            diff = np.any(srt[:, 1:] != srt[:, :-1], axis=0)
            firsts = order[np.concatenate([[True], diff])]
            firsts.sort()
            got = allc[:, firsts]
        else:
            for m, d in enumerate(dims):
                key = key * np.uint64(d) + allc[m]
            got = allc[:, _dedup(key)]
    got = got[:, :nnz]
    vals = 1.0 - rng.random(got.shape[1])
    return compact_empty([got[m].copy() for m in range(len(dims))], vals, dims)


def _bits(dims):
    return sum(int(np.ceil(np.log2(max(int(d), 2)))) for d in dims)


def compact_empty(inds, vals, dims):
    """Drop empty slices in every mode, renumbering the kept indices in
    increasing order (src/sptensor.c:190-252 tt_remove_empty)."""
    out, nd = [], []
    for m, d in enumerate(dims):
        used = np.zeros(int(d), bool)
        used[inds[m].astype(np.int64)] = True
        newid = np.cumsum(used) - 1
        out.append(newid[inds[m].astype(np.int64)].astype(np.uint64))
        nd.append(int(used.sum()))
    return out, vals, np.asarray(nd, np.uint64)


def zipf_tensor_torch(torch, dims, nnz, s, seed, device="cuda"):
    """The static-MTTKRP workload's generator on a torch device (CUDA for the
    400M-nonzero tensor): seeded bounded-Zipf(s) coordinates per mode (hot
    ranks scattered by a permutation), duplicates dropped, empty slices
    compacted in every mode (kept indices renumbered in order), values U(0,1].
    Returns (int32 index tensors, float32 values, dims after compaction).
    `nnz` is the number of distinct coordinates asked for; fewer are returned
    only when the index space cannot hold that many."""
    dev = torch.device(device)
    g = torch.Generator(device=dev).manual_seed(seed)
    samplers = []
    for d in dims:
        w = torch.arange(1, d + 1, device=dev, dtype=torch.float64).pow_(-s)
        cdf = torch.cumsum(w, 0)
        cdf /= cdf[-1].clone()
        perm = torch.randperm(d, device=dev, generator=g)
        samplers.append((cdf, perm))
    # two int64 keys: (mode 0, mode 1) and (mode 2, mode 3)
    hi_mult = dims[1]
    lo_mult = dims[3]
    keys_hi = torch.empty(0, dtype=torch.int64, device=dev)
    keys_lo = torch.empty(0, dtype=torch.int64, device=dev)
    draw = int(nnz * 1.15)
    for _ in range(24):
        cols = []
        for (cdf, perm), d in zip(samplers, dims):
            u = torch.rand(draw, device=dev, dtype=torch.float64, generator=g)
            r = torch.searchsorted(cdf, u, right=True).clamp_(max=d - 1)
            cols.append(perm[r].to(torch.int64))
            del u, r
        keys_hi = torch.cat([keys_hi, cols[0] * hi_mult + cols[1]])
        keys_lo = torch.cat([keys_lo, cols[2] * lo_mult + cols[3]])
        del cols
        o = torch.sort(keys_lo, stable=True).indices
        keys_hi, keys_lo = keys_hi[o], keys_lo[o]
        o = torch.sort(keys_hi, stable=True).indices
        keys_hi, keys_lo = keys_hi[o], keys_lo[o]
        del o
        dup = torch.zeros(keys_hi.numel(), dtype=torch.bool, device=dev)
        dup[1:] = (keys_hi[1:] == keys_hi[:-1]) & (keys_lo[1:] == keys_lo[:-1])
        keys_hi, keys_lo = keys_hi[~dup], keys_lo[~dup]
        del dup
        have = keys_hi.numel()
        if have >= nnz:
            break
        draw = int((nnz - have) * 2.0) + 1024
    nnz = min(nnz, keys_hi.numel())
    pick = torch.randperm(keys_hi.numel(), device=dev, generator=g)[:nnz]
    keys_hi, keys_lo = keys_hi[pick], keys_lo[pick]
    del pick
    idx = [keys_hi // hi_mult, keys_hi % hi_mult, keys_lo // lo_mult, keys_lo % lo_mult]
    del keys_hi, keys_lo
    out, nd = [], []
    for x in idx:
        u, inv = torch.unique(x, return_inverse=True)
        out.append(inv.to(torch.int32))
        nd.append(int(u.numel()))
    vals = 1.0 - torch.rand(nnz, device=dev, dtype=torch.float32, generator=g)
    return out, vals, nd


def planted_stream(I, J, T, rank, rows, cols, active, noise, seed):
    """A streamed 3-mode tensor (time = mode 3) that is exactly of rank
    `rank` up to noise: component r owns a block of `rows` rows and `cols`
    columns (drawn once, overlaps allowed) and appears in slice t with
    probability `active`, with factor entries U(0.5, 1.5) in every mode; a
    slice holds every coordinate of its active blocks, valued by the sum of
    its active components' rank-one terms, plus Gaussian noise of standard
    deviation `noise` times the values' RMS.  Every entry of an active block
    is present, so the sparse tensor itself (zeros elsewhere) has that low
    rank and a rank-`rank` factorisation has a well-defined optimum with fit
    near 1 - noise.  Returns (inds, vals, dims) with slices in time order."""
    rng = np.random.default_rng(seed)
    R = rank
    rset = [rng.choice(I, rows, replace=False).astype(np.uint64) for _ in range(R)]
    cset = [rng.choice(J, cols, replace=False).astype(np.uint64) for _ in range(R)]
    A = rng.uniform(0.5, 1.5, (I, R))
    B = rng.uniform(0.5, 1.5, (J, R))
    Cw = rng.uniform(0.5, 1.5, (T, R)) * (rng.random((T, R)) < active)
    for t in range(T):
        if not Cw[t].any():
            Cw[t, rng.integers(R)] = 1.0
    ii, jj, tt, vv = [], [], [], []
    for t in range(T):
        on = np.nonzero(Cw[t])[0]
        keys = np.unique(np.concatenate([(rset[r][:, None] * np.uint64(J) + cset[r][None, :]).ravel()
                                         for r in on]))
        i = keys // np.uint64(J)
        j = keys % np.uint64(J)
        v = (A[i.astype(np.int64)] * B[j.astype(np.int64)] * Cw[t]).sum(axis=1)
        ii.append(i); jj.append(j); tt.append(np.full(len(i), t, np.uint64)); vv.append(v)
    vals = np.concatenate(vv)
    rms = float(np.sqrt(np.mean(vals * vals)))
    vals = vals + noise * rms * rng.standard_normal(len(vals))
    return ([np.concatenate(ii), np.concatenate(jj), np.concatenate(tt)], vals,
            np.array([I, J, T], np.uint64))
