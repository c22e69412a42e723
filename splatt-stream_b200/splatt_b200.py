"""ctypes binding of libsplatt_b200.so (the C ABI declared in
include/splatt_b200.h) for tests, the bench and Python callers.

The binding only marshals numpy arrays; all computation happens in the
library's CUDA kernels.  Loading fails loudly when the shared library is
missing: there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATHS = {64: os.path.join(HERE, "libsplatt_b200.so"),
             32: os.path.join(HERE, "libsplatt_b200_w32.so")}

SPLATT_SUCCESS = 1
SPLATT_ERROR_BADINPUT = 2
SPLATT_ERROR_NOMEMORY = 3
SPLATT_ERROR_DEVICE = 4

OPT = dict(NTHREADS=0, TOLERANCE=1, REGULARIZE=2, NITER=3, VERBOSITY=4, RANDSEED=5,
           CSF_ALLOC=6, TILE=7, TILELEVEL=8, PRIVTHRESH=9, DECOMP=10, COMM=11)
NOPTIONS = 12
CSF_ONEMODE, CSF_TWOMODE, CSF_ALLMODE = 0, 1, 2
NOTILE, DENSETILE = 0, 1
FP64, FP32 = 0, 1
PLAIN, FUSED = 0, 1
PROX_MAXCOLNORM, PROX_MAXCOLNORM_NONNEG, PROX_LASSO, PROX_ROWSIMP = 0, 1, 2, 3
PROX_NTF_LASSO, PROX_NTF_FROB, PROX_COLSIMP = 4, 5, 6

_libc = C.CDLL(None)


def srand(seed):
    """Seed glibc rand(), which SPLATT's factor initialisation draws from."""
    _libc.srand(C.c_uint(seed))


class SplattError(RuntimeError):
    pass


def _types(width):
    it = C.c_uint64 if width == 64 else C.c_uint32
    vt = C.c_double if width == 64 else C.c_float
    return it, vt


def _structs(width):
    it, vt = _types(width)

    class CsfSparsity(C.Structure):
        _fields_ = [("nfibs", it * 8), ("fptr", C.POINTER(it) * 8),
                    ("fids", C.POINTER(it) * 8), ("vals", C.POINTER(vt))]

    class Csf(C.Structure):
        _fields_ = [("nnz", it), ("nmodes", it), ("dims", it * 8), ("dim_perm", it * 8),
                    ("dim_iperm", it * 8), ("which_tile", C.c_int), ("ntiles", it),
                    ("ntiled_modes", it), ("tile_dims", it * 8),
                    ("pt", C.POINTER(CsfSparsity)), ("dev", C.c_void_p)]

    class Kruskal(C.Structure):
        _fields_ = [("rank", it), ("factors", C.POINTER(vt) * 8), ("lam", C.POINTER(vt)),
                    ("nmodes", it), ("dims", it * 8), ("fit", C.c_double)]

    class Constraint(C.Structure):
        _fields_ = [("solve_type", C.c_int), ("row_separable", C.c_bool),
                    ("sparsity_inducing", C.c_bool), ("data", C.c_void_p),
                    ("description", C.c_char * 256)] + \
                   [(n, C.c_void_p) for n in ("init", "gram", "prox", "clsd", "post", "free")]

    class CpdOpts(C.Structure):
        _fields_ = [("tolerance", vt), ("max_iterations", it), ("inner_tolerance", vt),
                    ("max_inner_iterations", it), ("constraints", C.POINTER(Constraint) * 8),
                    ("chunk_sizes", it * 8)]

    return CsfSparsity, Csf, Kruskal, CpdOpts


def coord_struct(width):
    """splatt_coord (include/splatt/coord.h): nmodes, dims, nnz, ind, vals,
    tiled, indmap."""
    it, vt = _types(width)

    class Coord(C.Structure):
        _fields_ = [("nmodes", it), ("dims", it * 8), ("nnz", it),
                    ("ind", C.POINTER(it) * 8), ("vals", C.POINTER(vt)),
                    ("tiled", C.c_int), ("indmap", C.POINTER(it) * 8)]

    return Coord


class CsfSet:
    """CSF tree(s) owned by the library; freed with .free() or on GC."""

    def __init__(self, lib, ptr, opts, count):
        self.lib, self.ptr, self.opts, self.count = lib, ptr, opts, count

    def ntiles(self, t):
        return int(self.ptr[t].ntiles)

    def tree(self, t, tile=0):
        """Host mirror of tile `tile` of tree `t` (SPLATT's csf_sparsity);
        absent arrays of an empty tile read as [0] / empty."""
        c = self.ptr[t]
        n = int(c.nmodes)
        pt = c.pt[tile]
        nf = [int(pt.nfibs[l]) for l in range(n)]
        idt = self.lib.idx_dtype

        def arr(p, k):
            if not bool(p):
                return np.zeros(k, idt)
            return np.ctypeslib.as_array(p, (k,)).astype(idt).copy() if k else np.zeros(0, idt)
        fptr, fids = [], []
        for l in range(n):
            fptr.append(arr(pt.fptr[l], nf[l] + 1) if l < n - 1 else None)
            fids.append(arr(pt.fids[l], nf[l]) if bool(pt.fids[l]) else None)
        vals = (np.ctypeslib.as_array(pt.vals, (nf[n - 1],)).copy() if bool(pt.vals) and nf[n - 1]
                else np.zeros(0, self.lib.val_dtype))
        return dict(nfibs=np.array(nf), dim_perm=np.array([int(c.dim_perm[l]) for l in range(n)]),
                    fptr=fptr, fids=fids, vals=vals, root_null=not bool(pt.fids[0]),
                    dims=np.array([int(c.dims[m]) for m in range(n)]),
                    tile_dims=np.array([int(c.tile_dims[m]) for m in range(n)]))

    def free(self):
        if self.ptr is not None:
            self.lib.L.splatt_free_csf(self.ptr, self.opts)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Lib:
    """The loaded library at one index/value width (64 default, 32)."""

    def __init__(self, width=64, path=None):
        path = path or LIB_PATHS[width]
        if not os.path.exists(path):
            raise SplattError("libsplatt_b200 not built: %s (run splatt-stream_b200/build.py)" % path)
        self.width = width
        self.path = path
        self.L = L = C.CDLL(path)
        self.it, self.vt = _types(width)
        self.idx_dtype = np.uint64 if width == 64 else np.uint32
        self.val_dtype = np.float64 if width == 64 else np.float32
        self.CsfSparsity, self.Csf, self.Kruskal, self.CpdOpts = _structs(width)
        self.Coord = coord_struct(width)
        it, vt = self.it, self.vt
        PD = C.POINTER(C.c_double)
        L.splatt_default_opts.restype = PD
        L.splatt_free_opts.argtypes = [PD]
        L.splatt_csf_convert.argtypes = [it, it, C.POINTER(C.POINTER(it)), C.POINTER(vt),
                                         C.POINTER(C.POINTER(self.Csf)), PD]
        L.splatt_csf_convert.restype = C.c_int
        L.splatt_free_csf.argtypes = [C.POINTER(self.Csf), PD]
        L.splatt_mttkrp.argtypes = [it, it, C.POINTER(self.Csf), C.POINTER(C.POINTER(vt)),
                                    C.POINTER(vt), PD]
        L.splatt_mttkrp.restype = C.c_int
        L.splatt_alloc_cpd.argtypes = [C.POINTER(self.Csf), it]
        L.splatt_alloc_cpd.restype = C.POINTER(self.Kruskal)
        L.splatt_free_cpd.argtypes = [C.POINTER(self.Kruskal)]
        L.splatt_alloc_cpd_opts.restype = C.POINTER(self.CpdOpts)
        L.splatt_free_cpd_opts.argtypes = [C.POINTER(self.CpdOpts)]
        L.splatt_cpd.argtypes = [C.POINTER(self.Csf), it, C.POINTER(self.CpdOpts), C.c_void_p,
                                 C.POINTER(self.Kruskal)]
        L.splatt_cpd.restype = C.c_int
        L.splatt_csf_frobsq.argtypes = [C.POINTER(self.Csf)]
        L.splatt_csf_frobsq.restype = vt
        L.splatt_b200_init.argtypes = [C.c_int]
        L.splatt_b200_init.restype = C.c_int
        L.splatt_b200_get_stream.restype = C.c_void_p
        L.splatt_b200_set_stream.argtypes = [C.c_void_p]
        L.splatt_b200_error_string.restype = C.c_char_p
        L.splatt_b200_mttkrp_device.argtypes = [it, it, C.POINTER(self.Csf), PD,
                                                C.POINTER(C.c_void_p), it, C.c_void_p, it, C.c_int]
        L.splatt_b200_mttkrp_device.restype = C.c_int
        L.splatt_b200_csf_set_precision.argtypes = [C.POINTER(self.Csf), PD, C.c_int]
        L.splatt_b200_csf_set_precision.restype = C.c_int
        L.sb_sync.restype = C.c_int

    # ---- helpers -------------------------------------------------------------
    def check(self, rc, what):
        if rc != SPLATT_SUCCESS:
            raise SplattError("%s failed with %d (%s)" % (what, rc,
                              self.L.splatt_b200_error_string().decode()))

    def init(self, device=0):
        self.check(self.L.splatt_b200_init(device), "splatt_b200_init")

    def opts(self, **kw):
        p = self.L.splatt_default_opts()
        for k, v in kw.items():
            p[OPT[k.upper()]] = float(v)
        return p

    def _idx_ptrs(self, inds):
        keep = [np.ascontiguousarray(i, dtype=self.idx_dtype) for i in inds]
        arr = (C.POINTER(self.it) * len(keep))(*[k.ctypes.data_as(C.POINTER(self.it)) for k in keep])
        return keep, arr

    def _val_ptrs(self, mats):
        keep = [np.ascontiguousarray(m, dtype=self.val_dtype) for m in mats]
        arr = (C.POINTER(self.vt) * len(keep))(*[k.ctypes.data_as(C.POINTER(self.vt)) for k in keep])
        return keep, arr

    # ---- API -----------------------------------------------------------------
    def csf_convert(self, inds, vals, alloc=CSF_TWOMODE, tile=None):
        """splatt_csf_convert on host COO arrays.  tile=(nthreads, tilelevel)
        builds dense-tiled trees (SPLATT_DENSETILE)."""
        nmodes = len(inds)
        keep, arr = self._idx_ptrs(inds)
        v = np.ascontiguousarray(vals, dtype=self.val_dtype)
        opts = self.opts(csf_alloc=alloc)
        if tile is not None:
            opts[OPT["TILE"]] = float(DENSETILE)
            opts[OPT["NTHREADS"]] = float(tile[0])
            opts[OPT["TILELEVEL"]] = float(tile[1])
        out = C.POINTER(self.Csf)()
        rc = self.L.splatt_csf_convert(self.it(nmodes), self.it(len(v)), arr,
                                       v.ctypes.data_as(C.POINTER(self.vt)), C.byref(out), opts)
        self.check(rc, "splatt_csf_convert")
        count = {CSF_ONEMODE: 1, CSF_TWOMODE: 2}.get(alloc, nmodes)
        return CsfSet(self, out, opts, count)

    def mttkrp(self, csf, mode, mats):
        """splatt_mttkrp with host factor matrices; returns the output."""
        R = mats[0].shape[1]
        keep, arr = self._val_ptrs(mats)
        rows = int(csf.ptr[0].dims[mode])
        out = np.zeros((rows, R), self.val_dtype)
        rc = self.L.splatt_mttkrp(self.it(mode), self.it(R), csf.ptr, arr,
                                  out.ctypes.data_as(C.POINTER(self.vt)), csf.opts)
        self.check(rc, "splatt_mttkrp")
        return out

    def frobsq(self, csf):
        return float(self.L.splatt_csf_frobsq(csf.ptr))

    def cpd(self, csf, rank, niters=20, tol=0.0, seed=1, reg=None):
        """srand(seed); splatt_alloc_cpd; splatt_cpd -> dict(factors, lam, fit)."""
        srand(seed)
        k = self.L.splatt_alloc_cpd(csf.ptr, self.it(rank))
        o = self.L.splatt_alloc_cpd_opts()
        o.contents.max_iterations = niters
        o.contents.tolerance = tol
        try:
            rc = self.L.splatt_cpd(csf.ptr, self.it(rank), o, None, k)
            self.check(rc, "splatt_cpd")
            kk = k.contents
            n = int(kk.nmodes)
            facs = [np.ctypeslib.as_array(kk.factors[m], (int(kk.dims[m]), rank)).copy()
                    for m in range(n)]
            lam = np.ctypeslib.as_array(kk.lam, (rank,)).copy()
            return dict(factors=facs, lam=lam, fit=float(kk.fit))
        finally:
            self.L.splatt_free_cpd(k)
            self.L.splatt_free_cpd_opts(o)


def parse_stream(inds, vals, dims, stream_mode, presorted=False):
    """ParserSimple's preparation of a streamed tensor
    (src/cpd/stream/ParserSimple.cc:13-79): sort by the streamed mode then the
    following modes cyclically, relabel every other mode by first appearance.
    Returns (sorted relabelled inds, vals, slice offsets, iperm per mode)."""
    N = len(inds)
    if presorted:
        s_inds = [np.asarray(inds[m], dtype=np.uint64) for m in range(N)]
        s_vals = np.asarray(vals)
    else:
        keys = [np.asarray(inds[(stream_mode + k) % N]) for k in range(N)]
        order = np.lexsort(keys[::-1])
        s_inds = [np.asarray(inds[m])[order].astype(np.uint64) for m in range(N)]
        s_vals = np.asarray(vals)[order]
    iperm = [None] * N
    for m in range(N):
        if m == stream_mode:
            continue
        uniq, first = np.unique(s_inds[m], return_index=True)
        by_first = uniq[np.argsort(first, kind="stable")]
        lab = np.zeros(int(dims[m]), np.uint64)
        lab[by_first.astype(np.int64)] = np.arange(len(by_first), dtype=np.uint64)
        s_inds[m] = lab[s_inds[m].astype(np.int64)]
        iperm[m] = by_first
    T = int(s_inds[stream_mode].max()) + 1 if len(s_vals) else 0
    offs = np.searchsorted(s_inds[stream_mode], np.arange(T + 1, dtype=np.uint64), side="left")
    return s_inds, s_vals, offs, iperm


def _setup_stream(lib):
    L, it, vt = lib.L, lib.it, lib.vt
    L.splatt_b200_stream_alloc.argtypes = [it, it, C.POINTER(it), it, C.c_double, C.c_double,
                                           it, C.c_int, C.c_int]
    L.splatt_b200_stream_alloc.restype = C.c_void_p
    L.splatt_b200_stream_free.argtypes = [C.c_void_p]
    L.splatt_b200_stream_push.argtypes = [C.c_void_p, it, C.POINTER(C.POINTER(it)),
                                          C.POINTER(vt), C.POINTER(vt)]
    L.splatt_b200_stream_push.restype = it
    L.splatt_b200_stream_push_device.argtypes = [C.c_void_p, it, C.POINTER(C.c_void_p),
                                                 C.c_void_p, C.POINTER(it)]
    L.splatt_b200_stream_push_device.restype = C.c_int
    L.splatt_b200_stream_status.argtypes = [C.c_void_p]
    L.splatt_b200_stream_status.restype = C.c_int
    L.splatt_b200_stream_factors.argtypes = [C.c_void_p, C.POINTER(C.POINTER(vt)), C.POINTER(it)]
    L.splatt_b200_stream_factors.restype = C.c_int
    L.splatt_b200_stream_local_errsq.argtypes = [C.c_void_p]
    L.splatt_b200_stream_local_errsq.restype = C.c_double
    L.splatt_b200_stream_last_outer.argtypes = [C.c_void_p]
    L.splatt_b200_stream_last_outer.restype = it
    L.splatt_b200_stream_last_inner.argtypes = [C.c_void_p, it]
    L.splatt_b200_stream_last_inner.restype = it
    L.splatt_b200_stream_rows.argtypes = [C.c_void_p, it]
    L.splatt_b200_stream_rows.restype = it
    L.splatt_b200_stream_sync.argtypes = [C.c_void_p]
    L.splatt_b200_stream_sync.restype = C.c_int
    L.splatt_b200_stream_set_prox.argtypes = [C.c_void_p, it, C.c_int, C.c_double, it]
    L.splatt_b200_stream_set_prox.restype = C.c_int


class Stream:
    """A streaming CPD on the device (splatt_b200_stream_*)."""

    def __init__(self, lib, nmodes, stream_mode, max_dims, rank, forget=0.95, reg=1e-2,
                 max_its=200, precision=FP64, exec_=FUSED):
        if not hasattr(lib, "_stream_ready"):
            _setup_stream(lib)
            lib._stream_ready = True
        self.lib, self.N, self.sm, self.R = lib, nmodes, stream_mode, rank
        md = (lib.it * nmodes)(*[int(x) for x in max_dims])
        self.h = lib.L.splatt_b200_stream_alloc(lib.it(nmodes), lib.it(stream_mode), md,
                                                lib.it(rank), forget, reg, lib.it(max_its),
                                                precision, exec_)
        if not self.h:
            raise SplattError("splatt_b200_stream_alloc failed (%s)" %
                              lib.L.splatt_b200_error_string().decode())
        self.max_dims = [int(x) for x in max_dims]

    def push(self, inds, vals):
        """One slice as host COO; returns (outer iterations, time row)."""
        lib = self.lib
        keep, arr = lib._idx_ptrs(inds)
        v = np.ascontiguousarray(vals, dtype=lib.val_dtype)
        row = np.zeros(self.R, lib.val_dtype)
        its = lib.L.splatt_b200_stream_push(self.h, lib.it(len(v)), arr,
                                            v.ctypes.data_as(C.POINTER(lib.vt)),
                                            row.ctypes.data_as(C.POINTER(lib.vt)))
        if its == 0:
            raise SplattError("stream push failed: %d (%s)" % (
                lib.L.splatt_b200_stream_status(self.h), lib.L.splatt_b200_error_string().decode()))
        return int(its), row

    def push_device(self, dind_ptrs, dval_ptr, nnz, slice_dims):
        lib = self.lib
        arr = (C.c_void_p * self.N)(*dind_ptrs)
        sd = (lib.it * self.N)(*[int(x) for x in slice_dims])
        rc = lib.L.splatt_b200_stream_push_device(self.h, lib.it(nnz), arr, C.c_void_p(dval_ptr), sd)
        lib.check(rc, "splatt_b200_stream_push_device")

    def set_prox(self, mode, kind, multiplier=0.0, chunk_rows=0):
        """splatt_b200_stream_set_prox: PROX_MAXCOLNORM, PROX_MAXCOLNORM_NONNEG,
        PROX_ROWSIMP, or PROX_LASSO / PROX_NTF_LASSO / PROX_NTF_FROB with their
        multiplier (the last four with chunk_rows) for non-streamed mode
        `mode`."""
        self.lib.check(self.lib.L.splatt_b200_stream_set_prox(
            self.h, self.lib.it(mode), kind, float(multiplier), self.lib.it(chunk_rows)),
            "splatt_b200_stream_set_prox")

    def local_errsq(self):
        return float(self.lib.L.splatt_b200_stream_local_errsq(self.h))

    def last_outer(self):
        return int(self.lib.L.splatt_b200_stream_last_outer(self.h))

    def sync(self):
        self.lib.check(self.lib.L.splatt_b200_stream_sync(self.h), "splatt_b200_stream_sync")

    def stats(self):
        """(outer iterations, {mode: ADMM iterations}, {mode: rows}) of the
        last slice; call sync() first after push_device."""
        L, it = self.lib.L, self.lib.it
        inner = {m: int(L.splatt_b200_stream_last_inner(self.h, it(m)))
                 for m in range(self.N) if m != self.sm}
        rows = {m: int(L.splatt_b200_stream_rows(self.h, it(m))) for m in range(self.N)}
        return self.last_outer(), inner, rows

    def factors(self, nslices):
        lib = self.lib
        rows = (lib.it * self.N)()
        bufs = [np.zeros(((nslices if m == self.sm else self.max_dims[m]) + 1, self.R),
                         lib.val_dtype) for m in range(self.N)]
        arr = (C.POINTER(lib.vt) * self.N)(*[b.ctypes.data_as(C.POINTER(lib.vt)) for b in bufs])
        lib.check(lib.L.splatt_b200_stream_factors(self.h, arr, rows), "stream_factors")
        return [bufs[m][:int(rows[m])] for m in range(self.N)]

    def free(self):
        if self.h:
            self.lib.L.splatt_b200_stream_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def stream_run(lib, inds, vals, dims, stream_mode, rank, forget=0.95, reg=1e-2, max_its=200,
               seed=1, precision=FP64, exec_=FUSED, max_slices=0, errs=False, nonneg=False,
               lasso=None, rowsimp=False, ntf_lasso=None, ntf_frob=None, colsimp=False):
    """Prepare like ParserSimple, srand(seed), push every slice; returns dict
    with time rows, factors (relabelled order), outer iterations, errors.
    nonneg: the non-negative max-column-norm prox on every non-streamed mode
    (what `--con=nonneg` gives them); lasso=L: L1 with multiplier L on them
    (`--reg=l1,L`, chunked ADMM); rowsimp: each row onto the probability
    simplex (`--con=rowsimp`, chunked ADMM); ntf_lasso=L / ntf_frob=L:
    `--reg=ntf-l1,L` / `--reg=ntf-frob,L` (chunked ADMM); colsimp: each
    column onto the probability simplex (`--con=colsimp`, single-chunk ADMM)."""
    s_inds, s_vals, offs, _ = parse_stream(inds, vals, dims, stream_mode)
    T = len(offs) - 1
    if max_slices:
        T = min(T, max_slices)
    srand(seed)
    st = Stream(lib, len(inds), stream_mode, dims, rank, forget, reg, max_its, precision, exec_)
    if (nonneg or lasso is not None or rowsimp or ntf_lasso is not None or ntf_frob is not None
            or colsimp):
        for m in range(len(inds)):
            if m != stream_mode:
                if colsimp:
                    st.set_prox(m, PROX_COLSIMP)
                elif ntf_frob is not None:
                    st.set_prox(m, PROX_NTF_FROB, ntf_frob)
                elif ntf_lasso is not None:
                    st.set_prox(m, PROX_NTF_LASSO, ntf_lasso)
                elif rowsimp:
                    st.set_prox(m, PROX_ROWSIMP)
                elif lasso is not None:
                    st.set_prox(m, PROX_LASSO, lasso)
                else:
                    st.set_prox(m, PROX_MAXCOLNORM_NONNEG)
    times, outer, le = [], [], []
    for t in range(T):
        a, b = int(offs[t]), int(offs[t + 1])
        its, row = st.push([x[a:b] for x in s_inds], s_vals[a:b])
        times.append(row.astype(np.float64))
        outer.append(its)
        if errs:
            le.append(st.local_errsq())
    facs = st.factors(T)
    st.free()
    return dict(time=np.array(times), factors=facs, outer=np.array(outer),
                local_errsq=np.array(le))


Lib.stream_run = stream_run
Lib.stream_alloc = Stream


def _setup_serve(lib):
    L, it, vt = lib.L, lib.it, lib.vt
    L.splatt_b200_stream_seed.argtypes = [C.c_void_p, C.c_uint]
    L.splatt_b200_stream_bytes.argtypes = [C.c_void_p]
    L.splatt_b200_stream_bytes.restype = C.c_size_t
    L.splatt_b200_batch_alloc.argtypes = [it, C.c_int, it]
    L.splatt_b200_batch_alloc.restype = C.c_void_p
    L.splatt_b200_batch_free.argtypes = [C.c_void_p]
    L.splatt_b200_batch_add.argtypes = [C.c_void_p, C.c_void_p, it, C.POINTER(C.c_void_p),
                                        C.c_void_p, C.POINTER(it)]
    L.splatt_b200_batch_add.restype = C.c_int
    L.splatt_b200_batch_run.argtypes = [C.c_void_p]
    L.splatt_b200_batch_run.restype = C.c_int
    L.splatt_b200_batch_sync.argtypes = [C.c_void_p]
    L.splatt_b200_batch_sync.restype = C.c_int
    L.splatt_b200_batch_set_group.argtypes = [C.c_void_p, C.c_int]
    L.splatt_b200_batch_last_group.argtypes = [C.c_void_p]
    L.splatt_b200_batch_set_factor.argtypes = [C.c_void_p, C.c_int]
    L.splatt_b200_batch_last_group.restype = C.c_int
    L.splatt_b200_batch_graph_used.argtypes = [C.c_void_p]
    L.splatt_b200_batch_graph_used.restype = C.c_int
    L.splatt_b200_batch_blocks.argtypes = [C.c_void_p]
    L.splatt_b200_batch_blocks.restype = C.c_int
    L.splatt_b200_server_alloc.argtypes = [C.c_size_t, C.c_int, it, it]
    L.splatt_b200_server_alloc.restype = C.c_void_p
    L.splatt_b200_server_free.argtypes = [C.c_void_p]
    L.splatt_b200_server_open.argtypes = [C.c_void_p, it, it, C.POINTER(it), it, C.c_double,
                                          C.c_double, it, C.c_uint]
    L.splatt_b200_server_open.restype = C.c_int
    L.splatt_b200_server_close.argtypes = [C.c_void_p, C.c_int]
    L.splatt_b200_server_close.restype = C.c_int
    L.splatt_b200_server_admitted.argtypes = [C.c_void_p, C.c_int]
    L.splatt_b200_server_admitted.restype = C.c_int
    L.splatt_b200_server_submit.argtypes = [C.c_void_p, C.c_int, it, C.POINTER(C.POINTER(it)),
                                            C.POINTER(vt), C.c_double]
    L.splatt_b200_server_submit.restype = C.c_int
    L.splatt_b200_server_poll.argtypes = [C.c_void_p, C.c_double]
    L.splatt_b200_server_poll.restype = it
    L.splatt_b200_server_drain.argtypes = [C.c_void_p, C.c_double]
    L.splatt_b200_server_drain.restype = C.c_int
    L.splatt_b200_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.POINTER(it), C.POINTER(it)]
    L.splatt_b200_server_stats.restype = C.c_int
    L.splatt_b200_server_stream.argtypes = [C.c_void_p, C.c_int]
    L.splatt_b200_server_stream.restype = C.c_void_p
    L.splatt_b200_server_reset_stats.argtypes = [C.c_void_p]
    L.splatt_b200_server_used.argtypes = [C.c_void_p]
    L.splatt_b200_server_used.restype = C.c_size_t
    L.splatt_b200_server_inflight.argtypes = [C.c_void_p]
    L.splatt_b200_server_inflight.restype = it


def _ensure(lib):
    if not hasattr(lib, "_stream_ready"):
        _setup_stream(lib)
        lib._stream_ready = True
    if not hasattr(lib, "_serve_ready"):
        _setup_serve(lib)
        lib._serve_ready = True


class Batch:
    """splatt_b200_batch: slices of many streams (several per stream allowed,
    run in the order added) updated by one scheduled launch."""

    def __init__(self, lib, max_slices, precision=FP64, max_rank=64):
        _ensure(lib)
        self.lib = lib
        self.h = lib.L.splatt_b200_batch_alloc(lib.it(max_slices), precision, lib.it(max_rank))
        if not self.h:
            raise SplattError("splatt_b200_batch_alloc failed")

    def add(self, stream, dind_ptrs, dval_ptr, nnz, slice_dims):
        lib = self.lib
        arr = (C.c_void_p * stream.N)(*dind_ptrs)
        sd = (lib.it * stream.N)(*[int(x) for x in slice_dims])
        lib.check(lib.L.splatt_b200_batch_add(self.h, stream.h, lib.it(nnz), arr,
                                              C.c_void_p(dval_ptr), sd), "batch_add")

    def run(self):
        self.lib.check(self.lib.L.splatt_b200_batch_run(self.h), "batch_run")

    def sync(self):
        self.lib.check(self.lib.L.splatt_b200_batch_sync(self.h), "batch_sync")

    def set_group(self, g):
        self.lib.L.splatt_b200_batch_set_group(self.h, int(g))

    def last_group(self):
        return int(self.lib.L.splatt_b200_batch_last_group(self.h))

    def set_factor(self, f):
        self.lib.L.splatt_b200_batch_set_factor(self.h, int(f))

    def graph_used(self):
        return int(self.lib.L.splatt_b200_batch_graph_used(self.h))

    def blocks(self):
        return int(self.lib.L.splatt_b200_batch_blocks(self.h))

    def free(self):
        if self.h:
            self.lib.L.splatt_b200_batch_free(self.h)
            self.h = None


class Server:
    """splatt_b200_server: admission by HBM budget + continuous batching."""

    def __init__(self, lib, budget_bytes, precision=FP32, max_batch=64, max_rank=64):
        _ensure(lib)
        self.lib = lib
        self.h = lib.L.splatt_b200_server_alloc(int(budget_bytes), precision, lib.it(max_batch),
                                                lib.it(max_rank))
        if not self.h:
            raise SplattError("splatt_b200_server_alloc failed")

    def open(self, nmodes, stream_mode, max_dims, rank, forget=0.95, reg=1e-2, max_its=200,
             seed=1):
        lib = self.lib
        md = (lib.it * nmodes)(*[int(x) for x in max_dims])
        sid = lib.L.splatt_b200_server_open(self.h, lib.it(nmodes), lib.it(stream_mode), md,
                                            lib.it(rank), forget, reg, lib.it(max_its), seed)
        if sid < 0:
            raise SplattError("server_open failed")
        return sid

    def close(self, sid):
        self.lib.check(self.lib.L.splatt_b200_server_close(self.h, sid), "server_close")

    def admitted(self, sid):
        return bool(self.lib.L.splatt_b200_server_admitted(self.h, sid))

    def submit(self, sid, inds, vals, arrival):
        lib = self.lib
        keep, arr = lib._idx_ptrs(inds)
        v = np.ascontiguousarray(vals, dtype=lib.val_dtype)
        lib.check(lib.L.splatt_b200_server_submit(self.h, sid, lib.it(len(v)), arr,
                                                  v.ctypes.data_as(C.POINTER(lib.vt)), arrival),
                  "server_submit")

    def poll(self, now):
        return int(self.lib.L.splatt_b200_server_poll(self.h, now))

    def drain(self, now=0.0):
        self.lib.check(self.lib.L.splatt_b200_server_drain(self.h, now), "server_drain")

    def stats(self):
        lib = self.lib
        p50, p99 = C.c_double(), C.c_double()
        done, nb = lib.it(), lib.it()
        lib.L.splatt_b200_server_stats(self.h, C.byref(p50), C.byref(p99), C.byref(done),
                                       C.byref(nb))
        return dict(p50=p50.value, p99=p99.value, completed=int(done.value), batches=int(nb.value))

    def stream_factors(self, sid, nslices, N, max_dims, R):
        """Factors of stream sid (its StreamCPD state) via splatt_b200_stream_factors."""
        lib = self.lib
        h = lib.L.splatt_b200_server_stream(self.h, sid)
        rows = (lib.it * N)()
        bufs = [np.zeros(((nslices if m == N - 1 else int(max_dims[m])) + 1, R), lib.val_dtype)
                for m in range(N)]
        arr = (C.POINTER(lib.vt) * N)(*[b.ctypes.data_as(C.POINTER(lib.vt)) for b in bufs])
        lib.check(lib.L.splatt_b200_stream_factors(h, arr, rows), "stream_factors")
        return [bufs[m][:int(rows[m])] for m in range(N)]

    def local_errsq(self, sid):
        """Local error^2 of the last slice served to stream sid
        (splatt_b200_stream_local_errsq on its handle); call after drain()."""
        L = self.lib.L
        return float(L.splatt_b200_stream_local_errsq(L.splatt_b200_server_stream(self.h, sid)))

    def used(self):
        return int(self.lib.L.splatt_b200_server_used(self.h))

    def inflight(self):
        """Slices of the launched batch the GPU is still running."""
        return int(self.lib.L.splatt_b200_server_inflight(self.h))

    def reset_stats(self):
        self.lib.L.splatt_b200_server_reset_stats(self.h)

    def free(self):
        if self.h:
            self.lib.L.splatt_b200_server_free(self.h)
            self.h = None


def stream_seed(stream, seed):
    _ensure(stream.lib)
    stream.lib.L.splatt_b200_stream_seed(stream.h, C.c_uint(seed))
