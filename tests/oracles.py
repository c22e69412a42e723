"""ctypes bindings for the two CPU oracles (test infrastructure only).

* ``Port``  -- oracle/liboracle.so, our C restatement of the SPLATT path.
* ``Ref``   -- oracle/_ref/libsplatt_ref{64,32}.so, the reference's own
  sources compiled by oracle/Makefile, driven through oracle/ref_harness.cc.

Both expose the same small surface (CSF build + arrays, CSF MTTKRP, COO
MTTKRP, CPD-ALS, streaming CPD) on numpy arrays so tests can compare any pair
of implementations.  Nothing in the product imports this module.
"""
import ctypes as C
import os
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PORT_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = {64: os.path.join(ROOT, "oracle", "_ref", "libsplatt_ref64.so"),
          32: os.path.join(ROOT, "oracle", "_ref", "libsplatt_ref32.so")}
# the SPLATT source tree (its test tensors are read where it is present; the
# oracle Makefile builds oracle/_ref from the same tree)
REF_SRC = os.environ.get("SPLATT_REF_SRC", "/root/reference")

u64 = C.c_uint64
PU = C.POINTER(C.c_uint64)
PU32 = C.POINTER(C.c_uint32)
PD = C.POINTER(C.c_double)
PF = C.POINTER(C.c_float)


def have_port():
    return os.path.exists(PORT_SO)


def have_ref(width=64):
    return os.path.exists(REF_SO[width])


class _Base:
    idx_dtype = np.uint64
    val_dtype = np.float64

    def _ptrs(self, arrs, dtype):
        ct = PU if dtype == np.uint64 else (PU32 if dtype == np.uint32 else
                                           (PD if dtype == np.float64 else PF))
        keep = [np.ascontiguousarray(a, dtype=dtype) for a in arrs]
        return keep, (ct * len(keep))(*[k.ctypes.data_as(ct) for k in keep])

    def _coo(self, inds, vals, dims):
        inds = [np.ascontiguousarray(i, dtype=self.idx_dtype) for i in inds]
        keep, pp = self._ptrs(inds, self.idx_dtype)
        d = np.ascontiguousarray(dims, dtype=self.idx_dtype)
        v = np.ascontiguousarray(vals, dtype=self.val_dtype)
        return keep, pp, d, v


# orc_prox / ref_prox numbering of the ADMM constraints' proximal operators
PROX_KINDS = {"maxcolnorm": 0, "maxcolnorm_nonneg": 1, "lasso": 2, "rowsimp": 3,
              "ntf_lasso": 4, "ntf_frob": 5, "colsimp": 6, "nonneg": 7}


def _con_args(nonneg, lasso, rowsimp, ntf_lasso, ntf_frob, colsimp=False):
    """(constraint code, multiplier) as orc_stream and ref_stream take them:
    0 none, 1 nonneg, 2 lasso, 3 row simplex, 4 ntf-l1, 5 ntf-frob,
    6 column simplex."""
    if colsimp:
        return C.c_int(6), C.c_double(0.)
    if ntf_frob is not None:
        return C.c_int(5), C.c_double(ntf_frob)
    if ntf_lasso is not None:
        return C.c_int(4), C.c_double(ntf_lasso)
    if rowsimp:
        return C.c_int(3), C.c_double(0.)
    if lasso is not None:
        return C.c_int(2), C.c_double(lasso)
    return C.c_int(1 if nonneg else 0), C.c_double(0.)


class Port(_Base):
    """Our CPU restatement (uint64 / double)."""

    def __init__(self):
        self.lib = C.CDLL(PORT_SO)
        L = self.lib
        L.orc_csf_alloc.restype = C.c_void_p
        L.orc_csf_count.restype = u64
        L.orc_csf_count.argtypes = [C.c_void_p]
        L.orc_csf_info.argtypes = [C.c_void_p, u64, PU, PU]
        L.orc_csf_level.argtypes = [C.c_void_p, u64, u64, C.c_void_p, C.c_void_p]
        L.orc_csf_vals.argtypes = [C.c_void_p, u64, C.c_void_p]
        L.orc_csf_free.argtypes = [C.c_void_p]
        L.orc_mttkrp.argtypes = [C.c_void_p, u64, u64, C.c_void_p, PD]
        L.orc_cpd.restype = C.c_double
        L.orc_stream.restype = u64
        L.orc_stream_window_errsq.restype = C.c_double

    def csf(self, inds, vals, dims, alloc_type):
        keep, pp, d, v = self._coo(inds, vals, dims)
        h = self.lib.orc_csf_alloc(u64(len(inds)), u64(len(v)), d.ctypes.data_as(PU),
                                   pp, v.ctypes.data_as(PD), C.c_int(alloc_type))
        return _CsfView(self.lib, "orc", h, len(inds), len(v), np.uint64, np.float64)

    def csf_tiled(self, inds, vals, dims, alloc_type, nthreads, tilelevel):
        """Dense-tiled CSF set: list (per tree) of lists (per tile) of dicts
        with nfibs, dim_perm, fptr, fids, vals."""
        keep, pp, d, v = self._coo(inds, vals, dims)
        L = self.lib
        L.orc_csf_alloc_tiled.restype = C.c_void_p
        L.orc_tcsf_count.restype = u64
        L.orc_tcsf_ntiles.restype = u64
        h = C.c_void_p(L.orc_csf_alloc_tiled(u64(len(inds)), u64(len(v)), d.ctypes.data_as(PU),
                                             pp, v.ctypes.data_as(PD), C.c_int(alloc_type),
                                             u64(nthreads), u64(tilelevel)))
        n = len(inds)
        out = []
        for t in range(int(L.orc_tcsf_count(h))):
            tiles = []
            for k in range(int(L.orc_tcsf_ntiles(h, u64(t)))):
                nf = np.zeros(n, np.uint64)
                dp = np.zeros(n, np.uint64)
                L.orc_tcsf_info(h, u64(t), u64(k), nf.ctypes.data_as(PU), dp.ctypes.data_as(PU))
                fptr, fids = [], []
                for l in range(n):
                    fp = np.zeros(int(nf[l]) + 1, np.uint64) if l < n - 1 else None
                    fi = np.zeros(int(nf[l]), np.uint64)
                    L.orc_tcsf_level(h, u64(t), u64(k), u64(l),
                                     fp.ctypes.data_as(PU) if fp is not None else None,
                                     fi.ctypes.data_as(PU))
                    fptr.append(fp)
                    fids.append(fi)
                vv = np.zeros(int(nf[n - 1]))
                L.orc_tcsf_vals(h, u64(t), u64(k), vv.ctypes.data_as(PD))
                tiles.append(dict(nfibs=nf.astype(np.int64), dim_perm=dp.astype(np.int64),
                                  fptr=fptr, fids=fids, vals=vv))
            out.append(tiles)
        L.orc_tcsf_free(h)
        return out

    def mttkrp_coo(self, inds, vals, dims, mode, mats):
        keep, pp, d, v = self._coo(inds, vals, dims)
        R = mats[0].shape[1]
        mk, mp = self._ptrs(mats, np.float64)
        out = np.zeros((int(dims[mode]), R))
        self.lib.orc_mttkrp_coo(u64(len(inds)), u64(len(v)), d.ctypes.data_as(PU), pp,
                                v.ctypes.data_as(PD), u64(mode), u64(R), mp,
                                out.ctypes.data_as(PD))
        return out

    def cpd(self, inds, vals, dims, rank, niters, tol, seed):
        keep, pp, d, v = self._coo(inds, vals, dims)
        facs = [np.zeros((int(x), rank)) for x in dims]
        fk, fp = self._ptrs(facs, np.float64)
        lam = np.zeros(rank)
        fit = C.c_double()
        fits = np.zeros(max(niters, 1))
        its = self.lib.orc_cpd(u64(len(inds)), u64(len(v)), d.ctypes.data_as(PU), pp,
                               v.ctypes.data_as(PD), u64(rank), u64(niters),
                               C.c_double(tol), C.c_int(seed), fp,
                               lam.ctypes.data_as(PD), C.byref(fit),
                               fits.ctypes.data_as(PD))
        return dict(factors=fk, lam=lam, fit=fit.value, fits=fits[:int(its)])

    def stream(self, inds, vals, dims, stream_mode, rank, forget=0.95, reg=1e-2,
               max_its=200, seed=1, max_slices=0, nonneg=False, lasso=None, rowsimp=False,
               ntf_lasso=None, ntf_frob=None, colsimp=False):
        """nonneg: `--con=nonneg` (non-negative max-column-norm on the
        non-streamed modes); lasso=L: `--reg=l1,L` (chunked lasso ADMM);
        rowsimp: `--con=rowsimp`; ntf_lasso=L: `--reg=ntf-l1,L`; ntf_frob=L:
        `--reg=ntf-frob,L` (both chunked)."""
        keep, pp, d, v = self._coo(inds, vals, dims)
        nmodes = len(inds)
        nsl = int(dims[stream_mode])
        tout = np.zeros((nsl, rank))
        facs = [np.zeros((int(x), rank)) for x in dims]
        fk, fp = self._ptrs(facs, np.float64)
        rows = np.zeros(nmodes, np.uint64)
        outer = np.zeros(nsl, np.uint64)
        errs = np.zeros(nsl)
        t = self.lib.orc_stream(u64(nmodes), u64(len(v)), d.ctypes.data_as(PU), pp,
                                v.ctypes.data_as(PD), u64(stream_mode), u64(rank),
                                C.c_double(forget), C.c_double(reg), u64(max_its),
                                C.c_int(seed), u64(max_slices), tout.ctypes.data_as(PD),
                                fp, rows.ctypes.data_as(PU), outer.ctypes.data_as(PU),
                                errs.ctypes.data_as(PD),
                                *_con_args(nonneg, lasso, rowsimp, ntf_lasso, ntf_frob, colsimp))
        t = int(t)
        return dict(time=tout[:t], factors=[fk[m][:int(rows[m])] for m in range(nmodes)],
                    rows=rows, outer=outer[:t], local_errsq=errs[:t])

    def stream_prepare(self, inds, vals, dims, stream_mode):
        """orc_stream_prepare: (sorted relabelled inds, vals)."""
        keep, pp, d, v = self._coo(inds, vals, dims)
        outs = [np.zeros(len(v), np.uint64) for _ in inds]
        ok, op = self._ptrs(outs, np.uint64)
        ov = np.zeros(len(v))
        self.lib.orc_stream_prepare(u64(len(inds)), u64(len(v)), d.ctypes.data_as(PU), pp,
                                    v.ctypes.data_as(PD), u64(stream_mode), op,
                                    ov.ctypes.data_as(PD))
        return ok, ov

    def prox(self, kind, mat, lam=0.0, rho=1.0):
        """orc_prox on a copy of the row-major matrix `mat` (kinds as
        PROX_KINDS); returns the result."""
        out = np.ascontiguousarray(mat, np.float64).copy()
        self.lib.orc_prox(C.c_int(kind), out.ctypes.data_as(PD), u64(out.shape[0]),
                          u64(out.shape[1]), C.c_double(lam), C.c_double(rho))
        return out

    def window_errsq(self, inds, vals, dims, stream_mode, time, factors, k):
        """error^2 of the last k slices of a stream that has run len(time)
        slices, against its time rows and (relabeled) factors."""
        keep, pp, d, v = self._coo(inds, vals, dims)
        nmodes = len(inds)
        R = time.shape[1]
        fl = [np.ascontiguousarray(factors[m] if m != stream_mode else time, np.float64)
              for m in range(nmodes)]
        fk, fp = self._ptrs(fl, np.float64)
        rows = np.array([f.shape[0] for f in fl], np.uint64)
        tr = np.ascontiguousarray(time, np.float64)
        return float(self.lib.orc_stream_window_errsq(
            u64(nmodes), u64(len(v)), d.ctypes.data_as(PU), pp, v.ctypes.data_as(PD),
            u64(stream_mode), u64(R), u64(time.shape[0]), tr.ctypes.data_as(PD), fp,
            rows.ctypes.data_as(PU), u64(k)))


class _CsfView:
    """Uniform accessor for a CSF set built by either oracle."""

    def __init__(self, lib, pfx, h, nmodes, nnz, idt, vdt):
        self.lib, self.pfx, self.h = lib, pfx, h
        self.nmodes, self.nnz, self.idt, self.vdt = nmodes, nnz, idt, vdt
        self.count = int(getattr(lib, pfx + "_csf_count")(C.c_void_p(h)))

    def tensor(self, t):
        n = self.nmodes
        ipt = PU if self.idt == np.uint64 else PU32
        nf = np.zeros(n, self.idt)
        dp = np.zeros(n, self.idt)
        root_null = getattr(self.lib, self.pfx + "_csf_info")(
            C.c_void_p(self.h), C.c_uint64(t) if self.idt == np.uint64 else C.c_uint32(t),
            nf.ctypes.data_as(ipt), dp.ctypes.data_as(ipt))
        fptr, fids = [], []
        lvl = getattr(self.lib, self.pfx + "_csf_level")
        ix = (lambda x: C.c_uint64(x)) if self.idt == np.uint64 else (lambda x: C.c_uint32(x))
        for l in range(n):
            fp = np.zeros(int(nf[l]) + 1, self.idt) if l < n - 1 else None
            fi = np.zeros(int(nf[l]), self.idt)
            lvl(C.c_void_p(self.h), ix(t), ix(l),
                fp.ctypes.data_as(C.c_void_p) if fp is not None else None,
                fi.ctypes.data_as(C.c_void_p))
            fptr.append(fp)
            fids.append(fi)
        vals = np.zeros(self.nnz, self.vdt)
        getattr(self.lib, self.pfx + "_csf_vals")(C.c_void_p(self.h), ix(t),
                                                  vals.ctypes.data_as(C.c_void_p))
        return dict(nfibs=nf.astype(np.int64), dim_perm=dp.astype(np.int64), fptr=fptr,
                    fids=fids, vals=vals, root_null=bool(root_null))

    def free(self):
        getattr(self.lib, self.pfx + "_csf_free")(C.c_void_p(self.h))
        self.h = None


class Ref(_Base):
    """The compiled reference (width 64: uint64/double; 32: uint32/float)."""

    def __init__(self, width=64, nthreads=1):
        self.width = width
        self.nthreads = nthreads
        self.lib = C.CDLL(REF_SO[width])
        self.idx_dtype = np.uint64 if width == 64 else np.uint32
        self.val_dtype = np.float64 if width == 64 else np.float32
        L = self.lib
        L.ref_csf_alloc.restype = C.c_void_p
        L.ref_mttkrp.restype = C.c_double
        L.ref_cpd.restype = C.c_double
        if width == 64:
            L.ref_stream.restype = u64
        L.ref_csf_count.restype = u64 if width == 64 else C.c_uint32

    def _ix(self, x):
        return C.c_uint64(x) if self.width == 64 else C.c_uint32(x)

    def prox(self, kind, mat, lam=0.0, rho=1.0):
        """The reference's own proximal operator `kind` (as PROX_KINDS) on a
        copy of the row-major matrix `mat`; returns the result."""
        vt = C.c_double if self.width == 64 else C.c_float
        out = np.ascontiguousarray(mat, self.val_dtype).copy()
        rc = self.lib.ref_prox(C.c_int(kind), self._vp(out), self._ix(out.shape[0]),
                               self._ix(out.shape[1]), vt(lam), vt(rho))
        assert rc == 0, kind
        return out

    def _vp(self, a):
        return a.ctypes.data_as(PD if self.width == 64 else PF)

    def _ip(self, a):
        return a.ctypes.data_as(PU if self.width == 64 else PU32)

    def tt_read(self, path, write_bin=None, remove_empty=False):
        """The reference's own reader (tt_read): (inds, vals, dims).  With
        write_bin, also writes what it read with the reference's own binary
        writer (tt_write_binary) to that path.  With remove_empty, runs its
        tt_remove_empty first and returns (inds, vals, dims, indmaps,
        nremoved), indmaps[m] None where the mode needed no map."""
        L = self.lib
        L.ref_tt_read.restype = C.c_void_p
        it = self.idx_dtype
        n = np.zeros(1, it)
        z = np.zeros(1, it)
        dims = np.zeros(8, it)
        h = L.ref_tt_read(path.encode(), self._ip(n), self._ip(z), self._ip(dims))
        assert h, path
        h = C.c_void_p(h)
        nmodes, nnz = int(n[0]), int(z[0])
        maps, removed = None, 0
        if remove_empty:
            L.ref_tt_remove_empty.restype = u64 if self.width == 64 else C.c_uint32
            removed = int(L.ref_tt_remove_empty(h))
            L.ref_tt_dims(h, self._ip(dims))
            maps = []
            for m in range(nmodes):
                x = np.zeros(int(dims[m]), it)
                maps.append(x if L.ref_tt_indmap(h, self._ix(m), self._ip(x)) else None)
        inds = []
        for m in range(nmodes):
            x = np.zeros(nnz, it)
            L.ref_tt_get(h, self._ix(m), self._ip(x), None)
            inds.append(x)
        vals = np.zeros(nnz, self.val_dtype)
        L.ref_tt_get(h, self._ix(0), None, self._vp(vals))
        if write_bin is not None:
            L.ref_tt_write_bin(h, str(write_bin).encode())
        L.ref_tt_free(h)
        if remove_empty:
            return inds, vals, dims[:nmodes].copy(), maps, removed
        return inds, vals, dims[:nmodes].copy()

    def csf(self, inds, vals, dims, alloc_type):
        keep, pp, d, v = self._coo(inds, vals, dims)
        h = self.lib.ref_csf_alloc(self._ix(len(inds)), self._ix(len(v)), self._ip(d), pp,
                                   self._vp(v), C.c_int(alloc_type), C.c_int(self.nthreads))
        return _CsfView(self.lib, "ref", h, len(inds), len(v), self.idx_dtype,
                        self.val_dtype)

    def csf_tiled(self, inds, vals, dims, alloc_type, nthreads, tilelevel):
        """csf_alloc with SPLATT_DENSETILE; same layout as Port.csf_tiled, plus
        root_null and tile_dims per tile."""
        keep, pp, d, v = self._coo(inds, vals, dims)
        L = self.lib
        ix, ipt, it = self._ix, (PU if self.width == 64 else PU32), self.idx_dtype
        L.ref_csf_alloc_tiled.restype = C.c_void_p
        L.ref_csf_ntiles.restype = u64 if self.width == 64 else C.c_uint32
        h = C.c_void_p(L.ref_csf_alloc_tiled(ix(len(inds)), ix(len(v)), self._ip(d), pp,
                                             self._vp(v), C.c_int(alloc_type),
                                             C.c_int(nthreads), C.c_int(tilelevel)))
        n = len(inds)
        out = []
        for t in range(int(L.ref_csf_count(h))):
            tiles = []
            for k in range(int(L.ref_csf_ntiles(h, ix(t)))):
                nf = np.zeros(n, it)
                td = np.zeros(n, it)
                root_null = L.ref_csf_tile_info(h, ix(t), ix(k), nf.ctypes.data_as(ipt),
                                                td.ctypes.data_as(ipt))
                fptr, fids = [], []
                for l in range(n):
                    fp = np.zeros(int(nf[l]) + 1, it) if l < n - 1 else None
                    fi = np.zeros(int(nf[l]), it)
                    L.ref_csf_tile_level(h, ix(t), ix(k), ix(l),
                                         fp.ctypes.data_as(ipt) if fp is not None else None,
                                         fi.ctypes.data_as(ipt))
                    fptr.append(fp)
                    fids.append(fi)
                vv = np.zeros(int(nf[n - 1]), self.val_dtype)
                L.ref_csf_tile_vals(h, ix(t), ix(k), self._vp(vv))
                tiles.append(dict(nfibs=nf.astype(np.int64), fptr=fptr, fids=fids, vals=vv,
                                  root_null=bool(root_null), tile_dims=td.astype(np.int64)))
            out.append(tiles)
        L.ref_csf_free(h)
        return out

    def mttkrp_tiled(self, inds, vals, dims, alloc_type, nthreads, tilelevel, mats):
        """splatt_mttkrp into every mode on a SPLATT_DENSETILE CSF of
        `nthreads` ranges on the bottom `tilelevel` levels, run with
        `nthreads` threads (as the reference's tests/mttkrp_test.c runs it);
        returns one output per mode."""
        keep, pp, d, v = self._coo(inds, vals, dims)
        L = self.lib
        ix = self._ix
        L.ref_csf_alloc_tiled.restype = C.c_void_p
        h = C.c_void_p(L.ref_csf_alloc_tiled(ix(len(inds)), ix(len(v)), self._ip(d), pp,
                                             self._vp(v), C.c_int(alloc_type),
                                             C.c_int(nthreads), C.c_int(tilelevel)))
        R = mats[0].shape[1]
        mk, mp = self._ptrs(mats, self.val_dtype)
        nrows = max(m.shape[0] for m in mats)
        outs = []
        for mode in range(len(inds)):
            out = np.zeros((nrows, R), self.val_dtype)
            L.ref_mttkrp(h, ix(mode), ix(R), mp, self._vp(out), C.c_int(nthreads))
            outs.append(out[:mats[mode].shape[0]].copy())
        L.ref_csf_free(h)
        return outs

    def mttkrp(self, view, mode, mats):
        R = mats[0].shape[1]
        mk, mp = self._ptrs(mats, self.val_dtype)
        nrows = max(m.shape[0] for m in mats)
        out = np.zeros((nrows, R), self.val_dtype)
        secs = self.lib.ref_mttkrp(C.c_void_p(view.h), self._ix(mode), self._ix(R), mp,
                                   self._vp(out), C.c_int(self.nthreads))
        return out[:mats[mode].shape[0]], secs

    def mttkrp_coo(self, inds, vals, dims, mode, mats):
        keep, pp, d, v = self._coo(inds, vals, dims)
        R = mats[0].shape[1]
        mk, mp = self._ptrs(mats, self.val_dtype)
        out = np.zeros((int(dims[mode]), R), self.val_dtype)
        self.lib.ref_mttkrp_coo(self._ix(len(inds)), self._ix(len(v)), self._ip(d), pp,
                                self._vp(v), self._ix(mode), self._ix(R), mp, self._vp(out),
                                C.c_int(self.nthreads))
        return out

    def cpd(self, inds, vals, dims, rank, niters, tol, seed):
        keep, pp, d, v = self._coo(inds, vals, dims)
        facs = [np.zeros((int(x), rank), self.val_dtype) for x in dims]
        fk, fp = self._ptrs(facs, self.val_dtype)
        lam = np.zeros(rank, self.val_dtype)
        fit = C.c_double()
        secs = self.lib.ref_cpd(self._ix(len(inds)), self._ix(len(v)), self._ip(d), pp,
                                self._vp(v), self._ix(rank), self._ix(niters), C.c_double(tol),
                                C.c_int(seed), C.c_int(self.nthreads), fp, self._vp(lam),
                                C.byref(fit))
        return dict(factors=fk, lam=lam, fit=fit.value, secs=secs)

    def stream(self, inds, vals, dims, stream_mode, rank, forget=0.95, reg=1e-2,
               max_its=200, seed=1, nonneg=False, lasso=None, rowsimp=False,
               ntf_lasso=None, ntf_frob=None, colsimp=False):
        assert self.width == 64
        keep, pp, d, v = self._coo(inds, vals, dims)
        nmodes = len(inds)
        nsl = int(dims[stream_mode])
        tout = np.zeros((nsl, rank))
        facs = [np.zeros((int(x), rank)) for x in dims]
        fk, fp = self._ptrs(facs, np.float64)
        rows = np.zeros(nmodes, np.uint64)
        secs = np.zeros(nsl)
        errs = np.zeros(nsl)
        with tempfile.TemporaryDirectory() as td:
            binp = os.path.join(td, "stream.bin").encode()
            logp = os.path.join(td, "stream.log").encode()
            t = self.lib.ref_stream(u64(nmodes), u64(len(v)), d.ctypes.data_as(PU), pp,
                                    v.ctypes.data_as(PD), u64(stream_mode), u64(rank),
                                    C.c_double(forget), C.c_double(reg), u64(max_its),
                                    C.c_int(seed), C.c_int(self.nthreads), binp, logp,
                                    tout.ctypes.data_as(PD), fp, rows.ctypes.data_as(PU),
                                    secs.ctypes.data_as(PD), errs.ctypes.data_as(PD),
                                    *_con_args(nonneg, lasso, rowsimp, ntf_lasso, ntf_frob, colsimp))
            with open(logp.decode()) as f:
                log = f.read()
            reports = _stream_reports(log)
        t = int(t)
        return dict(time=tout[:t], factors=[fk[m][:int(rows[m])] for m in range(nmodes)],
                    rows=rows, batch_secs=secs[:t], local_errsq=errs[:t], reports=reports,
                    outer=_stream_outer(log)[:t])


def _stream_outer(log):
    """Outer iterations of every batch: the streaming driver prints one
    "delta:" line per outer iteration (StreamCPD.cc:472) before the batch's
    "batch N:" line (StreamCPD.cc:530)."""
    out, n = [], 0
    for line in log.splitlines():
        s = line.strip()
        if s.startswith("delta:"):
            n += 1
        elif s.startswith("batch"):
            out.append(n)
            n = 0
    return np.array(out, np.uint64)


def _stream_reports(log):
    """The streaming driver's printed error reports (StreamCPD.cc:509-528,
    553-556): per reporting batch (every 100th and the last) its "global" and
    "local-10" error^2, and the final "final-err" error^2, 5 decimals each."""
    import re
    rep = {}
    for line in log.splitlines():
        m = re.match(r"batch\s+(\d+):.*global: ([-+0-9.eE]+) local-1: [-+0-9.eE]+ "
                     r"local-10: ([-+0-9.eE]+)", line)
        if m and float(m.group(2)) >= 0.0:
            rep[int(m.group(1))] = dict(global_=float(m.group(2)), local10=float(m.group(3)))
        m = re.match(r"final-err: ([-+0-9.eE]+)", line)
        if m:
            rep["final"] = float(m.group(1))
    return rep
