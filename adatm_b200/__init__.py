"""B200-native AdaTM: memoized sparse MTTKRP sequence and CP-ALS on sm_100a.

The product is ``libadatm_b200.so`` (C ABI: ``include/splatt.h`` and
``include/adatm_b200.h``). This module binds it with ctypes so Python callers
and tests use the same entry points a C caller of the reference would:

* SPLATT's public API -- :func:`splatt_default_opts`, :func:`splatt_csf_convert`,
  :func:`splatt_mttkrp`, :func:`splatt_cpd_als`;
* AdaTM's entry points -- :func:`decide_parameters_auto`,
  :func:`csf_alloc_adaptive`, :func:`rcsf_alloc_adaptive`,
  :func:`decide_use_csfs`, :func:`mttkrp_csf_adaptive`,
  :func:`cpd_als_iterate_adaptive`;
* the device-resident interface -- :class:`Tensor`, :func:`plan_analytic`,
  :func:`plan_splatt`, :class:`Engine`.

There is no CPU fallback: importing works anywhere, but every call needs the
compiled library and a CUDA device, and raises otherwise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native as N
from ._native import (SPLATT_SUCCESS, SPLATT_ERROR_BADINPUT, SPLATT_ERROR_NOMEMORY,
                      ADATM_ERROR_CUDA, SplattCsf, SplattKruskal, GroupProperties,
                      RcsfSeq, MatrixT, SpTensorT, AdatmPlan, AdatmCandidate)
from ._native import lib, library_path, build

MAX_NMODES = N.MAX_NMODES

# options (include/splatt.h)
OPT_NTHREADS, OPT_TOLERANCE, OPT_NITER, OPT_VERBOSITY, OPT_RANDSEED, OPT_CSF_ALLOC, \
    OPT_TILE, OPT_TILEDEPTH, OPT_DECOMP, OPT_COMM, OPT_NOPTIONS = range(11)
CSF_ONEMODE, CSF_TWOMODE, CSF_ALLMODE, ADAPTIVE, ADAPTIVE_TIME_EFFICIENT, \
    ADAPTIVE_SPACE_EFFICIENT = range(6)


class AdatmError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed with code {code}: {N.last_error()}")
        self.code = code


def _check(rc, what):
    if rc != SPLATT_SUCCESS:
        raise AdatmError(rc, what)


def _u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(C.POINTER(C.c_uint64))


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _row_ptrs(arrays, ctype=C.c_uint64):
    P = C.POINTER(ctype)
    return (P * len(arrays))(*[a.ctypes.data_as(P) for a in arrays])


# ---------------------------------------------------------------------------
# SPLATT public API
# ---------------------------------------------------------------------------

def splatt_default_opts():
    p = lib().splatt_default_opts()
    arr = np.ctypeslib.as_array(p, shape=(OPT_NOPTIONS,)).copy()
    lib().splatt_free_opts(p)
    return arr


class CsfSet:
    """Trees returned by splatt_csf_convert / csf_alloc_adaptive (host view in
    the reference layout; device copies stay resident until free())."""

    def __init__(self, ptr, n, opts):
        self.ptr = ptr
        self.n = n
        self.opts = np.ascontiguousarray(opts, dtype=np.float64)

    def __len__(self):
        return self.n

    def tree(self, g):
        c = self.ptr[g]
        Nm = int(c.nmodes)
        pt = c.pt.contents
        out = {"nnz": int(c.nnz), "nmodes": Nm,
               "dims": np.array(c.dims[:Nm], dtype=np.uint64),
               "dim_perm": np.array(c.dim_perm[:Nm], dtype=np.uint64),
               "nfibs": np.array(pt.nfibs[:Nm], dtype=np.uint64), "fptr": [], "fids": []}
        for l in range(Nm):
            F = int(pt.nfibs[l])
            out["fptr"].append(np.ctypeslib.as_array(pt.fptr[l], shape=(F + 1,)).copy()
                               if (l < Nm - 1 and pt.fptr[l]) else None)
            out["fids"].append(np.ctypeslib.as_array(pt.fids[l], shape=(F,)).copy()
                               if (pt.fids[l] and F > 0) else (None if l == 0 else np.zeros(0, np.uint64)))
        out["vals"] = (np.ctypeslib.as_array(pt.vals, shape=(int(c.nnz),)).copy()
                       if c.nnz else np.zeros(0))
        return out

    def free(self):
        if self.ptr:
            lib().splatt_free_csf(self.ptr, self.opts.ctypes.data_as(C.POINTER(C.c_double)))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def splatt_csf_convert(inds, vals, opts=None):
    """COO (inds[N, nnz], vals[nnz]) -> CsfSet per opts[CSF_ALLOC]."""
    opts = splatt_default_opts() if opts is None else np.ascontiguousarray(opts, np.float64)
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    Nm, nnz = inds.shape
    rows = [inds[m] for m in range(Nm)]
    out = C.POINTER(SplattCsf)()
    rc = lib().splatt_csf_convert(Nm, nnz, _row_ptrs(rows), vals.ctypes.data_as(C.POINTER(C.c_double)),
                                  C.byref(out), opts.ctypes.data_as(C.POINTER(C.c_double)))
    _check(rc, "splatt_csf_convert")
    alloc = int(opts[OPT_CSF_ALLOC])
    if alloc == CSF_ONEMODE:
        n = 1
    elif alloc == CSF_TWOMODE:
        n = 2
    elif alloc == CSF_ALLMODE:
        n = Nm
    else:
        n = _count_trees(out)
    return CsfSet(out, n, opts)


def _count_trees(ptr):
    n = C.c_int(0)
    _check(lib().adatm_csf_tree_count(ptr, C.byref(n)), "adatm_csf_tree_count")
    return n.value


def splatt_mttkrp(mode, ncolumns, csf: CsfSet, mats, opts=None):
    opts = csf.opts if opts is None else np.ascontiguousarray(opts, np.float64)
    mats = [np.ascontiguousarray(m, dtype=np.float64) for m in mats]
    dims = csf.tree(0)["dims"]
    out = np.zeros((int(dims[mode]), ncolumns))
    rc = lib().splatt_mttkrp(mode, ncolumns, csf.ptr, _row_ptrs(mats, C.c_double),
                             out.ctypes.data_as(C.POINTER(C.c_double)),
                             opts.ctypes.data_as(C.POINTER(C.c_double)))
    _check(rc, "splatt_mttkrp")
    return out


def _kruskal_to_py(k):
    Nm = int(k.nmodes)
    R = int(k.rank)
    out = {"rank": R, "nmodes": Nm, "fit": float(k.fit),
           "lambda": np.ctypeslib.as_array(k.lambda_, shape=(R,)).copy(),
           "factors": [np.ctypeslib.as_array(k.factors[m], shape=(int(k.dims[m]), R)).copy()
                       for m in range(Nm)]}
    lib().splatt_free_kruskal(C.byref(k))
    return out


def splatt_cpd_als(csf: CsfSet, nfactors, opts=None):
    opts = csf.opts if opts is None else np.ascontiguousarray(opts, np.float64)
    k = SplattKruskal()
    rc = lib().splatt_cpd_als(csf.ptr, nfactors, opts.ctypes.data_as(C.POINTER(C.c_double)),
                              C.byref(k))
    _check(rc, "splatt_cpd_als")
    return _kruskal_to_py(k)


# ---------------------------------------------------------------------------
# AdaTM entry points (reference src/adatm_*.h)
# ---------------------------------------------------------------------------

class _SpTensor:
    def __init__(self, inds, vals, dims):
        self.inds = np.ascontiguousarray(inds, dtype=np.uint64)
        self.vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.dims = np.ascontiguousarray(dims, dtype=np.uint64)
        Nm, nnz = self.inds.shape
        self.rows = [self.inds[m] for m in range(Nm)]
        self._ind = _row_ptrs(self.rows)
        self.tt = SpTensorT(nnz=nnz, nmodes=Nm,
                            dims=self.dims.ctypes.data_as(C.POINTER(C.c_uint64)),
                            ind=self._ind, vals=self.vals.ctypes.data_as(C.POINTER(C.c_double)),
                            tiled=0, type=0 if Nm == 3 else 1)


def _groups_from_c(gp, n, Nm):
    return [{"memo_mode": int(gp[g].memo_mode), "begin_imten": int(gp[g].begin_imten),
             "n_imten": int(gp[g].n_imten), "o_opt": [int(gp[g].o_opt[m]) for m in range(Nm)]}
            for g in range(n)]


class _GroupArray:
    def __init__(self, groups, Nm):
        self.arr = (GroupProperties * max(1, len(groups)))()
        self.o = [np.array(g["o_opt"][:Nm], dtype=np.uint64) for g in groups]
        for i, g in enumerate(groups):
            self.arr[i].memo_mode = g["memo_mode"]
            self.arr[i].begin_imten = g["begin_imten"]
            self.arr[i].n_imten = g["n_imten"]
            self.arr[i].o_opt = self.o[i].ctypes.data_as(C.POINTER(C.c_uint64))
        self.n = len(groups)


def decide_parameters_auto(inds, vals, dims, nfactors, strategy=1):
    t = _SpTensor(inds, vals, dims)
    Nm = len(dims)
    po_rows = [np.zeros(2 * Nm, dtype=np.uint64) for _ in range(Nm)]
    po = _row_ptrs(po_rows)
    lib().decide_product_order(C.byref(t.tt), po)
    gp = C.POINTER(GroupProperties)()
    n = lib().decide_parameters_auto(C.byref(t.tt), nfactors, strategy, po, C.byref(gp))
    if n == 0:
        raise AdatmError(SPLATT_ERROR_BADINPUT, "decide_parameters_auto")
    groups = _groups_from_c(gp, n, Nm)
    lib().adatm_free_groups(gp, n)
    return groups


def decide_product_order(nmodes):
    rows = [np.zeros(2 * nmodes, dtype=np.uint64) for _ in range(nmodes)]
    dims = np.ones(nmodes, dtype=np.uint64)
    tt = SpTensorT(nnz=0, nmodes=nmodes, dims=dims.ctypes.data_as(C.POINTER(C.c_uint64)))
    lib().decide_product_order(C.byref(tt), _row_ptrs(rows))
    return np.stack(rows)


def csf_alloc_adaptive(inds, vals, dims, groups, opts=None):
    opts = splatt_default_opts() if opts is None else np.ascontiguousarray(opts, np.float64)
    t = _SpTensor(inds, vals, dims)
    ga = _GroupArray(groups, len(dims))
    n_csf = C.c_uint64(0)
    ptr = lib().csf_alloc_adaptive(C.byref(t.tt), ga.arr, ga.n,
                                   opts.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n_csf))
    if not ptr:
        raise AdatmError(SPLATT_ERROR_BADINPUT, "csf_alloc_adaptive")
    return CsfSet(ptr, n_csf.value, opts)


class RcsfSet:
    def __init__(self, ptr, n):
        self.ptr = ptr
        self.n = n

    def pull(self):
        _check(lib().adatm_rcsf_pull(self.ptr, self.n), "adatm_rcsf_pull")

    def memo(self, j, deg):
        r = self.ptr[j].rcsfs[deg]
        return {"nmodes": int(r.nmodes), "nnz": int(r.nnz),
                "vals": np.ctypeslib.as_array(r.pt.contents.vals, shape=(int(r.nnz),)).copy()}


def rcsf_alloc_adaptive(csf: CsfSet, nfactors, groups, opts=None):
    opts = csf.opts if opts is None else np.ascontiguousarray(opts, np.float64)
    ga = _GroupArray(groups, csf.tree(0)["nmodes"])
    n = C.c_uint64(0)
    ptr = lib().rcsf_alloc_adaptive(csf.ptr, nfactors, ga.arr, ga.n, len(csf),
                                    opts.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n))
    if not ptr:
        raise AdatmError(SPLATT_ERROR_BADINPUT, "rcsf_alloc_adaptive")
    return RcsfSet(ptr, n.value)


def decide_use_csfs(nmodes, groups, n_csf=None):
    ga = _GroupArray(groups, nmodes)
    uc = np.zeros(nmodes, dtype=np.uint64)
    ut = np.zeros(nmodes, dtype=np.uint64)
    lib().decide_use_csfs(nmodes, ga.arr, ga.n, len(groups) if n_csf is None else n_csf,
                          uc.ctypes.data_as(C.POINTER(C.c_uint64)),
                          ut.ctypes.data_as(C.POINTER(C.c_uint64)))
    return uc, ut


def _matrix_array(mats, out_rows, R):
    Nm = len(mats)
    keep = [np.ascontiguousarray(m, dtype=np.float64) for m in mats]
    out = np.zeros((out_rows, R))
    structs = [MatrixT(I=k.shape[0], J=R, vals=k.ctypes.data_as(C.POINTER(C.c_double)), rowmajor=1)
               for k in keep]
    ostruct = MatrixT(I=out_rows, J=R, vals=out.ctypes.data_as(C.POINTER(C.c_double)), rowmajor=1)
    arr = (C.POINTER(MatrixT) * (MAX_NMODES + 1))()
    for m in range(Nm):
        arr[m] = C.pointer(structs[m])
    arr[MAX_NMODES] = C.pointer(ostruct)
    return arr, keep, out, structs, ostruct


def mttkrp_csf_adaptive(csf: CsfSet, rcsf: RcsfSet, mats, mode, groups, use_csfs, use_tags,
                        opts=None):
    opts = csf.opts if opts is None else np.ascontiguousarray(opts, np.float64)
    R = mats[0].shape[1]
    rows = max(m.shape[0] for m in mats)
    arr, keep, out, s1, s2 = _matrix_array(mats, rows, R)
    ga = _GroupArray(groups, len(mats))
    lib().mttkrp_csf_adaptive(csf.ptr, rcsf.ptr if rcsf else None, len(csf), arr, mode, None,
                              ga.arr, ga.n, int(use_csfs[mode]), int(use_tags[mode]),
                              opts.ctypes.data_as(C.POINTER(C.c_double)))
    if N.last_error():
        raise AdatmError(SPLATT_ERROR_BADINPUT, "mttkrp_csf_adaptive")
    return out[: mats[mode].shape[0]].copy()


def cpd_als_iterate_adaptive(csf: CsfSet, rcsf: RcsfSet, groups, use_csfs, use_tags, mats,
                             niters, tol, opts=None):
    opts = (csf.opts if opts is None else np.ascontiguousarray(opts, np.float64)).copy()
    opts[OPT_NITER] = niters
    opts[OPT_TOLERANCE] = tol
    R = mats[0].shape[1]
    arr, keep, out, s1, s2 = _matrix_array([m.copy() for m in mats], max(m.shape[0] for m in mats), R)
    lam = np.zeros(R)
    ga = _GroupArray(groups, len(mats))
    uc, ucp = _u64(use_csfs)
    ut, utp = _u64(use_tags)
    fit = lib().cpd_als_iterate_adaptive(csf.ptr, rcsf.ptr if rcsf else None, len(csf), ga.arr, ga.n,
                                         ucp, utp, arr, lam.ctypes.data_as(C.POINTER(C.c_double)),
                                         R, None, opts.ctypes.data_as(C.POINTER(C.c_double)))
    if N.last_error():
        raise AdatmError(SPLATT_ERROR_BADINPUT, "cpd_als_iterate_adaptive")
    return {"fit": fit, "lambda": lam, "factors": keep}


class CpdIterator:
    """Repeated cpd_als_iterate_adaptive calls on the same host factor
    buffers, as a C caller makes them: the matrix_t array is built once and
    the library updates the factors in place (host FP64 in, host FP64 out)."""

    def __init__(self, csf: CsfSet, rcsf: RcsfSet, groups, use_csfs, use_tags, mats, opts=None):
        self.csf, self.rcsf = csf, rcsf
        self.opts = (csf.opts if opts is None else np.ascontiguousarray(opts, np.float64)).copy()
        self.R = mats[0].shape[1]
        self.arr, self.factors, self._out, self._s1, self._s2 = _matrix_array(
            [np.array(m, dtype=np.float64, order="C", copy=True) for m in mats],
            max(m.shape[0] for m in mats), self.R)
        self.lam = np.zeros(self.R)
        self._ga = _GroupArray(groups, len(mats))
        self._uc, self._ucp = _u64(use_csfs)
        self._ut, self._utp = _u64(use_tags)
        self._lamp = self.lam.ctypes.data_as(C.POINTER(C.c_double))
        self._optp = self.opts.ctypes.data_as(C.POINTER(C.c_double))

    def step(self, niters=1, tol=0.0):
        self.opts[OPT_NITER] = niters
        self.opts[OPT_TOLERANCE] = tol
        return lib().cpd_als_iterate_adaptive(self.csf.ptr, self.rcsf.ptr if self.rcsf else None,
                                              len(self.csf), self._ga.arr, self._ga.n, self._ucp,
                                              self._utp, self.arr, self._lamp, self.R, None,
                                              self._optp)


# ---------------------------------------------------------------------------
# device-resident interface
# ---------------------------------------------------------------------------

def _plan_to_py(p: AdatmPlan):
    Nm = p.nmodes
    return {"nmodes": Nm, "n_grp": p.n_grp,
            "groups": [{"memo_mode": int(p.memo_mode[g]), "begin_imten": int(p.begin_imten[g]),
                        "n_imten": int(p.n_imten[g]), "o_opt": [int(p.o_opt[g][l]) for l in range(Nm)]}
                       for g in range(p.n_grp)],
            "use_csfs": [int(p.use_csfs[m]) for m in range(Nm)],
            "use_tags": [int(p.use_tags[m]) for m in range(Nm)],
            "space_efficient": bool(p.space_efficient)}


def plan_to_c(plan) -> AdatmPlan:
    p = AdatmPlan()
    p.nmodes = plan["nmodes"]
    p.n_grp = len(plan["groups"])
    for g, gr in enumerate(plan["groups"]):
        p.memo_mode[g] = gr["memo_mode"]
        p.begin_imten[g] = gr["begin_imten"]
        p.n_imten[g] = gr["n_imten"]
        for l, v in enumerate(gr["o_opt"]):
            p.o_opt[g][l] = v
    p.space_efficient = 1 if plan.get("space_efficient") else 0
    uc = plan.get("use_csfs")
    ut = plan.get("use_tags")
    if uc is None or ut is None:
        uc, ut = decide_use_csfs(plan["nmodes"], plan["groups"])
    for m in range(plan["nmodes"]):
        p.use_csfs[m] = int(uc[m])
        p.use_tags[m] = int(ut[m])
    return p


class Tensor:
    """A COO tensor resident in HBM."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_coo(cls, inds, vals, dims, clean=False):
        inds = np.ascontiguousarray(inds, dtype=np.uint64)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        d, dp = _u64(dims)
        Nm, nnz = inds.shape
        h = C.c_void_p()
        rc = lib().adatm_tensor_from_coo(Nm, nnz, dp, _row_ptrs([inds[m] for m in range(Nm)]),
                                         vals.ctypes.data_as(C.POINTER(C.c_double)), int(clean),
                                         C.byref(h))
        _check(rc, "adatm_tensor_from_coo")
        return cls(h)

    @classmethod
    def generate(cls, dims, nnz, alpha=None, value_kind=0, mu=0.0, sigma=1.0, seed=0):
        d, dp = _u64(dims)
        a = np.zeros(len(dims)) if alpha is None else np.array(
            [alpha] * len(dims) if np.isscalar(alpha) else alpha, dtype=np.float64)
        h = C.c_void_p()
        rc = lib().adatm_tensor_generate(len(dims), dp, nnz, a.ctypes.data_as(C.POINTER(C.c_double)),
                                         value_kind, mu, sigma, seed, C.byref(h))
        _check(rc, "adatm_tensor_generate")
        return cls(h)

    def info(self):
        n = C.c_int(0)
        z = C.c_uint64(0)
        dims = np.zeros(8, dtype=np.uint64)
        _check(lib().adatm_tensor_info(self._h, C.byref(n), C.byref(z),
                                       dims.ctypes.data_as(C.POINTER(C.c_uint64))), "info")
        return n.value, z.value, [int(x) for x in dims[: n.value]]

    def download(self):
        Nm, nnz, dims = self.info()
        inds = np.zeros((Nm, nnz), dtype=np.uint64)
        vals = np.zeros(nnz)
        _check(lib().adatm_tensor_download(self._h, inds.ctypes.data_as(C.POINTER(C.c_uint64)),
                                           vals.ctypes.data_as(C.POINTER(C.c_double))), "download")
        return inds, vals, dims

    def count_nfibs(self, perm):
        p, pp = _u64(perm)
        out = np.zeros(len(perm), dtype=np.uint64)
        _check(lib().adatm_tensor_count_nfibs(self._h, pp, out.ctypes.data_as(C.POINTER(C.c_uint64))),
               "count_nfibs")
        return out

    def free(self):
        if self._h:
            lib().adatm_tensor_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def plan_analytic(tensor: Tensor, rank, strategy=1):
    p = AdatmPlan()
    cands = (AdatmCandidate * 64)()
    nc = C.c_int(0)
    ch = C.c_int(0)
    rc = lib().adatm_plan_analytic(tensor._h, rank, strategy, C.byref(p), cands, 64, C.byref(nc),
                                   C.byref(ch))
    _check(rc, "adatm_plan_analytic")
    cl = [dict(_plan_to_py(cands[i].plan), pspace=int(cands[i].pspace), pops=int(cands[i].pops))
          for i in range(min(nc.value, 64))]
    return _plan_to_py(p), cl, ch.value


def plan_splatt(tensor: Tensor, csf_alloc):
    p = AdatmPlan()
    _check(lib().adatm_plan_splatt(tensor._h, csf_alloc, C.byref(p)), "adatm_plan_splatt")
    return _plan_to_py(p)


# ---------------------------------------------------------------------------
# Learned plan model
# ---------------------------------------------------------------------------

PLAN_FEATURES = 16


def plan_features(tensor: Tensor, rank):
    """Candidate plans of decide_candidate_configs with their features
    (ncand x PLAN_FEATURES, float32) and exact device bytes."""
    X = np.zeros((64, PLAN_FEATURES), dtype=np.float32)
    b = np.zeros(64)
    cands = (AdatmCandidate * 64)()
    nc = C.c_int(0)
    rc = lib().adatm_plan_features(tensor._h, rank, X.ctypes.data_as(C.POINTER(C.c_float)),
                                   b.ctypes.data_as(C.POINTER(C.c_double)), cands, 64, C.byref(nc))
    _check(rc, "adatm_plan_features")
    n = min(nc.value, 64)
    cl = [dict(_plan_to_py(cands[i].plan), pspace=int(cands[i].pspace), pops=int(cands[i].pops))
          for i in range(n)]
    return X[:n].copy(), b[:n].copy(), cl


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The plan model's network on the GPU (forward, gradient and Adam
    training by the library's own kernels)."""

    def __init__(self, widths, seed=0):
        w = (C.c_int * len(widths))(*widths)
        h = C.c_void_p()
        _check(lib().adatm_mlp_create(len(widths), w, seed, C.byref(h)), "adatm_mlp_create")
        self._h = h
        self.widths = list(widths)
        n = C.c_uint64(0)
        _check(lib().adatm_mlp_nparams(h, C.byref(n)), "adatm_mlp_nparams")
        self.nparams = n.value

    def get_params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        _check(lib().adatm_mlp_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float))),
               "adatm_mlp_get_params")
        return out

    def set_params(self, params):
        a, p = _f32(params)
        assert a.size == self.nparams
        _check(lib().adatm_mlp_set_params(self._h, p), "adatm_mlp_set_params")

    def forward(self, X):
        a, p = _f32(X)
        y = np.zeros(a.shape[0], dtype=np.float32)
        _check(lib().adatm_mlp_forward(self._h, p, a.shape[0], y.ctypes.data_as(C.POINTER(C.c_float))),
               "adatm_mlp_forward")
        return y

    def gradient(self, X, T):
        a, p = _f32(X)
        t, tp = _f32(T)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double(0)
        _check(lib().adatm_mlp_gradient(self._h, p, tp, a.shape[0], g.ctypes.data_as(C.POINTER(C.c_float)),
                                        C.byref(loss)), "adatm_mlp_gradient")
        return loss.value, g

    def train(self, X, T, epochs, batch, lr, seed=0):
        a, p = _f32(X)
        t, tp = _f32(T)
        loss = C.c_double(0)
        _check(lib().adatm_mlp_train(self._h, p, tp, a.shape[0], epochs, batch, lr, seed,
                                     C.byref(loss)), "adatm_mlp_train")
        return loss.value

    def free(self):
        if self._h:
            lib().adatm_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PlanModel:
    """A trained plan model: network widths and parameters plus the feature
    standardisation, stored as one .npz."""

    def __init__(self, widths, params, mean, std):
        self.widths = [int(w) for w in widths]
        self.mean = np.ascontiguousarray(mean, dtype=np.float32)
        self.std = np.ascontiguousarray(std, dtype=np.float32)
        self.net = Mlp(self.widths)
        self.net.set_params(params)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(z["widths"], z["params"], z["mean"], z["std"])

    def save(self, path, **extra):
        np.savez(path, widths=np.array(self.widths), params=self.net.get_params(), mean=self.mean,
                 std=self.std, **extra)

    def predict(self, X):
        return self.net.forward((np.asarray(X, dtype=np.float32) - self.mean) / self.std)


def plan_learned(tensor: Tensor, rank, model: PlanModel | None):
    """The learned plan (lowest predicted sweep time within the storage
    limit); the analytic plan when model is None. Returns (plan, chosen
    candidate index, whether the model decided)."""
    p = AdatmPlan()
    ch = C.c_int(0)
    used = C.c_int(0)
    if model is None:
        rc = lib().adatm_plan_learned(tensor._h, rank, None, None, None, C.byref(p), C.byref(ch),
                                      C.byref(used))
    else:
        rc = lib().adatm_plan_learned(tensor._h, rank, model.net._h,
                                      model.mean.ctypes.data_as(C.POINTER(C.c_float)),
                                      model.std.ctypes.data_as(C.POINTER(C.c_float)), C.byref(p),
                                      C.byref(ch), C.byref(used))
    _check(rc, "adatm_plan_learned")
    return _plan_to_py(p), ch.value, bool(used.value)


class Engine:
    """Trees, memo rows and factors of one plan and rank, resident in HBM."""

    def __init__(self, tensor: Tensor, rank, plan, bf16=False, chunk_leaf=0, chunk_rows=0):
        self.plan = plan
        self.R = rank
        self.nmodes, self.nnz, self.dims = tensor.info()
        h = C.c_void_p()
        cp = plan_to_c(plan)
        rc = lib().adatm_engine_create(tensor._h, rank, C.byref(cp), int(bf16), chunk_leaf,
                                       chunk_rows, C.byref(h))
        _check(rc, "adatm_engine_create")
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            lib().adatm_engine_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def n_csf(self):
        n = C.c_int(0)
        _check(lib().adatm_engine_csf_count(self._h, C.byref(n)), "csf_count")
        return n.value

    def csf_shape(self, g):
        nf = np.zeros(self.nmodes, dtype=np.uint64)
        dp = np.zeros(self.nmodes, dtype=np.uint64)
        _check(lib().adatm_engine_csf_shape(self._h, g, nf.ctypes.data_as(C.POINTER(C.c_uint64)),
                                            dp.ctypes.data_as(C.POINTER(C.c_uint64))), "csf_shape")
        return nf, dp

    def csf_arrays(self, g):
        nf, dp = self.csf_shape(g)
        Nm = self.nmodes
        fptr = [np.zeros(int(nf[l]) + 1, dtype=np.uint64) for l in range(Nm - 1)] + [np.zeros(1, np.uint64)]
        fids = [np.zeros(max(1, int(nf[l])), dtype=np.uint64) for l in range(Nm)]
        vals = np.zeros(max(1, self.nnz))
        _check(lib().adatm_engine_csf_arrays(self._h, g, _row_ptrs(fptr), _row_ptrs(fids),
                                             vals.ctypes.data_as(C.POINTER(C.c_double))), "csf_arrays")
        return {"nfibs": nf, "dim_perm": dp, "fptr": fptr[: Nm - 1] + [None],
                "fids": [fids[l][: int(nf[l])] for l in range(Nm)], "vals": vals[: self.nnz]}

    def memory(self):
        a = C.c_uint64(0)
        b = C.c_uint64(0)
        _check(lib().adatm_engine_memory(self._h, C.byref(a), C.byref(b)), "memory")
        return a.value, b.value

    def init_factors(self, seed=0):
        _check(lib().adatm_engine_init_factors(self._h, seed), "init_factors")

    def set_factors(self, mats):
        keep = [np.ascontiguousarray(m, dtype=np.float64) for m in mats]
        _check(lib().adatm_engine_set_factors(self._h, _row_ptrs(keep, C.c_double)), "set_factors")

    def get_factors(self):
        mats = [np.zeros((d, self.R)) for d in self.dims]
        lam = np.zeros(self.R)
        _check(lib().adatm_engine_get_factors(self._h, _row_ptrs(mats, C.c_double),
                                              lam.ctypes.data_as(C.POINTER(C.c_double))), "get_factors")
        return mats, lam

    def mttkrp(self, mode):
        out = np.zeros((self.dims[mode], self.R))
        _check(lib().adatm_engine_mttkrp(self._h, mode, out.ctypes.data_as(C.POINTER(C.c_double))),
               "mttkrp")
        return out

    def mttkrp_direct(self, mode):
        out = np.zeros((self.dims[mode], self.R))
        _check(lib().adatm_engine_mttkrp_direct(self._h, mode,
                                                out.ctypes.data_as(C.POINTER(C.c_double))),
               "mttkrp_direct")
        return out

    def memo(self, g, deg):
        nf, _ = self.csf_shape(g)
        gr = self.plan["groups"][g]
        rows = int(nf[gr["begin_imten"] - 1 - deg])
        out = np.zeros((rows, self.R))
        _check(lib().adatm_engine_memo(self._h, g, deg, out.ctypes.data_as(C.POINTER(C.c_double))),
               "memo")
        return out

    def als(self, niters, tol=0.0, graph=True):
        fit = C.c_double(0)
        it = C.c_uint64(0)
        trace = np.zeros(max(1, niters))
        _check(lib().adatm_engine_als(self._h, niters, tol, int(graph), C.byref(fit), C.byref(it),
                                      trace.ctypes.data_as(C.POINTER(C.c_double))), "als")
        return {"fit": fit.value, "iters": it.value, "trace": trace[: it.value].copy()}

    def als_begin(self, graph=True):
        _check(lib().adatm_engine_als_begin(self._h, int(graph)), "als_begin")

    def time_sweeps(self, count):
        ms = C.c_float(0)
        _check(lib().adatm_engine_time_sweeps(self._h, count, C.byref(ms)), "time_sweeps")
        return ms.value

    def time_mttkrp(self, mode, count):
        ms = C.c_float(0)
        _check(lib().adatm_engine_time_mttkrp(self._h, mode, count, C.byref(ms)), "time_mttkrp")
        return ms.value

    def fit(self):
        f = C.c_double(0)
        _check(lib().adatm_engine_fit(self._h, C.byref(f)), "fit")
        return f.value

    def mttkrp_bytes(self, mode):
        b = C.c_double(0)
        _check(lib().adatm_engine_mttkrp_bytes(self._h, mode, C.byref(b)), "mttkrp_bytes")
        return b.value

    def hot_rows(self, mode):
        """Output rows the mode's walk sums per block in shared memory."""
        n = C.c_int(0)
        _check(lib().adatm_engine_hot_rows(self._h, mode, C.byref(n)), "hot_rows")
        return n.value

    def launch_counts(self, mode=0):
        a = C.c_int(0)
        b = C.c_int(0)
        _check(lib().adatm_engine_launch_counts(self._h, mode, C.byref(a), C.byref(b)), "launch_counts")
        return a.value, b.value

    def autotune(self, options=((128, 64), (256, 128), (512, 256), (1024, 512)), sweeps=3):
        """Keep the fastest (chunk_leaf, chunk_rows) of `options` by timing a
        captured sweep of each; returns its index. Initialise the factors
        afterwards."""
        leaf = (C.c_uint32 * len(options))(*[o[0] for o in options])
        rows = (C.c_uint32 * len(options))(*[o[1] for o in options])
        best = C.c_int(0)
        _check(lib().adatm_engine_autotune(self._h, leaf, rows, len(options), sweeps, C.byref(best)),
               "adatm_engine_autotune")
        return best.value

    def set_resident_grid(self, on):
        """Contraction walks as a resident grid claiming chunks (True, the
        default) or one chunk per warp (False, as in a batch)."""
        _check(lib().adatm_engine_set_resident_grid(self._h, int(bool(on))),
               "adatm_engine_set_resident_grid")

    # one shard of a tensor split across ranks (adatm_b200.shard)
    def mttkrp_into(self, mode, dev_ptr):
        """This shard's MTTKRP of `mode` into a device buffer (dims[mode] x ldr FP64)."""
        _check(lib().adatm_engine_mttkrp_into(self._h, mode, C.c_void_p(dev_ptr)),
               "adatm_engine_mttkrp_into")

    def update_from(self, mode, dev_ptr):
        """The mode's update from the summed MTTKRP in a device buffer."""
        _check(lib().adatm_engine_update_from(self._h, mode, C.c_void_p(dev_ptr)),
               "adatm_engine_update_from")

    def fit_step(self):
        f = C.c_double(0)
        _check(lib().adatm_engine_fit_step(self._h, C.byref(f)), "adatm_engine_fit_step")
        return f.value

    def ttnorm(self):
        v = C.c_double(0)
        _check(lib().adatm_engine_ttnorm(self._h, C.byref(v)), "adatm_engine_ttnorm")
        return v.value

    def set_ttnorm(self, v):
        _check(lib().adatm_engine_set_ttnorm(self._h, float(v)), "adatm_engine_set_ttnorm")

    def set_walkers(self, walkers):
        """Walkers per warp in the contraction source loop (1, 2, 4; 0 =
        the default for the rank)."""
        _check(lib().adatm_engine_set_walkers(self._h, int(walkers)), "adatm_engine_set_walkers")

    def set_fold(self, fold):
        """Unstored levels folded into the contraction source loop (0, 1, 2;
        -1 = chosen from each tree's fan-out)."""
        _check(lib().adatm_engine_set_fold(self._h, int(fold)), "adatm_engine_set_fold")

    def set_deterministic(self, on=True):
        """Deterministic accumulation (no float atomics): sweeps repeat bit
        for bit from the same start."""
        _check(lib().adatm_engine_set_deterministic(self._h, int(bool(on))),
               "adatm_engine_set_deterministic")


class BatchSweep:
    """One ALS iteration of every engine in one CUDA graph; the engines must
    stay alive while the batch is used."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._h for e in self.engines])
        h = C.c_void_p()
        _check(lib().adatm_batch_create(arr, len(self.engines), C.byref(h)), "adatm_batch_create")
        self._h = h

    def begin(self):
        _check(lib().adatm_batch_begin(self._h), "adatm_batch_begin")

    def time_sweeps(self, count):
        ms = C.c_float(0)
        _check(lib().adatm_batch_time_sweeps(self._h, count, C.byref(ms)), "adatm_batch_time_sweeps")
        return ms.value

    def kernels(self):
        k = C.c_int(0)
        _check(lib().adatm_batch_kernels(self._h, C.byref(k)), "adatm_batch_kernels")
        return k.value

    def free(self):
        if getattr(self, "_h", None):
            lib().adatm_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def gram_device(A_ptr, rows, R, ldr, G_ptr):
    """G = A^T A (FP64) for a device row matrix; pointers are device addresses
    (e.g. torch tensor .data_ptr())."""
    _check(lib().adatm_gram(C.c_void_p(A_ptr), rows, R, ldr, C.c_void_p(G_ptr)), "adatm_gram")
