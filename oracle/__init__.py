"""CPU FP64 oracle for AdaTM's memoized MTTKRP sequence and CP-ALS sweep.

TEST INFRASTRUCTURE ONLY. tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py use this package as
the checker. The product (``adatm_b200``) never imports it.

Two native libraries sit behind it:

* ``liboracle.so`` -- ``adatm_oracle.c``, the restatement of the reference
  algorithm (every function cites the reference file:line it follows);
* ``_ref/libadatm_ref.so`` -- the reference's own AdaTM C files compiled
  against a SPLATT stand-in (``shim/``), used to pin the restatement. It is
  built only where the reference checkout exists and then travels as a
  prebuilt file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAXN = 16
SLIMIT = 90e9

u64 = C.c_uint64
P_u64 = C.POINTER(u64)
P_f64 = C.POINTER(C.c_double)


class OrcCsf(C.Structure):
    _fields_ = [
        ("nmodes", C.c_int),
        ("nnz", u64),
        ("dims", u64 * MAXN),
        ("dim_perm", u64 * MAXN),
        ("nfibs", u64 * MAXN),
        ("fptr", P_u64 * MAXN),
        ("fids", P_u64 * MAXN),
        ("root_ids", P_u64),
        ("vals", P_f64),
    ]


class OrcGrp(C.Structure):
    _fields_ = [
        ("memo_mode", u64),
        ("begin_imten", u64),
        ("n_imten", u64),
        ("o_opt", u64 * MAXN),
    ]


class OrcConfig(C.Structure):
    _fields_ = [
        ("n_grp", u64),
        ("grp", OrcGrp * MAXN),
        ("pspace", u64),
        ("pops", u64),
    ]


_lib = None
_ref = None


def build(ref_dir: str | None = None) -> None:
    """Compile liboracle.so and, when a reference checkout is given (the
    argument, else the ADATM_REFERENCE_DIR environment variable) and exists,
    _ref/libadatm_ref.so from its sources."""
    subprocess.check_call(["make", "-s", "liboracle.so"], cwd=HERE)
    ref = ref_dir or os.environ.get("ADATM_REFERENCE_DIR")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.check_call(["make", "-s", "ref", f"REF={ref}"], cwd=HERE)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "liboracle.so"], cwd=HERE)
        L = C.CDLL(path)
        L.orc_sort_order.argtypes = [C.c_int, u64, P_u64, P_u64, P_u64, P_u64]
        L.orc_coo_clean.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64]
        L.orc_coo_clean.restype = u64
        L.orc_csf_build.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64, P_u64]
        L.orc_csf_build.restype = C.POINTER(OrcCsf)
        L.orc_csf_free.argtypes = [C.POINTER(OrcCsf)]
        L.orc_count_nfibs.argtypes = [C.c_int, u64, P_u64, P_u64, P_u64, P_u64]
        L.orc_splatt_perm.argtypes = [C.c_int, P_u64, C.c_int, u64, P_u64]
        L.orc_candidate_configs.argtypes = [C.c_int, P_u64, C.POINTER(OrcConfig), C.c_int]
        L.orc_candidate_configs.restype = C.c_int
        L.orc_predict_candidates.argtypes = [C.c_int, u64, P_u64, P_u64, u64,
                                             C.POINTER(OrcConfig), C.c_int]
        L.orc_choose_config.argtypes = [C.POINTER(OrcConfig), C.c_int, C.c_int, C.c_double]
        L.orc_choose_config.restype = C.c_int
        L.orc_plan.argtypes = [C.c_int, u64, P_u64, P_u64, u64, C.c_int,
                               C.POINTER(OrcGrp), C.POINTER(OrcConfig), C.POINTER(C.c_int)]
        L.orc_plan.restype = u64
        L.orc_decide_use_csfs.argtypes = [C.c_int, C.POINTER(OrcGrp), u64, u64, P_u64, P_u64]
        L.orc_pair_sort.argtypes = [P_u64, P_u64, u64]
        L.orc_model_build.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64, u64, u64,
                                      C.POINTER(OrcGrp)]
        L.orc_model_build.restype = C.c_void_p
        L.orc_model_free.argtypes = [C.c_void_p]
        L.orc_mttkrp_adaptive.argtypes = [C.c_void_p, C.POINTER(P_f64), u64, P_f64]
        L.orc_mttkrp_csf.argtypes = [C.POINTER(OrcCsf), C.POINTER(P_f64), u64, u64, P_f64]
        L.orc_factor_init.argtypes = [u64, u64, u64, u64, P_f64]
        L.orc_cpd_als.argtypes = [C.c_void_p, C.POINTER(C.POINTER(OrcCsf)), u64,
                                  C.POINTER(P_f64), P_f64, u64, C.c_double, P_f64, P_u64]
        L.orc_cpd_als.restype = C.c_double
        L.orc_generate.argtypes = [C.c_int, P_u64, u64, P_f64, C.c_int, C.c_double, C.c_double,
                                   u64, P_u64, P_f64]
        L.orc_mttkrp_coo.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64, C.POINTER(P_f64), u64, u64,
                                     P_f64]
        L.orc_cpd_als_coo.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64, u64, C.POINTER(P_f64),
                                      P_f64, u64, C.c_double, P_f64, P_u64]
        L.orc_cpd_als_coo.restype = C.c_double
        L.orc_threads.argtypes = [C.c_int]
        L.orc_threads.restype = C.c_int
        _lib = L
    return _lib


def _u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(P_u64)


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(P_f64)


def _mats_ptrs(mats):
    keep = [np.ascontiguousarray(m, dtype=np.float64) for m in mats]
    arr = (P_f64 * len(keep))(*[k.ctypes.data_as(P_f64) for k in keep])
    return keep, arr


# --------------------------------------------------------------------------
# COO and CSF
# --------------------------------------------------------------------------

def sort_order(inds, dims, perm):
    """Lexicographic order of the nonzeros by perm (stable)."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    p, pp = _u64(perm)
    i, ip = _u64(inds)
    out = np.zeros(nnz, dtype=np.uint64)
    lib().orc_sort_order(N, nnz, dp, ip, pp, out.ctypes.data_as(P_u64))
    return out


def coo_clean(inds, vals, dims):
    """Sum duplicates in input order and compact empty slices of every mode.
    Returns (inds[N, nnz'], vals[nnz'], dims')."""
    inds = np.array(inds, dtype=np.uint64, order="C", copy=True)
    vals = np.array(vals, dtype=np.float64, copy=True)
    dims = np.array(dims, dtype=np.uint64, copy=True)
    N, nnz = inds.shape
    n = lib().orc_coo_clean(N, nnz, dims.ctypes.data_as(P_u64),
                            inds.ctypes.data_as(P_u64), vals.ctypes.data_as(P_f64))
    flat = inds.reshape(-1)[: N * n].reshape(N, n).copy()
    return flat, vals[:n].copy(), dims


def _csf_to_dict(p):
    c = p.contents
    N = c.nmodes
    nnz = c.nnz
    out = {"nmodes": N, "nnz": nnz,
           "dims": np.array(c.dims[:N], dtype=np.uint64),
           "dim_perm": np.array(c.dim_perm[:N], dtype=np.uint64),
           "nfibs": np.array(c.nfibs[:N], dtype=np.uint64),
           "fptr": [], "fids": []}
    for l in range(N):
        F = c.nfibs[l]
        if l < N - 1 and c.fptr[l]:
            out["fptr"].append(np.ctypeslib.as_array(c.fptr[l], shape=(F + 1,)).copy())
        else:
            out["fptr"].append(None)
        if l >= 1 and c.fids[l] and F > 0:
            out["fids"].append(np.ctypeslib.as_array(c.fids[l], shape=(F,)).copy())
        elif l >= 1:
            out["fids"].append(np.zeros(0, dtype=np.uint64))
        else:
            out["fids"].append(None)
    F0 = c.nfibs[0]
    out["root_ids"] = (np.ctypeslib.as_array(c.root_ids, shape=(F0,)).copy()
                       if (c.root_ids and F0 > 0) else np.zeros(0, dtype=np.uint64))
    out["vals"] = (np.ctypeslib.as_array(c.vals, shape=(nnz,)).copy()
                   if nnz > 0 else np.zeros(0))
    return out


def csf_build(inds, vals, dims, perm):
    """CSF arrays of the tensor in dim_perm order, reference layout."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    v, vp = _f64(vals)
    p, pp = _u64(perm)
    ptr = lib().orc_csf_build(N, nnz, dp, inds.ctypes.data_as(P_u64), vp, pp)
    try:
        return _csf_to_dict(ptr)
    finally:
        lib().orc_csf_free(ptr)


def count_nfibs(inds, dims, o_opt):
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    o, op = _u64(o_opt)
    out = np.zeros(N, dtype=np.uint64)
    lib().orc_count_nfibs(N, nnz, dp, inds.ctypes.data_as(P_u64), op, out.ctypes.data_as(P_u64))
    return out


def splatt_perm(dims, which, root=0):
    d, dp = _u64(dims)
    out = np.zeros(len(dims), dtype=np.uint64)
    lib().orc_splatt_perm(len(dims), dp, which, root, out.ctypes.data_as(P_u64))
    return out


# --------------------------------------------------------------------------
# planner
# --------------------------------------------------------------------------

def _grp_to_py(g, N):
    return {"memo_mode": int(g.memo_mode), "begin_imten": int(g.begin_imten),
            "n_imten": int(g.n_imten), "o_opt": [int(x) for x in g.o_opt[:N]]}


def _grp_from_py(groups, N):
    arr = (OrcGrp * MAXN)()
    for gi, g in enumerate(groups):
        arr[gi].memo_mode = g["memo_mode"]
        arr[gi].begin_imten = g["begin_imten"]
        arr[gi].n_imten = g["n_imten"]
        for m in range(N):
            arr[gi].o_opt[m] = g["o_opt"][m]
    return arr


def candidate_configs(dims):
    N = len(dims)
    d, dp = _u64(dims)
    arr = (OrcConfig * (4 * MAXN))()
    n = lib().orc_candidate_configs(N, dp, arr, 4 * MAXN)
    return [{"n_grp": int(arr[c].n_grp),
             "grp": [_grp_to_py(arr[c].grp[g], N) for g in range(arr[c].n_grp)]}
            for c in range(n)]


def plan(inds, dims, nfactors, strategy=1):
    """Analytic memo plan (decide_parameters_auto). Returns
    (groups, configs-with-predictions, chosen position)."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    grp = (OrcGrp * MAXN)()
    cfgs = (OrcConfig * (4 * MAXN))()
    nc = C.c_int(0)
    n_grp = lib().orc_plan(N, nnz, dp, inds.ctypes.data_as(P_u64), nfactors, strategy,
                           grp, cfgs, C.byref(nc))
    configs = [{"n_grp": int(cfgs[c].n_grp),
                "grp": [_grp_to_py(cfgs[c].grp[g], N) for g in range(cfgs[c].n_grp)],
                "pspace": int(cfgs[c].pspace), "pops": int(cfgs[c].pops)}
               for c in range(nc.value)]
    return [_grp_to_py(grp[g], N) for g in range(n_grp)], configs


def decide_use_csfs(nmodes, groups, n_csf=None):
    arr = _grp_from_py(groups, nmodes)
    uc = np.zeros(nmodes, dtype=np.uint64)
    ut = np.zeros(nmodes, dtype=np.uint64)
    lib().orc_decide_use_csfs(nmodes, arr, len(groups),
                              len(groups) if n_csf is None else n_csf,
                              uc.ctypes.data_as(P_u64), ut.ctypes.data_as(P_u64))
    return uc, ut


def pair_sort(xs, ys):
    x, xp = _u64(xs)
    y, yp = _u64(ys)
    x = x.copy()
    y = y.copy()
    lib().orc_pair_sort(x.ctypes.data_as(P_u64), y.ctypes.data_as(P_u64), len(x))
    return x, y


# --------------------------------------------------------------------------
# MTTKRP and CP-ALS
# --------------------------------------------------------------------------

def factor_init(seed, mode, rows, nfactors):
    out = np.zeros((rows, nfactors), dtype=np.float64)
    lib().orc_factor_init(seed, mode, rows, nfactors, out.ctypes.data_as(P_f64))
    return out


def init_factors(dims, nfactors, seed=0):
    return [factor_init(seed, m, int(d), nfactors) for m, d in enumerate(dims)]


class Model:
    """Memoized model: TIME_EFFICIENT CSFs per group plus memo trees."""

    def __init__(self, inds, vals, dims, nfactors, groups):
        inds = np.ascontiguousarray(inds, dtype=np.uint64)
        self.N, self.nnz = inds.shape
        self.dims = [int(x) for x in dims]
        self.R = int(nfactors)
        self.groups = groups
        d, dp = _u64(dims)
        v, vp = _f64(vals)
        self._h = lib().orc_model_build(self.N, self.nnz, dp, inds.ctypes.data_as(P_u64), vp,
                                        self.R, len(groups), _grp_from_py(groups, self.N))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_model_free(self._h)
            self._h = None

    def mttkrp(self, mats, mode):
        keep, arr = _mats_ptrs(mats)
        out = np.zeros((self.dims[mode], self.R), dtype=np.float64)
        lib().orc_mttkrp_adaptive(self._h, arr, mode, out.ctypes.data_as(P_f64))
        return out

    def cpd_als(self, mats, niters, tol):
        return _cpd(self._h, None, self.R, mats, niters, tol)


def mttkrp_csf(inds, vals, dims, perm, mats, mode, nfactors):
    """Plain CSF MTTKRP of `mode` on a tree in `perm` order."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    v, vp = _f64(vals)
    p, pp = _u64(perm)
    ptr = lib().orc_csf_build(N, nnz, dp, inds.ctypes.data_as(P_u64), vp, pp)
    try:
        keep, arr = _mats_ptrs(mats)
        out = np.zeros((int(dims[mode]), nfactors), dtype=np.float64)
        lib().orc_mttkrp_csf(ptr, arr, mode, nfactors, out.ctypes.data_as(P_f64))
        return out
    finally:
        lib().orc_csf_free(ptr)


def _cpd(handle, plain, R, mats, niters, tol):
    keep, arr = _mats_ptrs([m.copy() for m in mats])
    lam = np.zeros(R, dtype=np.float64)
    trace = np.zeros(max(1, niters), dtype=np.float64)
    done = u64(0)
    fit = lib().orc_cpd_als(handle, plain, R, arr, lam.ctypes.data_as(P_f64), niters, tol,
                            trace.ctypes.data_as(P_f64), C.byref(done))
    return {"fit": fit, "lambda": lam, "factors": keep,
            "trace": trace[: done.value].copy(), "iters": int(done.value)}


def threads(n=0):
    """OpenMP threads of the parallel oracle paths (n > 0 sets them)."""
    return int(lib().orc_threads(int(n)))


def generate(dims, nnz, alpha=None, value_kind=0, mu=0.0, sigma=1.0, seed=0, clean=True):
    """The seeded synthetic tensor of the library's device generator, made on
    the host: (inds N x nnz uint64, vals, dims). With clean, duplicates are
    summed and empty slices compacted (orc_coo_clean), as the library does
    after generating."""
    N = len(dims)
    d = np.ascontiguousarray(dims, dtype=np.uint64).copy()
    a = np.zeros(N) if alpha is None else np.ascontiguousarray(
        [alpha] * N if np.isscalar(alpha) else alpha, dtype=np.float64)
    inds = np.empty((N, int(nnz)), dtype=np.uint64)
    vals = np.empty(int(nnz), dtype=np.float64)
    lib().orc_generate(N, d.ctypes.data_as(P_u64), int(nnz), a.ctypes.data_as(P_f64), int(value_kind),
                       float(mu), float(sigma), int(seed), inds.ctypes.data_as(P_u64),
                       vals.ctypes.data_as(P_f64))
    if not clean:
        return inds, vals, [int(x) for x in d]
    # clean in place (the arrays are ours): no copies of a large draw
    n = lib().orc_coo_clean(N, int(nnz), d.ctypes.data_as(P_u64), inds.ctypes.data_as(P_u64),
                            vals.ctypes.data_as(P_f64))
    flat = inds.reshape(-1)[: N * n].reshape(N, n)
    return flat, vals[:n], [int(x) for x in d]


def mttkrp_coo(inds, vals, dims, mats, mode, nfactors):
    """FP64 MTTKRP of `mode` from the coordinates (OpenMP)."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    v, vp = _f64(vals)
    keep, arr = _mats_ptrs(mats)
    out = np.zeros((int(dims[mode]), nfactors), dtype=np.float64)
    lib().orc_mttkrp_coo(N, nnz, dp, inds.ctypes.data_as(P_u64), vp, arr, mode, nfactors,
                         out.ctypes.data_as(P_f64))
    return out


def cpd_als_coo(inds, vals, dims, nfactors, mats, niters, tol):
    """CP-ALS with the FP64 COO MTTKRP (the same ALS steps as Model.cpd_als)."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    v, vp = _f64(vals)
    keep, arr = _mats_ptrs([np.array(m, dtype=np.float64, copy=True) for m in mats])
    lam = np.zeros(nfactors, dtype=np.float64)
    trace = np.zeros(max(1, niters), dtype=np.float64)
    done = u64(0)
    fit = lib().orc_cpd_als_coo(N, nnz, dp, inds.ctypes.data_as(P_u64), vp, nfactors, arr,
                                lam.ctypes.data_as(P_f64), niters, tol,
                                trace.ctypes.data_as(P_f64), C.byref(done))
    return {"fit": fit, "lambda": lam, "factors": keep,
            "trace": trace[: done.value].copy(), "iters": int(done.value)}


def cpd_als_plain(inds, vals, dims, nfactors, mats, niters, tol):
    """CP-ALS with one plain CSF per mode (SPLATT_CSF_ALLMODE)."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    v, vp = _f64(vals)
    ptrs = []
    for m in range(N):
        p, pp = _u64(splatt_perm(dims, 1, m))
        ptrs.append(lib().orc_csf_build(N, nnz, dp, inds.ctypes.data_as(P_u64), vp, pp))
    try:
        arr = (C.POINTER(OrcCsf) * N)(*ptrs)
        return _cpd(None, arr, nfactors, mats, niters, tol)
    finally:
        for p in ptrs:
            lib().orc_csf_free(p)


# --------------------------------------------------------------------------
# the reference's own code (oracle/_ref)
# --------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libadatm_ref.so"))


def _host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = set(line.split(":", 1)[1].split())
                    return {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= fl
    except OSError:
        pass
    return False


def ref_build_arch() -> str:
    """The build of the reference's code this host loads: x86-64-v4 (AVX-512)
    where the CPU has it and that build exists, else x86-64-v3."""
    v4 = os.path.join(HERE, "_ref", "libadatm_ref_v4.so")
    return "x86-64-v4" if _host_has_avx512() and os.path.exists(v4) else "x86-64-v3"


def ref():
    global _ref
    if _ref is None:
        name = "libadatm_ref_v4.so" if ref_build_arch() == "x86-64-v4" else "libadatm_ref.so"
        L = C.CDLL(os.path.join(HERE, "_ref", name))
        L.ref_plan.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64, u64, P_u64]
        L.ref_plan.restype = u64
        L.ref_build.argtypes = [C.c_int, u64, P_u64, P_u64, P_f64, u64, P_u64, C.c_int]
        L.ref_build.restype = C.c_void_p
        L.ref_n_csf.argtypes = [C.c_void_p]
        L.ref_n_csf.restype = u64
        L.ref_use.argtypes = [C.c_void_p, P_u64, P_u64]
        L.ref_set_use.argtypes = [C.c_void_p, P_u64, P_u64]
        L.ref_csf_shape.argtypes = [C.c_void_p, C.c_int, P_u64, P_u64]
        L.ref_csf_array.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, P_u64]
        L.ref_csf_array.restype = C.c_int
        L.ref_csf_vals.argtypes = [C.c_void_p, C.c_int, P_f64]
        L.ref_memo_shape.argtypes = [C.c_void_p, C.c_int, C.c_int, P_u64]
        L.ref_memo_vals.argtypes = [C.c_void_p, C.c_int, C.c_int, P_f64]
        L.ref_mttkrp.argtypes = [C.c_void_p, C.POINTER(P_f64), u64, P_f64, C.c_int]
        L.ref_mttkrp_sequence.argtypes = [C.c_void_p, C.c_int]
        L.ref_mttkrp_sequence.restype = C.c_double
        L.ref_cpd.argtypes = [C.c_void_p, C.POINTER(P_f64), P_f64, u64, C.c_double, C.c_int]
        L.ref_cpd.restype = C.c_double
        L.ref_free.argtypes = [C.c_void_p]
        _ref = L
    return _ref


def _pack_plan(groups, N):
    flat = [len(groups)]
    for g in groups:
        flat += [g["memo_mode"], g["begin_imten"], g["n_imten"]] + list(g["o_opt"][:N])
    return np.array(flat, dtype=np.uint64)


def ref_plan(inds, vals, dims, nfactors):
    """The reference's decide_parameters_auto; None for N == 3."""
    inds = np.ascontiguousarray(inds, dtype=np.uint64)
    N, nnz = inds.shape
    d, dp = _u64(dims)
    v, vp = _f64(vals)
    out = np.zeros(1 + MAXN * (3 + N), dtype=np.uint64)
    n = ref().ref_plan(N, nnz, dp, inds.ctypes.data_as(P_u64), vp, nfactors,
                       out.ctypes.data_as(P_u64))
    if n == 0:
        return None
    groups = []
    for g in range(n):
        o = out[1 + g * (3 + N): 1 + (g + 1) * (3 + N)]
        groups.append({"memo_mode": int(o[0]), "begin_imten": int(o[1]),
                       "n_imten": int(o[2]), "o_opt": [int(x) for x in o[3:3 + N]]})
    return groups


class RefModel:
    """The reference's csf_alloc_adaptive/rcsf_alloc_adaptive/mttkrp and
    cpd_als_iterate_adaptive on one plan."""

    def __init__(self, inds, vals, dims, nfactors, groups, nthreads=1):
        inds = np.ascontiguousarray(inds, dtype=np.uint64)
        self.N, self.nnz = inds.shape
        self.dims = [int(x) for x in dims]
        self.R = int(nfactors)
        d, dp = _u64(dims)
        v, vp = _f64(vals)
        pk, pkp = _u64(_pack_plan(groups, self.N))
        self._h = ref().ref_build(self.N, self.nnz, dp, inds.ctypes.data_as(P_u64), vp,
                                  self.R, pkp, nthreads)

    def __del__(self):
        if getattr(self, "_h", None):
            ref().ref_free(self._h)
            self._h = None

    def n_csf(self):
        return int(ref().ref_n_csf(self._h))

    def use(self):
        uc = np.zeros(self.N, dtype=np.uint64)
        ut = np.zeros(self.N, dtype=np.uint64)
        ref().ref_use(self._h, uc.ctypes.data_as(P_u64), ut.ctypes.data_as(P_u64))
        return uc, ut

    def set_use(self, use_csfs, use_tags):
        """Per-mode trees and tags passed to the reference from now on."""
        uc, ucp = _u64(use_csfs)
        ut, utp = _u64(use_tags)
        ref().ref_set_use(self._h, ucp, utp)

    def csf(self, g):
        N = self.N
        nf = np.zeros(N, dtype=np.uint64)
        dpm = np.zeros(N, dtype=np.uint64)
        ref().ref_csf_shape(self._h, g, nf.ctypes.data_as(P_u64), dpm.ctypes.data_as(P_u64))
        out = {"nfibs": nf, "dim_perm": dpm, "fptr": [], "fids": []}
        for l in range(N):
            if l < N - 1:
                a = np.zeros(int(nf[l]) + 1, dtype=np.uint64)
                ok = ref().ref_csf_array(self._h, g, l, 0, a.ctypes.data_as(P_u64))
                out["fptr"].append(a if ok else None)
            else:
                out["fptr"].append(None)
            a = np.zeros(max(1, int(nf[l])), dtype=np.uint64)
            ok = ref().ref_csf_array(self._h, g, l, 1, a.ctypes.data_as(P_u64))
            out["fids"].append(a[: int(nf[l])] if ok else None)
        vals = np.zeros(max(1, self.nnz))
        ref().ref_csf_vals(self._h, g, vals.ctypes.data_as(P_f64))
        out["vals"] = vals[: self.nnz]
        return out

    def memo_shape(self, j, deg):
        o = np.zeros(4, dtype=np.uint64)
        ref().ref_memo_shape(self._h, j, deg, o.ctypes.data_as(P_u64))
        return [int(x) for x in o]

    def mttkrp(self, mats, mode, zero_memo=True):
        keep, arr = _mats_ptrs(mats)
        out = np.zeros((self.dims[mode], self.R), dtype=np.float64)
        ref().ref_mttkrp(self._h, arr, mode, out.ctypes.data_as(P_f64), int(zero_memo))
        return out

    def cpd_als(self, mats, niters, tol, zero_memo=True):
        keep, arr = _mats_ptrs([m.copy() for m in mats])
        lam = np.zeros(self.R)
        fit = ref().ref_cpd(self._h, arr, lam.ctypes.data_as(P_f64), niters, tol,
                            int(zero_memo))
        return {"fit": fit, "lambda": lam, "factors": keep}

    def sequence_seconds(self, mats, zero_memo=True):
        keep, arr = _mats_ptrs(mats)
        out = np.zeros((max(self.dims), self.R))
        ref().ref_mttkrp(self._h, arr, 0, out.ctypes.data_as(P_f64), int(zero_memo))
        return ref().ref_mttkrp_sequence(self._h, int(zero_memo))
