"""The C-ABI library loads and exports every function the public headers
declare; host-only entry points (no GPU needed) match the oracle."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import adatm_b200 as A
import oracle as O
from conftest import ROOT, golden_cases, load_golden


def declared_functions():
    names = set()
    for h in ("splatt.h", "adatm_b200.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol():
    A.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", A.library_path()], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines()}
    declared = declared_functions()
    assert len(declared) >= 50
    missing = [n for n in declared if n not in exported]
    assert not missing, missing


def test_default_opts_layout():
    o = A.splatt_default_opts()
    assert len(o) == A.OPT_NOPTIONS
    assert o[A.OPT_CSF_ALLOC] == A.ADAPTIVE_TIME_EFFICIENT
    assert o[A.OPT_TILE] == 0


@pytest.mark.parametrize("N", [3, 4, 5, 6, 7, 8])
def test_product_order_matches_reference_definition(N):
    po = A.decide_product_order(N)
    for m in range(N):
        for k in range(2 * N):
            expect = 1 if (k < N and k > m) or (k >= N and k - N < m) else 0
            assert po[m, k] == expect


@pytest.mark.parametrize("name", golden_cases())
def test_use_csfs_host_logic(name):
    d = load_golden(name)
    uc, ut = A.decide_use_csfs(d["N"], d["groups"])
    np.testing.assert_array_equal(uc, d["use_csfs"])
    np.testing.assert_array_equal(ut, d["use_tags"])


@pytest.mark.parametrize("dims", [[30, 40, 50], [40, 35, 25, 20], [20, 20, 20, 20], [14, 12, 10, 9, 8],
                                  [6, 7, 5, 8, 6, 7], [5, 6, 4, 5, 6, 4, 5], [4, 5, 4, 3, 5, 4, 3, 4]])
def test_candidate_configs_host_logic(dims):
    """decide_candidate_configs through the C ABI (no GPU work) equals the
    oracle's enumeration: group counts, memo modes, begin/n_imten, o_opt."""
    from adatm_b200._native import GroupProperties
    N = len(dims)
    inds = np.zeros((N, 1), dtype=np.uint64)
    t = A._SpTensor(inds, np.ones(1), dims)
    po = A._row_ptrs([np.zeros(2 * N, dtype=np.uint64) for _ in range(N)])

    class Cfg(C.Structure):
        _fields_ = [("n_grp", C.c_uint64), ("grp_prop", C.POINTER(GroupProperties)),
                    ("pspace", C.c_size_t), ("pops", C.c_size_t), ("ptime", C.c_double),
                    ("rtime", C.c_double)]
    out = C.POINTER(Cfg)()
    n = A.lib().decide_candidate_configs(C.byref(t.tt), po, C.byref(out))
    ref = O.candidate_configs(dims)
    assert n == len(ref)
    for c in range(n):
        got = A._groups_from_c(out[c].grp_prop, out[c].n_grp, N)
        assert got == ref[c]["grp"]


def test_errors_are_reported_not_raised_in_c():
    # an unknown splatt_csf pointer is rejected with SPLATT_ERROR_BADINPUT
    bogus = (A.SplattCsf * 1)()
    out = np.zeros((4, 2))
    mats = [np.zeros((4, 2))] * 3
    rc = A.lib().splatt_mttkrp(0, 2, bogus, A._row_ptrs(mats, C.c_double),
                               out.ctypes.data_as(C.POINTER(C.c_double)),
                               A.splatt_default_opts().ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == A.SPLATT_ERROR_BADINPUT
    assert "not built by this library" in A._native.last_error()


PRINT_WORKER = r"""
import ctypes as C, sys
sys.path.insert(0, {root!r})
import numpy as np
import adatm_b200 as A
from adatm_b200 import _native as N
L = A.lib()
groups = [{{"memo_mode": 0, "begin_imten": 2, "n_imten": 1, "o_opt": [0, 1, 3, 2]}},
          {{"memo_mode": 2, "begin_imten": 2, "n_imten": 1, "o_opt": [2, 3, 0, 1]}}]
ga = A._GroupArray(groups, 4)
L.print_group_properties.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_char_p]
L.print_group_properties(C.cast(ga.arr, C.c_void_p), 2, 4, b"Optimal grp_prop")
pt = N.CsfSparsity()
pt.vals = (C.c_double * 1)(1.0)
ct = N.SplattCsf(nnz=123, nmodes=4, which_tile=0, ntiles=1)
for m, (d, p) in enumerate(zip([50, 40, 30, 20], [0, 1, 3, 2])):
    ct.dims[m] = d; ct.dim_perm[m] = p; ct.tile_dims[m] = 1
ct.pt = C.pointer(pt)
L.stats_csf_adaptive.argtypes = [C.c_void_p, C.c_uint64]
L.stats_csf_adaptive(C.cast(C.pointer(ct), C.c_void_p), 1)
L.iprint_array.argtypes = [C.c_void_p, C.c_uint64, C.c_char_p]
a = np.array([0, 0, 1, 1], dtype=np.uint64)
L.iprint_array(a.ctypes.data_as(C.c_void_p), 4, b"use_csfs")
"""


def test_report_lines_have_the_reference_format():
    """print_group_properties (adatm_debug.c:58-72), stats_csf_adaptive
    (adatm_stats.c:19-67) and iprint_array (adatm_debug.c:5-15) print the
    reference's text (host only, no GPU)."""
    out = subprocess.run([__import__("sys").executable, "-c", PRINT_WORKER.format(root=ROOT)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    want = ("====== Optimal grp_prop =======\n"
            "[memo_mode, begin_imten, n_imten, o_opt]\n"
            "0, 2, 1, \no_opt: \n 0 1 3 2\n"
            "2, 2, 1, \no_opt: \n 2 3 0 1\n\n"
            "CSF-0\nnmodes: 4 nnz: 123\ndims: 50x40x30x20 (0->1->3->2)\n"
            "ntiles: 1 tile dims: 1x1x1x1  empty: 0 (0.0%)\n"
            "use_csfs: \n 0 0 1 1\n")
    assert out.stdout == want, out.stdout
